// Cyclic cellular automaton with 32 states: a cell advances when any Moore
// neighbour holds its successor (rule of the reference src/cyclic/algorithm.hpp:11-23).
#ifndef CYCLIC_ALGORITHM_HPP
#define CYCLIC_ALGORITHM_HPP

#include "core/ast.hpp"

namespace cyclic {
using namespace cellato::ast;

using cyclic_cell_state = int;

constexpr int BITS = 5;
constexpr int STATES = 1 << BITS;

using successor = p<p<current_state, plus, constant<1>>, modulo, constant<STATES>>;
using successor_nearby = p<count_neighbors<successor, moore_8_neighbors>, greater_than, constant<0>>;

using cyclic_algorithm = if_<successor_nearby>::then_<successor>::else_<current_state>;
}  // namespace cyclic

#endif
