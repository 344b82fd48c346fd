// Critters, a reversible Margolus-block rule
// (rule of the reference src/critters/algorithm.hpp:16-31).
#ifndef CRITTERS_ALGORITHM_HPP
#define CRITTERS_ALGORITHM_HPP

#include "core/ast.hpp"

namespace critters {
using namespace cellato::ast;

enum class critters_cell_state { dead, alive };

using dead = state_constant<critters_cell_state::dead>;
using alive = state_constant<critters_cell_state::alive>;

using block_alive = count_neighbors<alive, margolus_alternating_neighborhood>;

using flip_opposite = if_<p<margolus_180_neighbor, equals, alive>>::then_<dead>::else_<alive>;
using flip_self = if_<p<current_state, equals, alive>>::then_<dead>::else_<alive>;

using critters_algorithm =
    if_<p<block_alive, equals, constant<3>>>::then_<flip_opposite>
    ::elif_<p<block_alive, equals, constant<2>>>::then_<current_state>
    ::else_<flip_self>;
}  // namespace critters

#endif
