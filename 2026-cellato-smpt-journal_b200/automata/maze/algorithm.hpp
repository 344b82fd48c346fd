// Maze, B3/S12345 (rule of the reference src/maze/algorithm.hpp:29-35).
#ifndef MAZE_ALGORITHM_HPP
#define MAZE_ALGORITHM_HPP

#include "core/ast.hpp"

namespace maze {
using namespace cellato::ast;

enum class maze_cell_state { empty, wall };

using empty = state_constant<maze_cell_state::empty>;
using wall = state_constant<maze_cell_state::wall>;

using walls = count_neighbors<wall, moore_8_neighbors>;

using maze_algorithm =
    if_<p<walls, equals, constant<3>>>::then_<wall>
    ::elif_<p<p<current_state, equals, wall>, and_, p<walls, less_than, constant<6>>>>::then_<wall>
    ::else_<empty>;
}  // namespace maze

#endif
