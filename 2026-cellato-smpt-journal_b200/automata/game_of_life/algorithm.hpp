// Conway's Game of Life, B3/S23 on the Moore neighbourhood
// (rule of the reference src/game_of_life/algorithm.hpp:35-49).
#ifndef GAME_OF_LIFE_ALGORITHM_HPP
#define GAME_OF_LIFE_ALGORITHM_HPP

#include "core/ast.hpp"

namespace game_of_life {
using namespace cellato::ast;

enum class gol_cell_state { dead, alive };

using alive = state_constant<gol_cell_state::alive>;
using dead = state_constant<gol_cell_state::dead>;

using live_neighbours = count_neighbors<alive, moore_8_neighbors>;
using born = p<live_neighbours, equals, constant<3>>;
using survives = p<p<live_neighbours, equals, constant<2>>, or_, born>;

using gol_algorithm =
    if_<p<current_state, equals, alive>>::then_<
        if_<survives>::then_<alive>::else_<dead>
    >::else_<
        if_<born>::then_<alive>::else_<dead>
    >;
}  // namespace game_of_life

#endif
