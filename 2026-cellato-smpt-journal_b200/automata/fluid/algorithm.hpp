// HPP lattice gas: four particle directions per cell, head-on collisions turn
// by 90 degrees (rule of the reference src/fluid/algorithm.hpp:11-60).
#ifndef FLUID_ALGORITHM_HPP
#define FLUID_ALGORITHM_HPP

#include "core/ast.hpp"

namespace fluid {
using namespace cellato::ast;

using fluid_cell_state = int;

constexpr int TOP_bit = 0, TOP = 1 << TOP_bit;
constexpr int BOTTOM_bit = 1, BOTTOM = 1 << BOTTOM_bit;
constexpr int LEFT_bit = 2, LEFT = 1 << LEFT_bit;
constexpr int RIGHT_bit = 3, RIGHT = 1 << RIGHT_bit;

using above = neighbor_at<0, -1>;
using below = neighbor_at<0, 1>;
using to_left = neighbor_at<-1, 0>;
using to_right = neighbor_at<1, 0>;

// particles streaming into this cell
using vertical_in = p<p<above, bit_and_, constant<TOP>>, bit_or_, p<below, bit_and_, constant<BOTTOM>>>;
using horizontal_in = p<p<to_left, bit_and_, constant<LEFT>>, bit_or_, p<to_right, bit_and_, constant<RIGHT>>>;

using head_on_vertical = p<has_bit_set<above, TOP_bit>, bit_and_, has_bit_set<below, BOTTOM_bit>>;
using head_on_horizontal = p<has_bit_set<to_left, LEFT_bit>, bit_and_, has_bit_set<to_right, RIGHT_bit>>;

using only_vertical_collision = p<head_on_vertical, bit_and_, p<horizontal_in, equals, constant<0>>>;
using only_horizontal_collision = p<head_on_horizontal, bit_and_, p<vertical_in, equals, constant<0>>>;

using vertical_out = if_<only_vertical_collision>::then_<state_constant<LEFT | RIGHT>>::else_<vertical_in>;
using horizontal_out = if_<only_horizontal_collision>::then_<state_constant<TOP | BOTTOM>>::else_<horizontal_in>;

using fluid_algorithm = p<vertical_out, bit_or_, horizontal_out>;
}  // namespace fluid

#endif
