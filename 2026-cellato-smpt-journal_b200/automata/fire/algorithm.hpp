// Forest fire on the von Neumann neighbourhood
// (rule of the reference src/fire/algorithm.hpp:39-57).
#ifndef FOREST_FIRE_ALGORITHM_HPP
#define FOREST_FIRE_ALGORITHM_HPP

#include "core/ast.hpp"

namespace fire {
using namespace cellato::ast;

enum class fire_cell_state { empty, tree, ash, fire };

using empty = state_constant<fire_cell_state::empty>;
using tree = state_constant<fire_cell_state::tree>;
using ash = state_constant<fire_cell_state::ash>;
using fire = state_constant<fire_cell_state::fire>;

using burning_neighbour = p<count_neighbors<fire, von_neumann_4_neighbors>, greater_than, constant<0>>;

using fire_algorithm =
    if_<p<current_state, equals, fire>>::then_<ash>
    ::elif_<p<current_state, equals, ash>>::then_<
        if_<burning_neighbour>::then_<ash>::else_<empty>
    >::elif_<p<current_state, equals, tree>>::then_<
        if_<burning_neighbour>::then_<fire>::else_<tree>
    >::else_<empty>;
}  // namespace fire

#endif
