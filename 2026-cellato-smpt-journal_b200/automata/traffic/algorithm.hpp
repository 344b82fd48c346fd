// Biham-Middleton-Levine traffic: red cars move right on even steps, blue cars
// move down on odd steps (rule of the reference src/traffic/algorithm.hpp:15-61).
#ifndef TRAFFIC_ALGORITHM_HPP
#define TRAFFIC_ALGORITHM_HPP

#include "core/ast.hpp"

namespace traffic {
using namespace cellato::ast;

enum class traffic_cell_state { empty, red_car, blue_car };

using empty = state_constant<traffic_cell_state::empty>;
using red_car = state_constant<traffic_cell_state::red_car>;
using blue_car = state_constant<traffic_cell_state::blue_car>;

// One half-step: `mover` cars advance from `behind` into `ahead` when the cell
// ahead is empty; `other` cars stay put.
template <typename mover, typename other, typename behind, typename ahead>
struct one_direction {
    using algorithm =
        typename if_<p<current_state, equals, mover>>::template then_<
            typename if_<p<ahead, equals, empty>>::template then_<empty>::template else_<mover>
        >::template elif_<p<current_state, equals, empty>>::template then_<
            typename if_<p<behind, equals, mover>>::template then_<mover>::template else_<empty>
        >::template else_<other>;
};

using up = neighbor_at<0, -1>;
using down = neighbor_at<0, 1>;
using left = neighbor_at<-1, 0>;
using right = neighbor_at<1, 0>;

using traffic_algorithm = alternate_algorithms<
    one_direction<red_car, blue_car, left, right>::algorithm,
    one_direction<blue_car, red_car, up, down>::algorithm>;
}  // namespace traffic

#endif
