// Greenberg-Hastings excitable medium with six refractory states
// (rule of the reference src/excitable/algorithm.hpp:57-71).
#ifndef GREENBERG_HASTINGS_ALGORITHM_HPP
#define GREENBERG_HASTINGS_ALGORITHM_HPP

#include "core/ast.hpp"

namespace excitable {
using namespace cellato::ast;

enum class ghm_cell_state {
    quiescent = 0, excited = 1,
    refractory_1 = 2, refractory_2 = 3, refractory_3 = 4, refractory_4 = 5, refractory_5 = 6, refractory_6 = 7
};

template <ghm_cell_state S>
using is = p<current_state, equals, state_constant<S>>;
template <ghm_cell_state S>
using st = state_constant<S>;

using excited_nearby = p<count_neighbors<st<ghm_cell_state::excited>, moore_8_neighbors>, greater_than, constant<0>>;

using ghm_algorithm =
    if_<is<ghm_cell_state::quiescent>>::then_<
        if_<excited_nearby>::then_<st<ghm_cell_state::excited>>::else_<st<ghm_cell_state::quiescent>>
    >::elif_<is<ghm_cell_state::excited>>::then_<st<ghm_cell_state::refractory_1>>
    ::elif_<is<ghm_cell_state::refractory_1>>::then_<st<ghm_cell_state::refractory_2>>
    ::elif_<is<ghm_cell_state::refractory_2>>::then_<st<ghm_cell_state::refractory_3>>
    ::elif_<is<ghm_cell_state::refractory_3>>::then_<st<ghm_cell_state::refractory_4>>
    ::elif_<is<ghm_cell_state::refractory_4>>::then_<st<ghm_cell_state::refractory_5>>
    ::elif_<is<ghm_cell_state::refractory_5>>::then_<st<ghm_cell_state::refractory_6>>
    ::else_<st<ghm_cell_state::quiescent>>;
}  // namespace excitable

#endif
