// Brian's Brain (rule of the reference src/brian/algorithm.hpp:31-44).
#ifndef BRIAN_ALGORITHM_HPP
#define BRIAN_ALGORITHM_HPP

#include "core/ast.hpp"

namespace brian {
using namespace cellato::ast;

enum class brian_cell_state { dead, dying, alive };

using dead = state_constant<brian_cell_state::dead>;
using dying = state_constant<brian_cell_state::dying>;
using alive = state_constant<brian_cell_state::alive>;

using ignites = p<count_neighbors<alive, moore_8_neighbors>, equals, constant<2>>;

using brian_algorithm =
    if_<p<current_state, equals, dead>>::then_<
        if_<ignites>::then_<alive>::else_<dead>
    >::elif_<p<current_state, equals, alive>>::then_<dying>
    ::else_<dead>;
}  // namespace brian

#endif
