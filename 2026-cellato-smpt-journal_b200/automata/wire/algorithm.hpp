// WireWorld (rule of the reference src/wire/algorithm.hpp:48-59).
#ifndef WIRE_ALGORITHM_HPP
#define WIRE_ALGORITHM_HPP

#include "core/ast.hpp"

namespace wire {
using namespace cellato::ast;

enum class wire_cell_state { empty, electron_head, electron_tail, conductor };

using empty = state_constant<wire_cell_state::empty>;
using electron_head = state_constant<wire_cell_state::electron_head>;
using electron_tail = state_constant<wire_cell_state::electron_tail>;
using conductor = state_constant<wire_cell_state::conductor>;

using heads = count_neighbors<electron_head, moore_8_neighbors>;
using fires = p<p<heads, equals, constant<1>>, or_, p<heads, equals, constant<2>>>;

using wire_algorithm =
    if_<p<current_state, equals, electron_head>>::then_<electron_tail>
    ::elif_<p<current_state, equals, electron_tail>>::then_<conductor>
    ::elif_<p<current_state, equals, conductor>>::then_<
        if_<fires>::then_<electron_head>::else_<conductor>
    >::else_<empty>;
}  // namespace wire

#endif
