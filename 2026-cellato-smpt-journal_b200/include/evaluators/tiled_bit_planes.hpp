// evaluators::tiled_bit_planes::evaluator<word, dictionary, rule> (reference
// include/evaluators/tiled_bit_planes.hpp:69-75); see evaluators/bit_planes.hpp.
#ifndef CELLATO_EVALUATORS_TILED_BIT_PLANES_HPP
#define CELLATO_EVALUATORS_TILED_BIT_PLANES_HPP

#include "../core/ast.hpp"
#include "../memory/tiled_bit_planes_grid.hpp"

namespace cellato::evaluators::tiled_bit_planes {

template <typename cell_row_type, typename state_dictionary_type, typename Expression>
struct evaluator {
    using word_t = cell_row_type;
    using state_dictionary_t = state_dictionary_type;
    using expression = Expression;
};

}  // namespace cellato::evaluators::tiled_bit_planes

#endif
