// evaluators::bit_planes::evaluator<word, dictionary, rule> -- the type that
// names a rule on the linear bit-plane layout (reference
// include/evaluators/bit_planes.hpp:45-49).  In this library the evaluation is
// the compile-time lowering in b200/lower.cuh, run by the sm_100a kernels of
// libcellato_b200.so; this type only carries the three parameters to the
// traversers.
#ifndef CELLATO_EVALUATORS_BIT_PLANES_HPP
#define CELLATO_EVALUATORS_BIT_PLANES_HPP

#include "../core/ast.hpp"
#include "../memory/bit_planes_grid.hpp"

namespace cellato::evaluators::bit_planes {

template <typename cell_row_type, typename state_dictionary_type, typename Expression>
struct evaluator {
    using word_t = cell_row_type;
    using state_dictionary_t = state_dictionary_type;
    using expression = Expression;
};

}  // namespace cellato::evaluators::bit_planes

#endif
