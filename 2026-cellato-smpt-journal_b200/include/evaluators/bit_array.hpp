// evaluators::bit_array::evaluator<grid, rule> -- the type that names a rule on
// the bit_array layout (reference include/evaluators/bit_array.hpp:16-105, which
// evaluates cell by cell inside each packed word).  In this library the steps
// run on bit planes: the bit_array traverser converts the grid on the device
// and the compile-time lowering in b200/lower.cuh evaluates the rule, so this
// type only carries its parameters to the traverser.
#ifndef CELLATO_EVALUATORS_BIT_ARRAY_HPP
#define CELLATO_EVALUATORS_BIT_ARRAY_HPP

#include "../core/ast.hpp"
#include "../memory/bit_array_grid.hpp"

namespace cellato::evaluators::bit_array {

template <typename grid_type, typename Expression>
struct evaluator {
    using grid_t = grid_type;
    using state_dictionary_t = typename grid_type::states_dict_t;
    using expression = Expression;
};

}  // namespace cellato::evaluators::bit_array

#endif
