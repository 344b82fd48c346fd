// Suite selection for the B200 bit-plane path: the on_cuda bit-plane suites of
// the reference include/experiments/test_suites.hpp:115-225 (same type
// triples and the same is_for() matching on automaton, device, traverser,
// evaluator, layout and word size), and its on_cuda bit_array suite
// (:84-113), whose steps run on bit planes here.  The reference's CPU suites
// and its standard CUDA suite are outside this library's scope.
#ifndef CELLATO_TEST_SUITES_HPP
#define CELLATO_TEST_SUITES_HPP

#include "../evaluators/bit_array.hpp"
#include "../evaluators/bit_planes.hpp"
#include "../evaluators/tiled_bit_planes.hpp"
#include "../memory/bit_array_grid.hpp"
#include "../memory/bit_planes_grid.hpp"
#include "../memory/tiled_bit_planes_grid.hpp"
#include "../traversers/cuda/bit_array.hpp"
#include "../traversers/cuda/simple.hpp"
#include "../traversers/cuda/temporal.hpp"
#include "./run_params.hpp"

namespace cellato::run::test_suites {

namespace grids = cellato::memory::grids;
namespace evaluators = cellato::evaluators;

namespace on_cuda {
namespace traversers = cellato::traversers::cuda;

template <typename store_word_type>
struct using_ {
    template <typename A, bool TILED, bool TEMPORAL>
    struct suite {
        using automaton = A;
        using original_cell_t = typename A::cell_state;
        using grid_store_word_t = store_word_type;
        using algorithm_t = typename A::algorithm;
        using state_dictionary_t = typename A::state_dictionary;
        using grid_t = std::conditional_t<TILED, grids::tiled_bit_planes::grid<store_word_type, state_dictionary_t>,
                                          grids::bit_planes::grid<store_word_type, state_dictionary_t>>;
        using evaluator_t =
            std::conditional_t<TILED, evaluators::tiled_bit_planes::evaluator<store_word_type, state_dictionary_t, algorithm_t>,
                               evaluators::bit_planes::evaluator<store_word_type, state_dictionary_t, algorithm_t>>;
        using traverser_t =
            std::conditional_t<TEMPORAL, traversers::temporal::traverser<evaluator_t, grid_t, A::average_halo_radius>,
                               traversers::simple::traverser<evaluator_t, grid_t>>;
        constexpr static int x_margin = grid_t::x_word_tile_size;
        constexpr static int y_margin = grid_t::y_word_tile_size;

        static bool is_for(const cellato::run::run_params& params) {
            const char* layout = TILED ? "tiled_bit_planes" : "bit_planes";
            return params.automaton == A::name && params.traverser == (TEMPORAL ? "temporal" : "simple") &&
                   params.device == "CUDA" && params.evaluator == layout && params.layout == layout &&
                   params.word_size == int(sizeof(store_word_type) * 8);
        }
    };
    template <typename A>
    using bit_planes = suite<A, false, false>;
    template <typename A>
    using tiled_bit_planes = suite<A, true, false>;
    template <typename A>
    using temporal_linear_bit_planes = suite<A, false, true>;
    template <typename A>
    using temporal_tiled_bit_planes = suite<A, true, true>;

    template <typename A>
    struct bit_array {
        using automaton = A;
        using original_cell_t = typename A::cell_state;
        using grid_store_word_t = store_word_type;
        using algorithm_t = typename A::algorithm;
        using state_dictionary_t = typename A::state_dictionary;
        using grid_t = grids::bit_array::grid<state_dictionary_t, store_word_type>;
        using evaluator_t = evaluators::bit_array::evaluator<grid_t, algorithm_t>;
        using traverser_t = traversers::bit_array::traverser<evaluator_t, grid_t>;
        constexpr static int x_margin = grid_t::cells_per_word;
        constexpr static int y_margin = 1;

        static bool is_for(const cellato::run::run_params& params) {
            return params.automaton == A::name && params.traverser == "simple" && params.device == "CUDA" &&
                   params.evaluator == "bit_array" && params.layout == "bit_array" &&
                   params.word_size == int(sizeof(store_word_type) * 8);
        }
    };
};
}  // namespace on_cuda

}  // namespace cellato::run::test_suites

#endif
