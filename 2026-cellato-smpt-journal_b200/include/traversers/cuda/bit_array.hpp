// The CUDA traverser for bit_array grids (the reference runs them with
// traversers::simple, one cell-by-cell step per launch:
// include/experiments/test_suites.hpp:84-113): init(grid, params), run(steps
// [, callback]), fetch_result(), is_CUDA.
//
// init() uploads the bit_array words and converts them on the device into bit
// planes that the traverser owns (linear layout, 32-bit words);
// run() advances them with cellato_run_simple, one step per launch, exactly
// the steps of the simple traverser; fetch_result() converts the final planes
// back into the device bit_array and downloads it.  A per-step callback sees a
// host bit_array grid converted the same way.
#ifndef CELLATO_TRAVERSERS_CUDA_BIT_ARRAY_HPP
#define CELLATO_TRAVERSERS_CUDA_BIT_ARRAY_HPP

#include <iostream>
#include <stdexcept>
#include <utility>

#include "../../experiments/run_params.hpp"
#include "../../memory/bit_array_grid.hpp"
#include "../traverser_utils.hpp"

namespace cellato::traversers::cuda::bit_array {

template <typename evaluator_type, typename grid_type>
class traverser {
    using grid_t = grid_type;
    using cuda_grid_t = typename grid_t::cuda_grid_t;
    using word_t = typename grid_t::store_type;
    static constexpr int NB = grid_t::bits_per_cell;
    static constexpr int ARRAY_BITS = int(sizeof(word_t) * 8);

public:
    static constexpr bool is_CUDA = true;

    void init(grid_t grid, const cellato::run::run_params& params) {
        (void)params;
        X_ = (int)grid.x_size_logical();
        Y_ = (int)grid.y_size_logical();
        if (cellato_check_dims(CELLATO_LAYOUT_BIT_PLANES, 32, X_, Y_) != CELLATO_OK) {
            std::cerr << "Grid size not supported: " << cellato_last_error() << "\n";
            throw std::runtime_error("Invalid grid size for CUDA traverser.");
        }
        input_ = std::move(grid);
        dev_ = input_.to_cuda();
        plane_bytes_ = cellato_plane_bytes(X_, Y_);
        utils::check(cellato_planes_alloc(NB, plane_bytes_, a_), "cellato_planes_alloc");
        utils::check(cellato_planes_alloc(NB, plane_bytes_, b_), "cellato_planes_alloc");
        utils::check(cellato_bit_array_to_planes(NB, ARRAY_BITS, dev_.raw_data(), X_, Y_, CELLATO_LAYOUT_BIT_PLANES, 32,
                                                 a_, nullptr),
                     "cellato_bit_array_to_planes");
        in_b_ = false;
        t_ = 0;
    }

    struct no_callback {};

    template <typename callback = no_callback>
    void run(int steps, callback&& cb = no_callback{}) {
        if constexpr (std::is_same_v<std::decay_t<callback>, no_callback>) {
            advance(steps);
        } else {
            cb(0, current());
            for (int s = 0; s < steps; ++s) {
                advance(1);
                cb(s + 1, current());
            }
        }
    }

    grid_t fetch_result() {
        grid_t r = current();
        cellato_planes_free(NB, a_);
        cellato_planes_free(NB, b_);
        dev_.free_cuda_memory();
        return r;
    }

private:
    void advance(int steps) {
        int in_b = 0;
        utils::check(cellato_run_simple(utils::rule_id<evaluator_type>(), CELLATO_LAYOUT_BIT_PLANES, 32,
                                        in_b_ ? b_ : a_, in_b_ ? a_ : b_, X_, Y_, t_, steps, /*tune=*/nullptr,
                                        /*stream=*/nullptr, &in_b),
                     "cellato_run_simple");
        if (in_b) in_b_ = !in_b_;
        t_ += steps;
    }

    // the current state as a host bit_array grid
    grid_t current() {
        utils::check(cellato_planes_to_bit_array(NB, CELLATO_LAYOUT_BIT_PLANES, 32, in_b_ ? b_ : a_, X_, Y_,
                                                 ARRAY_BITS, dev_.raw_data(), nullptr),
                     "cellato_planes_to_bit_array");
        return dev_.to_cpu();
    }

    grid_t input_;
    cuda_grid_t dev_;
    void* a_[8] = {};
    void* b_[8] = {};
    std::size_t plane_bytes_ = 0;
    int X_ = 0, Y_ = 0, t_ = 0;
    bool in_b_ = false;
};

}  // namespace cellato::traversers::cuda::bit_array

#endif
