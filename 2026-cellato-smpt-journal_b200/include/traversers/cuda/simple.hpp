// cuda::simple::traverser -- one time step per launch (interface of the
// reference include/traversers/cuda/simple.hpp:25-106 and simple.cu:43-97):
// init(grid, params), run(steps[, callback]), fetch_result(), is_CUDA.
// Backed by cellato_run_simple (the sm_100a single-step kernels).
#ifndef CELLATO_TRAVERSERS_CUDA_SIMPLE_HPP
#define CELLATO_TRAVERSERS_CUDA_SIMPLE_HPP

#include <functional>
#include <iostream>
#include <memory>
#include <utility>

#include "../../experiments/run_params.hpp"
#include "../../memory/interface.hpp"
#include "../traverser_utils.hpp"

namespace cellato::traversers::cuda::simple {

template <typename evaluator_type, typename grid_type>
class traverser {
    using grid_t = grid_type;
    using cuda_grid_t = typename grid_t::cuda_grid_t;
    using word_t = typename grid_t::store_type;

public:
    static constexpr bool is_CUDA = true;

    void init(grid_t grid, const cellato::run::run_params& params) {
        (void)params;
        if (cellato_check_dims(grid_t::cellato_layout, int(sizeof(word_t) * 8), (int)grid.x_size_original(),
                               (int)grid.y_size_original()) != CELLATO_OK) {
            std::cerr << "Grid size not supported: " << cellato_last_error() << "\n";
            throw std::runtime_error("Invalid grid size for CUDA traverser.");
        }
        input_ = std::move(grid);
        a_ = input_.to_cuda();
        b_ = input_.allocate_cuda_like();
        final_ = &a_;
        t_ = 0;
    }

    struct no_callback {};

    template <typename callback = no_callback>
    void run(int steps, callback&& cb = no_callback{}) {
        if constexpr (std::is_same_v<std::decay_t<callback>, no_callback>) {
            advance(steps);
        } else {
            auto host = final_->to_cpu();
            cb(0, host);
            for (int s = 0; s < steps; ++s) {
                advance(1);
                auto h = final_->to_cpu();
                cb(s + 1, h);
            }
        }
    }

    grid_t fetch_result() {
        grid_t r = final_->to_cpu();
        a_.free_cuda_memory();
        b_.free_cuda_memory();
        return r;
    }

private:
    void advance(int steps) {
        cuda_grid_t* other = (final_ == &a_) ? &b_ : &a_;
        auto in = final_->data();
        auto out = other->data();
        void* pin[grid_t::needed_bits];
        void* pout[grid_t::needed_bits];
        for (int p = 0; p < grid_t::needed_bits; ++p) pin[p] = in[p], pout[p] = out[p];
        int in_b = 0;
        utils::check(cellato_run_simple(utils::rule_id<evaluator_type>(), grid_t::cellato_layout, int(sizeof(word_t) * 8),
                                        pin, pout, (int)final_->x_size_original(), (int)final_->y_size_original(), t_,
                                        steps, /*tune=*/nullptr, /*stream=*/nullptr, &in_b),
                     "cellato_run_simple");
        if (in_b) final_ = other;
        t_ += steps;
    }

    grid_t input_;
    cuda_grid_t a_, b_;
    cuda_grid_t* final_ = nullptr;
    int t_ = 0;
};

}  // namespace cellato::traversers::cuda::simple

#endif
