// cuda::temporal::traverser -- k time steps per launch (interface of the
// reference include/traversers/cuda/temporal.hpp:24-150 and temporal.cu:137-272):
// init validates the reference's conditions and throws its messages; run()
// launches cellato_run_temporal (the sm_100a shared-memory tile kernel).
// temporal_tile_size_y counts tile rows in words as in the reference
// (rows for the linear layout, tile rows for the tiled one); 0 lets the
// library pick the tile.
#ifndef CELLATO_TRAVERSERS_CUDA_LINEAR_TEMPORAL_HPP
#define CELLATO_TRAVERSERS_CUDA_LINEAR_TEMPORAL_HPP

#include <iostream>
#include <utility>

#include "../../experiments/run_params.hpp"
#include "../../memory/interface.hpp"
#include "../traverser_utils.hpp"

namespace cellato::traversers::cuda::temporal {

template <typename evaluator_type, typename grid_type, double average_halo_radius>
class traverser {
    using grid_t = grid_type;
    using cuda_grid_t = typename grid_t::cuda_grid_t;
    using word_t = typename grid_t::store_type;

public:
    static constexpr bool is_CUDA = true;

    void init(grid_t grid, const cellato::run::run_params& params) {
        k_ = params.temporal_steps;
        if (k_ < 1 || k_ > 32) {
            std::cerr << "Error: temporal_steps must be in 1..32.\n";
            throw std::runtime_error("Invalid temporal tile size for temporal linear traverser.");
        }
        if (params.steps % k_ != 0) {
            std::cerr << "Total steps must be divisible by temporal steps.\n";
            throw std::runtime_error("Invalid steps for temporal linear traverser.");
        }
        if (cellato_check_dims(grid_t::cellato_layout, int(sizeof(word_t) * 8), (int)grid.x_size_original(),
                               (int)grid.y_size_original()) != CELLATO_OK) {
            std::cerr << "Grid size not supported: " << cellato_last_error() << "\n";
            throw std::runtime_error("Invalid grid size for CUDA traverser.");
        }
        const int R = grid_t::y_word_tile_size;
        tile_rows_ = 0;
        if (params.temporal_tile_size_y > 0) {
            const int rows = params.temporal_tile_size_y * R;
            tile_rows_ = (rows + 7) / 8 * 8;
            const int halo = (k_ + R - 1) / R * R;
            if (tile_rows_ - 2 * halo <= 0) {
                std::cerr << "Error: effective_y_tile_size must be greater than 0.\n";
                throw std::runtime_error("Invalid temporal tile size for temporal linear traverser.");
            }
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
            auto h0 = final_->to_cpu();
            cb(0, h0);
            for (int s = 0; s < steps; s += k_) {
                advance(std::min(k_, steps - s));
                auto h = final_->to_cpu();
                cb(s + k_, h);
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
        cellato_tune tune{};
        tune.tile_rows = tile_rows_;
        const int rc = cellato_run_temporal(utils::rule_id<evaluator_type>(), grid_t::cellato_layout,
                                            int(sizeof(word_t) * 8), pin, pout, (int)final_->x_size_original(),
                                            (int)final_->y_size_original(), t_, steps, k_, &tune, /*stream=*/nullptr,
                                            &in_b);
        if (rc == CELLATO_ESMEM)
            throw std::runtime_error("Configuration exceeds maximum shared memory size. The temporal tile is too large.");
        utils::check(rc, "cellato_run_temporal");
        if (in_b) final_ = other;
        t_ += steps;
    }

    grid_t input_;
    cuda_grid_t a_, b_;
    cuda_grid_t* final_ = nullptr;
    int k_ = 1, tile_rows_ = 0, t_ = 0;
};

}  // namespace cellato::traversers::cuda::temporal

#endif
