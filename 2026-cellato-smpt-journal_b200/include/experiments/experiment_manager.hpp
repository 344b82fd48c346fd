// Runs warm-up and timed rounds of one suite (reference
// include/experiments/experiment_manager.hpp:38-163): each round builds the
// grid from the initial state, init()s the traverser, times run() with CUDA
// events, fetches the result and records its checksum.
#ifndef EXPERIMENT_MANAGER_HPP
#define EXPERIMENT_MANAGER_HPP

#include <cuda_runtime.h>

#include <chrono>
#include <iostream>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "../memory/standard_grid.hpp"
#include "../traversers/cuda_utils.cuh"
#include "./experiment_report.hpp"
#include "./run_params.hpp"

namespace cellato::run {

template <typename test_suite>
class experiment_manager {
public:
    using original_cell_t = typename test_suite::original_cell_t;
    using grid_t = typename test_suite::grid_t;
    using traverser_t = typename test_suite::traverser_t;
    using standard_grid_t = cellato::memory::grids::standard::grid<original_cell_t>;
    using print_config_t = cellato::memory::grids::standard::print_config<original_cell_t>;

    experiment_report run_experiment(const run_params& params, const std::vector<original_cell_t>& initial) {
        experiment_report report;
        report.params = params;
        for (int i = 0; i < params.warmup_rounds + params.rounds; ++i) {
            auto [ms, checksum] = run_round(params, initial);
            if (i >= params.warmup_rounds) {
                report.execution_times_ms.push_back(ms);
                report.checksums.push_back(checksum);
            }
        }
        return report;
    }

    void set_print_config(print_config_t c) { print_config_ = c; }

private:
    print_config_t print_config_;

    std::tuple<double, std::string> run_round(const run_params& params, const std::vector<original_cell_t>& initial) {
        standard_grid_t g(params.x_size, params.y_size);
        std::copy(initial.begin(), initial.end(), g.data());
        grid_t grid(g);
        traverser_t traverser;
        traverser.init(grid, params);
        cudaEvent_t start, stop;
        CUCH(cudaEventCreate(&start));
        CUCH(cudaEventCreate(&stop));
        CUCH(cudaEventRecord(start));
        if (params.print) {
            traverser.run(params.steps, [&](int iteration, const auto& grid_now) {
                std::cerr << "\nIteration: " << iteration << "\n";
                grid_now.to_standard().print(std::cerr, print_config_);
                std::this_thread::sleep_for(std::chrono::milliseconds(400));
            });
        } else {
            traverser.run(params.steps);
        }
        CUCH(cudaEventRecord(stop));
        CUCH(cudaEventSynchronize(stop));
        float ms = 0;
        CUCH(cudaEventElapsedTime(&ms, start, stop));
        CUCH(cudaEventDestroy(start));
        CUCH(cudaEventDestroy(stop));
        CUCH(cudaDeviceSynchronize());
        grid_t result = traverser.fetch_result();
        auto standard = result.to_standard();
        if (params.print) {
            std::cerr << "\nFinal result:\n";
            standard.print(std::cerr, print_config_);
        }
        return {double(ms), standard.get_checksum()};
    }
};

}  // namespace cellato::run

#endif
