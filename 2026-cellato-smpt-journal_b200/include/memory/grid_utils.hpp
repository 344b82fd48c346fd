// Seeded random grids, interface of the reference
// include/memory/grid_utils.hpp:15-75 (used by the automata initialisers).
// Each cell draws r ~ U[0,1) from std::mt19937(seed) through
// std::uniform_real_distribution<double> and takes the first state whose
// cumulative probability is >= r; with the same standard library this yields
// the same grids as the reference's initialisers.
#ifndef GRID_UTILS_HPP
#define GRID_UTILS_HPP

#include <cmath>
#include <iostream>
#include <random>
#include <tuple>
#include <vector>

namespace cellato::memory::grids::utils {

template <typename CellState>
void generate_random_grid(std::vector<CellState>& grid, std::size_t height, std::size_t width,
                          const std::vector<std::tuple<CellState, double>>& probabilities,
                          unsigned int seed = 12345) {
    std::vector<std::tuple<CellState, double>> cumulative;
    double total = 0.0;
    for (const auto& [state, p] : probabilities) {
        total += p;
        cumulative.emplace_back(state, total);
    }
    if (std::abs(total - 1.0) > 0.001)
        std::cerr << "Warning: Probabilities sum to " << total << " instead of 1.0" << std::endl;

    std::mt19937 rng(seed);
    std::uniform_real_distribution<double> unit(0.0, 1.0);
    const std::size_t cells = height * width;
    for (std::size_t i = 0; i < cells; ++i) {
        const double r = unit(rng);
        for (const auto& [state, threshold] : cumulative) {
            if (r <= threshold) {
                grid[i] = state;
                break;
            }
        }
    }
}

template <typename CellState>
void generate_random_grid(std::vector<CellState>& grid, std::size_t height, std::size_t width,
                          CellState primary_state, double primary_probability, CellState secondary_state,
                          unsigned int seed = 12345) {
    generate_random_grid(grid, height, width,
                         std::vector<std::tuple<CellState, double>>{{primary_state, primary_probability},
                                                                    {secondary_state, 1.0 - primary_probability}},
                         seed);
}

}  // namespace cellato::memory::grids::utils

#endif  // GRID_UTILS_HPP
