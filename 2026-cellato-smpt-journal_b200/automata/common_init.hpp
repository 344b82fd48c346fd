// Seeded i.i.d. initialisers shared by the automaton configs: each draws its
// grid with memory/grid_utils.hpp's generate_random_grid (std::mt19937 +
// cumulative thresholds), from the distribution its automaton names.
#ifndef CELLATO_AUTOMATA_COMMON_INIT_HPP
#define CELLATO_AUTOMATA_COMMON_INIT_HPP

#include <tuple>
#include <vector>

#include "experiments/run_params.hpp"
#include "memory/grid_utils.hpp"

namespace cellato::automata {

template <typename State>
std::vector<State> iid_grid(const cellato::run::run_params& params,
                            const std::vector<std::tuple<State, double>>& distribution, unsigned seed) {
    std::vector<State> grid(std::size_t(params.x_size) * params.y_size);
    cellato::memory::grids::utils::generate_random_grid(grid, params.y_size, params.x_size, distribution, seed);
    return grid;
}

}  // namespace cellato::automata

#endif
