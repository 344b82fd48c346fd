#ifndef GREENBERG_HASTINGS_CONFIG_HPP
#define GREENBERG_HASTINGS_CONFIG_HPP

#include "../common_init.hpp"
#include "./algorithm.hpp"
#include "memory/state_dictionary.hpp"

namespace excitable {

struct config {
    static constexpr char name[] = "excitable";
    static constexpr double average_halo_radius = 1.0;
    using algorithm = ghm_algorithm;
    using cell_state = ghm_cell_state;
    using state_dictionary = cellato::memory::grids::state_dictionary<
        cell_state::quiescent, cell_state::excited, cell_state::refractory_1, cell_state::refractory_2,
        cell_state::refractory_3, cell_state::refractory_4, cell_state::refractory_5, cell_state::refractory_6>;

    struct input {
        // .70/.15/.05/.03/.03/.02/.01/.01 over states 0..7, seeded by --seed
        struct random {
            static std::vector<cell_state> init(cellato::run::run_params& params) {
                using s = cell_state;
                return cellato::automata::iid_grid<cell_state>(
                    params,
                    {{s::quiescent, 0.70}, {s::excited, 0.15}, {s::refractory_1, 0.05}, {s::refractory_2, 0.03},
                     {s::refractory_3, 0.03}, {s::refractory_4, 0.02}, {s::refractory_5, 0.01}, {s::refractory_6, 0.01}},
                    params.seed);
            }
        };
    };
};

}  // namespace excitable

#endif
