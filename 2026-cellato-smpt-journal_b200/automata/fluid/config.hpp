#ifndef FLUID_CONFIG_HPP
#define FLUID_CONFIG_HPP

#include "../common_init.hpp"
#include "./algorithm.hpp"
#include "memory/state_dictionary.hpp"

namespace fluid {

struct config {
    static constexpr char name[] = "fluid";
    static constexpr double average_halo_radius = 1.0;
    using algorithm = fluid_algorithm;
    using cell_state = fluid_cell_state;
    using state_dictionary = cellato::memory::grids::int_based_state_dictionary<4>;

    struct input {
        // uniform over the 16 states; the grid utility's default seed (12345)
        struct random {
            static std::vector<cell_state> init(cellato::run::run_params& params) {
                std::vector<std::tuple<cell_state, double>> d;
                for (int s = 0; s < 16; ++s) d.emplace_back(s, 1.0 / 16.0);
                return cellato::automata::iid_grid<cell_state>(params, d, 12345);
            }
        };
    };
};

}  // namespace fluid

#endif
