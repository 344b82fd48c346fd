#ifndef CRITTERS_CONFIG_HPP
#define CRITTERS_CONFIG_HPP

#include "../common_init.hpp"
#include "./algorithm.hpp"
#include "memory/state_dictionary.hpp"

namespace critters {

struct config {
    static constexpr char name[] = "critters";
    static constexpr double average_halo_radius = 1.0;
    using algorithm = critters_algorithm;
    using cell_state = critters_cell_state;
    using state_dictionary = cellato::memory::grids::state_dictionary<cell_state::dead, cell_state::alive>;

    struct input {
        // .5 / .5; the grid utility's default seed (12345)
        struct random {
            static std::vector<cell_state> init(cellato::run::run_params& params) {
                return cellato::automata::iid_grid<cell_state>(
                    params, {{cell_state::dead, 0.5}, {cell_state::alive, 0.5}}, 12345);
            }
        };
    };
};

}  // namespace critters

#endif
