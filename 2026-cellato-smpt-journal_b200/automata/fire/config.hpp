#ifndef FOREST_FIRE_CONFIG_HPP
#define FOREST_FIRE_CONFIG_HPP

#include "../common_init.hpp"
#include "./algorithm.hpp"
#include "memory/state_dictionary.hpp"

namespace fire {

struct config {
    static constexpr char name[] = "forest-fire";
    static constexpr double average_halo_radius = 1.0;
    using algorithm = fire_algorithm;
    using cell_state = fire_cell_state;
    // dictionary order (and so plane encoding) differs from the enum order
    using state_dictionary =
        cellato::memory::grids::state_dictionary<cell_state::empty, cell_state::tree, cell_state::fire, cell_state::ash>;

    struct input {
        // .20 empty / .79 tree / .01 fire; the grid utility's default seed (12345)
        struct random {
            static std::vector<cell_state> init(cellato::run::run_params& params) {
                return cellato::automata::iid_grid<cell_state>(
                    params,
                    {{cell_state::empty, 0.20}, {cell_state::tree, 0.79}, {cell_state::fire, 0.01}, {cell_state::ash, 0.0}},
                    12345);
            }
        };
    };
};

}  // namespace fire

#endif
