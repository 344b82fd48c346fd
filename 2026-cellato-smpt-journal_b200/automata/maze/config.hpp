#ifndef MAZE_CONFIG_HPP
#define MAZE_CONFIG_HPP

#include "../common_init.hpp"
#include "./algorithm.hpp"
#include "memory/state_dictionary.hpp"

namespace maze {

struct config {
    static constexpr char name[] = "maze";
    static constexpr double average_halo_radius = 1.0;
    using algorithm = maze_algorithm;
    using cell_state = maze_cell_state;
    using state_dictionary = cellato::memory::grids::state_dictionary<cell_state::empty, cell_state::wall>;

    struct input {
        // .80 empty / .20 wall; the grid utility's default seed (12345)
        struct random {
            static std::vector<cell_state> init(cellato::run::run_params& params) {
                return cellato::automata::iid_grid<cell_state>(
                    params, {{cell_state::empty, 0.80}, {cell_state::wall, 0.20}}, 12345);
            }
        };
    };
};

}  // namespace maze

#endif
