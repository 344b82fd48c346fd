#ifndef TRAFFIC_CONFIG_HPP
#define TRAFFIC_CONFIG_HPP

#include "../common_init.hpp"
#include "./algorithm.hpp"
#include "memory/state_dictionary.hpp"

namespace traffic {

struct config {
    static constexpr char name[] = "traffic";
    static constexpr double average_halo_radius = 1.0;
    using algorithm = traffic_algorithm;
    using cell_state = traffic_cell_state;
    using state_dictionary = cellato::memory::grids::state_dictionary<cell_state::empty, cell_state::red_car, cell_state::blue_car>;

    struct input {
        // .5 empty / .25 red / .25 blue; the grid utility's default seed (12345)
        struct random {
            static std::vector<cell_state> init(cellato::run::run_params& params) {
                return cellato::automata::iid_grid<cell_state>(
                    params, {{cell_state::empty, 0.5}, {cell_state::red_car, 0.25}, {cell_state::blue_car, 0.25}}, 12345);
            }
        };
    };
};

}  // namespace traffic

#endif
