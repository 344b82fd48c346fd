#ifndef BRIAN_CONFIG_HPP
#define BRIAN_CONFIG_HPP

#include "../common_init.hpp"
#include "./algorithm.hpp"
#include "memory/state_dictionary.hpp"

namespace brian {

struct config {
    static constexpr char name[] = "brian";
    static constexpr double average_halo_radius = 1.0;
    using algorithm = brian_algorithm;
    using cell_state = brian_cell_state;
    using state_dictionary = cellato::memory::grids::state_dictionary<cell_state::dead, cell_state::dying, cell_state::alive>;

    struct input {
        // alive with probability 0.2 (else dead), seeded by --seed
        struct random {
            static std::vector<cell_state> init(cellato::run::run_params& params) {
                return cellato::automata::iid_grid<cell_state>(
                    params, {{cell_state::alive, 0.2}, {cell_state::dead, 0.8}}, params.seed);
            }
        };
    };
};

}  // namespace brian

#endif
