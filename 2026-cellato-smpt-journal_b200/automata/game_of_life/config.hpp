#ifndef GAME_OF_LIFE_CONFIG_HPP
#define GAME_OF_LIFE_CONFIG_HPP

#include "../common_init.hpp"
#include "./algorithm.hpp"
#include "memory/state_dictionary.hpp"

namespace game_of_life {

struct config {
    static constexpr char name[] = "game-of-life";
    static constexpr double average_halo_radius = 1.0;
    using algorithm = gol_algorithm;
    using cell_state = gol_cell_state;
    using state_dictionary = cellato::memory::grids::state_dictionary<cell_state::dead, cell_state::alive>;

    struct input {
        // alive with probability 0.2, seeded by --seed
        struct random {
            static std::vector<cell_state> init(cellato::run::run_params& params) {
                return cellato::automata::iid_grid<cell_state>(
                    params, {{cell_state::alive, 0.2}, {cell_state::dead, 0.8}}, params.seed);
            }
        };
    };
};

}  // namespace game_of_life

#endif
