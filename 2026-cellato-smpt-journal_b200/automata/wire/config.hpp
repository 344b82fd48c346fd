#ifndef WIRE_CONFIG_HPP
#define WIRE_CONFIG_HPP

#include "../common_init.hpp"
#include "./algorithm.hpp"
#include "memory/state_dictionary.hpp"

namespace wire {

struct config {
    static constexpr char name[] = "wire";
    static constexpr double average_halo_radius = 1.0;
    using algorithm = wire_algorithm;
    using cell_state = wire_cell_state;
    using state_dictionary = cellato::memory::grids::state_dictionary<cell_state::empty, cell_state::electron_head,
                                                                      cell_state::electron_tail, cell_state::conductor>;

    struct input {
        // i.i.d. empty/conductor/head/tail = .50/.40/.05/.05, seeded by --seed
        struct random {
            static std::vector<cell_state> init(cellato::run::run_params& params) {
                return cellato::automata::iid_grid<cell_state>(
                    params,
                    {{cell_state::empty, 0.50}, {cell_state::conductor, 0.40}, {cell_state::electron_head, 0.05},
                     {cell_state::electron_tail, 0.05}},
                    params.seed);
            }
        };
    };
};

}  // namespace wire

#endif
