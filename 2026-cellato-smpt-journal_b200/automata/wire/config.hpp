#ifndef WIRE_CONFIG_HPP
#define WIRE_CONFIG_HPP

#include "./algorithm.hpp"
#include "./circuit_init.hpp"
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
        // the reference's seeded circuit (loops, runs, circles, crossings and
        // electrons), seeded by --seed
        struct random {
            static std::vector<cell_state> init(cellato::run::run_params& params) {
                return circuit_grid<cell_state>(params);
            }
        };
    };
};

}  // namespace wire

#endif
