// Rules outside the library.  A rule written in the rule DSL (core/ast.hpp) and
// described by a config struct with the members of the reference's
// src/<automaton>/config.hpp -- `name`, `algorithm`, `state_dictionary` -- is
// instantiated in the caller's own translation unit, compiled with nvcc for
// sm_100a:
//
//     #include "b200/custom_rule.cuh"
//     #include "my_rule/config.hpp"
//     int id = -1;
//     cellato::b200::register_rule<my_rule::config>(&id);   // links libcellato_b200
//     cellato_run_temporal(id, CELLATO_LAYOUT_TILED_BIT_PLANES, 64, ...);
//
// The lowering and the kernels are the library's own templates, instantiated
// here; the library receives the table of function pointers and runs the rule
// through every entry point (run_simple, run_temporal, batches, the server, the
// checksum) exactly like the ten built-in automata.  This replaces the
// reference's instantiation of each automaton from its template
// (src/_shared/cuda_instantiation_template.cuh:77-193), which needs the rule
// compiled into the framework.
#ifndef CELLATO_B200_CUSTOM_RULE_CUH
#define CELLATO_B200_CUSTOM_RULE_CUH

#include "b200/rule_kernels.cuh"
#include "cellato_b200.h"

namespace cellato::b200 {

// The kernel table of Config (instantiated in this translation unit).
template <class Config>
const cellato_rule_ops* rule_table() {
    return custom_rule_ops<Config>();
}

// Registers Config's table with the library; *rule_out receives its rule id.
// Returns a cellato_status.
template <class Config>
int register_rule(int* rule_out) {
    return cellato_rule_register(custom_rule_ops<Config>(), rule_out);
}

}  // namespace cellato::b200

#endif  // CELLATO_B200_CUSTOM_RULE_CUH
