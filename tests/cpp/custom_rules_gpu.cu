// Test library: the custom rules of custom_rules.hpp instantiated outside the
// B200 library, through the public header-only path (b200/custom_rule.cuh).
// Only the package's public headers are used; nothing of csrc/.  The tests
// load this library, hand its tables to cellato_rule_register and run the
// rules through the C ABI.
#include "b200/custom_rule.cuh"
#include "custom_rules.hpp"

extern "C" {

// Kernel table of custom rule `which` (0 highlife, 1 star-wars, 2
// parity-shift), or NULL.
const cellato_rule_ops* custom_rule_table(int which) {
    switch (which) {
        case 0: return cellato::b200::rule_table<highlife::config>();
        case 1: return cellato::b200::rule_table<star_wars::config>();
        case 2: return cellato::b200::rule_table<parity_shift::config>();
        default: return nullptr;
    }
}

int custom_rule_count(void) { return 3; }

}  // extern "C"
