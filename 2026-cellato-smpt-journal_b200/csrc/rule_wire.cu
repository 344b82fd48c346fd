// Kernels of the wire automaton (rule id 2).
#include "b200/rule_kernels.cuh"
#include "wire/config.hpp"

CELLATO_DEFINE_RULE_OPS(2, wire::config)
