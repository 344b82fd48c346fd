// Kernels of the fire automaton (rule id 1).
#include "rule_kernels.cuh"
#include "fire/config.hpp"

CELLATO_DEFINE_RULE_OPS(1, fire::config)
