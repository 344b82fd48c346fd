// Kernels of the fire automaton (rule id 1).
#include "b200/rule_kernels.cuh"
#include "fire/config.hpp"

CELLATO_DEFINE_RULE_OPS(1, fire::config)
