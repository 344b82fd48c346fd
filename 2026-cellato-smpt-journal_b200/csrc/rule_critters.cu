// Kernels of the critters automaton (rule id 8).
#include "b200/rule_kernels.cuh"
#include "critters/config.hpp"

CELLATO_DEFINE_RULE_OPS(8, critters::config)
