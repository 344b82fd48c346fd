// Kernels of the brian automaton (rule id 4).
#include "b200/rule_kernels.cuh"
#include "brian/config.hpp"

CELLATO_DEFINE_RULE_OPS(4, brian::config)
