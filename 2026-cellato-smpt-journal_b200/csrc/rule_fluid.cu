// Kernels of the fluid automaton (rule id 7).
#include "rule_kernels.cuh"
#include "fluid/config.hpp"

CELLATO_DEFINE_RULE_OPS(7, fluid::config)
