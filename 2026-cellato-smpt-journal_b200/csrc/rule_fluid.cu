// Kernels of the fluid automaton (rule id 7).
#include "b200/rule_kernels.cuh"
#include "fluid/config.hpp"

CELLATO_DEFINE_RULE_OPS(7, fluid::config)
