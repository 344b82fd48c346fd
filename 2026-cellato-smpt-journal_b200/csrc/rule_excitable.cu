// Kernels of the excitable automaton (rule id 3).
#include "b200/rule_kernels.cuh"
#include "excitable/config.hpp"

CELLATO_DEFINE_RULE_OPS(3, excitable::config)
