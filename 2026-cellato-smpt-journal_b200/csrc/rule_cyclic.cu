// Kernels of the cyclic automaton (rule id 6).
#include "b200/rule_kernels.cuh"
#include "cyclic/config.hpp"

CELLATO_DEFINE_RULE_OPS(6, cyclic::config)
