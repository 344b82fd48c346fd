// Kernels of the traffic automaton (rule id 9).
#include "b200/rule_kernels.cuh"
#include "traffic/config.hpp"

CELLATO_DEFINE_RULE_OPS(9, traffic::config)
