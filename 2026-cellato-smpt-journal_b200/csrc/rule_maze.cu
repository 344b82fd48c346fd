// Kernels of the maze automaton (rule id 5).
#include "b200/rule_kernels.cuh"
#include "maze/config.hpp"

CELLATO_DEFINE_RULE_OPS(5, maze::config)
