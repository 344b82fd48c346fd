// Kernels of the game_of_life automaton (rule id 0).
#include "b200/rule_kernels.cuh"
#include "game_of_life/config.hpp"

CELLATO_DEFINE_RULE_OPS(0, game_of_life::config)
