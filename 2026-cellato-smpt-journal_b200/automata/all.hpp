// The ten automata, in rule-id order (see include/cellato_b200.h):
// 0 game-of-life, 1 forest-fire, 2 wire, 3 excitable, 4 brian, 5 maze,
// 6 cyclic, 7 fluid, 8 critters, 9 traffic.
#ifndef CELLATO_AUTOMATA_ALL_HPP
#define CELLATO_AUTOMATA_ALL_HPP
#include "game_of_life/config.hpp"
#include "fire/config.hpp"
#include "wire/config.hpp"
#include "excitable/config.hpp"
#include "brian/config.hpp"
#include "maze/config.hpp"
#include "cyclic/config.hpp"
#include "fluid/config.hpp"
#include "critters/config.hpp"
#include "traffic/config.hpp"
#endif
