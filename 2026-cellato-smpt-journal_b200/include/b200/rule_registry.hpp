// Maps a rule type to the rule id of the prebuilt kernels in
// libcellato_b200.so (the C ABI selects kernels by id; see
// include/cellato_b200.h).  The ten automata of the reference are registered
// here; their kernels are instantiated in csrc/rule_<automaton>.cu.
#ifndef CELLATO_B200_RULE_REGISTRY_HPP
#define CELLATO_B200_RULE_REGISTRY_HPP

#include <type_traits>

#include "../../automata/all.hpp"

namespace cellato::b200 {

template <class Algorithm>
struct rule_id_of {
    static constexpr int value = -1;
};

#define CELLATO_REGISTER_RULE(ALGO, ID)       \
    template <>                               \
    struct rule_id_of<ALGO> {                 \
        static constexpr int value = ID;      \
    };
CELLATO_REGISTER_RULE(game_of_life::config::algorithm, 0)
CELLATO_REGISTER_RULE(fire::config::algorithm, 1)
CELLATO_REGISTER_RULE(wire::config::algorithm, 2)
CELLATO_REGISTER_RULE(excitable::config::algorithm, 3)
CELLATO_REGISTER_RULE(brian::config::algorithm, 4)
CELLATO_REGISTER_RULE(maze::config::algorithm, 5)
CELLATO_REGISTER_RULE(cyclic::config::algorithm, 6)
CELLATO_REGISTER_RULE(fluid::config::algorithm, 7)
CELLATO_REGISTER_RULE(critters::config::algorithm, 8)
CELLATO_REGISTER_RULE(traffic::config::algorithm, 9)
#undef CELLATO_REGISTER_RULE

}  // namespace cellato::b200

#endif
