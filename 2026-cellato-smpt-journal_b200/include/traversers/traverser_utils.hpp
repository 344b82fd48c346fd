// Shared pieces of the CUDA traverser shims (traversers/cuda/simple.hpp,
// temporal.hpp): rule id and layout of an evaluator/grid pair.
#ifndef CELLATO_TRAVERSERS_UTILS_HPP
#define CELLATO_TRAVERSERS_UTILS_HPP

#include <stdexcept>
#include <string>
#include <type_traits>

#include "cellato_b200.h"
#include "../b200/rule_registry.hpp"

namespace cellato::traversers::utils {

template <typename evaluator_t>
constexpr int rule_id() {
    constexpr int id = cellato::b200::rule_id_of<typename evaluator_t::expression>::value;
    static_assert(id >= 0,
                  "this rule has no prebuilt sm_100a kernels: register it in b200/rule_registry.hpp and "
                  "instantiate it in a csrc/rule_<name>.cu (see csrc/rule_kernels.cuh)");
    return id;
}

inline void check(int status, const char* what) {
    if (status != CELLATO_OK) throw std::runtime_error(std::string(what) + ": " + cellato_last_error());
}

}  // namespace cellato::traversers::utils

#endif
