// State dictionaries: the bijection between an automaton's states and the
// integers 0..n-1 that the bit planes store (bit i of the index in plane i).
// Interface of the reference include/memory/state_dictionary.hpp:10-70:
// number_of_values, needed_bits = floor(log2(n-1)) + 1, state_to_index and
// index_to_state (throwing std::out_of_range on unknown states/indices).
#ifndef CELLATO_MEMORY_STATE_DICTIONARY_HPP
#define CELLATO_MEMORY_STATE_DICTIONARY_HPP

#include <stdexcept>
#include <type_traits>

namespace cellato::memory::grids {

namespace detail {
constexpr int floor_log2(int n) {
    int r = 0;
    while (n >= 2) {
        n /= 2;
        ++r;
    }
    return r;
}
}  // namespace detail

// Enumerated states; the index of a state is its position in the list.
template <auto... states>
class state_dictionary {
public:
    using index_t = int;
    using state_t = std::common_type_t<decltype(states)...>;

    static constexpr index_t number_of_values = sizeof...(states);
    static constexpr index_t needed_bits = detail::floor_log2(number_of_values - 1) + 1;

    static constexpr index_t state_to_index(state_t state) {
        constexpr state_t table[] = {states...};
        for (index_t i = 0; i < number_of_values; ++i)
            if (table[i] == state) return i;
        throw std::out_of_range("State not found in dictionary");
    }

    static constexpr state_t index_to_state(index_t index) {
        constexpr state_t table[] = {states...};
        if (index >= 0 && index < number_of_values) return table[index];
        throw std::out_of_range("Index out of range");
    }
};

// Integer states 0 .. 2^bits - 1, stored as themselves.
template <int bits>
class int_based_state_dictionary {
public:
    using index_t = int;
    using state_t = int;

    static constexpr index_t number_of_values = 1 << bits;
    static constexpr index_t needed_bits = bits;

    static constexpr index_t state_to_index(state_t state) {
        if (state >= 0 && state < number_of_values) return state;
        throw std::out_of_range("State not found in dictionary");
    }

    static constexpr state_t index_to_state(index_t index) {
        if (index >= 0 && index < number_of_values) return index;
        throw std::out_of_range("Index out of range");
    }
};

}  // namespace cellato::memory::grids

#endif  // CELLATO_MEMORY_STATE_DICTIONARY_HPP
