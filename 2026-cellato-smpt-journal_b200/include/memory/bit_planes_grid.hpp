// bit_planes::grid -- linear bit-plane grid, interface of the reference
// include/memory/bit_planes_grid.hpp:30-271, over the C ABI (memory/plane_grid.hpp).
#ifndef CELLATO_BIT_PLANES_GRID_HPP
#define CELLATO_BIT_PLANES_GRID_HPP

#include "./plane_grid.hpp"

namespace cellato::memory::grids::bit_planes {

template <typename store_word_type, typename states_dict_t, device device_type = device::CPU>
class grid : public detail::plane_grid<grid, store_word_type, states_dict_t, device_type, false> {
    using base = detail::plane_grid<grid, store_word_type, states_dict_t, device_type, false>;

public:
    using base::base;
};

}  // namespace cellato::memory::grids::bit_planes

#endif
