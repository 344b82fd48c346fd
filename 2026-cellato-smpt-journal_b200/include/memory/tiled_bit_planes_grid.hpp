// tiled_bit_planes::grid -- 8 x W/8 tiled bit-plane grid, interface of the
// reference include/memory/tiled_bit_planes_grid.hpp:30-289, over the C ABI.
#ifndef TILED_BIT_PLANES_GRID_HPP
#define TILED_BIT_PLANES_GRID_HPP

#include "./plane_grid.hpp"

namespace cellato::memory::grids::tiled_bit_planes {

template <typename store_word_type, typename states_dict_t, device device_type = device::CPU>
class grid : public detail::plane_grid<grid, store_word_type, states_dict_t, device_type, true> {
    using base = detail::plane_grid<grid, store_word_type, states_dict_t, device_type, true>;

public:
    using base::base;
};

}  // namespace cellato::memory::grids::tiled_bit_planes

#endif
