// Shared implementation of the bit-plane grid classes (bit_planes_grid.hpp,
// tiled_bit_planes_grid.hpp): host planes on the CPU side, device planes owned
// through the C ABI (cellato_planes_alloc / upload / download / free) on the
// CUDA side.  Byte layouts are the reference's: linear words with the least
// significant bit leftmost (bit_planes_grid.hpp:255-263) or 8 x W/8 tiles with
// bit (y%R)*8 + x%8 (tiled_bit_planes_grid.hpp:270-282).
#ifndef CELLATO_MEMORY_PLANE_GRID_HPP
#define CELLATO_MEMORY_PLANE_GRID_HPP

#include <array>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "cellato_b200.h"
#include "./interface.hpp"
#include "./standard_grid.hpp"

namespace cellato::memory::grids::detail {

template <template <typename, typename, device> class Self, typename W, typename dict, device dev, bool TILED>
class plane_grid {
public:
    constexpr static bool HAS_OWN_PRINT = false;
    constexpr static int needed_bits = dict::needed_bits;
    static constexpr int word_store_bits = sizeof(W) * 8;
    static constexpr int x_word_tile_size = TILED ? 8 : word_store_bits;
    static constexpr int y_word_tile_size = TILED ? word_store_bits / 8 : 1;
    static constexpr int cellato_layout = TILED ? CELLATO_LAYOUT_TILED_BIT_PLANES : CELLATO_LAYOUT_BIT_PLANES;

    using storage_tuple_t = std::array<std::vector<W>, needed_bits>;
    using storage_tuple_of_pointers = std::array<W*, needed_bits>;
    using original_state_t = typename dict::state_t;
    using cell_t = W;
    using store_type = W;
    using cpu_grid_t = Self<W, dict, device::CPU>;
    using cuda_grid_t = Self<W, dict, device::CUDA>;

    plane_grid() = default;

    plane_grid(std::size_t y_size, std::size_t x_size)
        : xw_(x_size / x_word_tile_size), yw_(y_size / y_word_tile_size) {
        if constexpr (dev == device::CPU)
            for (auto& p : host_) p.assign(xw_ * yw_, W(0));
    }

    plane_grid(std::size_t y_size, std::size_t x_size, const original_state_t* cells)
        requires(dev == device::CPU)
    {
        pack(y_size, x_size, cells);
    }

    plane_grid(const standard::grid<original_state_t>& g)
        requires(dev == device::CPU)
    {
        pack(g.y_size_physical(), g.x_size_physical(), g.data());
    }

    void free_cuda_memory() {
        if constexpr (dev == device::CUDA) {
            void* p[needed_bits];
            for (int i = 0; i < needed_bits; ++i) p[i] = dev_[i];
            cellato_planes_free(needed_bits, p);
            for (auto& d : dev_) d = nullptr;
        }
    }

    original_state_t get_cell(std::size_t x, std::size_t y) const
        requires(dev == device::CPU)
    {
        if (x >= x_size_original() || y >= y_size_original()) throw std::out_of_range("Cell coordinates out of range");
        const auto [word, bit] = locate(x, y);
        int index = 0;
        for (int p = 0; p < needed_bits; ++p) index |= int((host_[p][word] >> bit) & 1) << p;
        return dict::index_to_state(index);
    }

    std::vector<original_state_t> to_original_representation() const
        requires(dev == device::CPU)
    {
        std::vector<original_state_t> out(x_size_original() * y_size_original());
        for (std::size_t y = 0; y < y_size_original(); ++y)
            for (std::size_t x = 0; x < x_size_original(); ++x) out[y * x_size_original() + x] = get_cell(x, y);
        return out;
    }

    standard::grid<original_state_t> to_standard() const
        requires(dev == device::CPU)
    {
        return standard::grid<original_state_t>(to_original_representation(), (int)x_size_original(),
                                                (int)y_size_original());
    }

    cuda_grid_t to_cuda() const
        requires(dev == device::CPU)
    {
        cuda_grid_t g;
        g.xw_ = xw_;
        g.yw_ = yw_;
        void* d[needed_bits];
        const void* h[needed_bits];
        if (cellato_planes_alloc(needed_bits, bytes(), d) != CELLATO_OK)
            throw std::runtime_error(std::string("cellato_planes_alloc: ") + cellato_last_error());
        for (int p = 0; p < needed_bits; ++p) {
            g.dev_[p] = static_cast<W*>(d[p]);
            h[p] = host_[p].data();
        }
        if (cellato_planes_upload(needed_bits, d, h, bytes(), nullptr) != CELLATO_OK)
            throw std::runtime_error(std::string("cellato_planes_upload: ") + cellato_last_error());
        return g;
    }

    // Device grid of the same shape with uninitialised planes.
    cuda_grid_t allocate_cuda_like() const {
        cuda_grid_t g;
        g.xw_ = xw_;
        g.yw_ = yw_;
        void* d[needed_bits];
        if (cellato_planes_alloc(needed_bits, bytes(), d) != CELLATO_OK)
            throw std::runtime_error(std::string("cellato_planes_alloc: ") + cellato_last_error());
        for (int p = 0; p < needed_bits; ++p) g.dev_[p] = static_cast<W*>(d[p]);
        return g;
    }

    cpu_grid_t to_cpu() const
        requires(dev == device::CUDA)
    {
        cpu_grid_t g(y_size_original(), x_size_original());
        void* h[needed_bits];
        const void* d[needed_bits];
        for (int p = 0; p < needed_bits; ++p) {
            h[p] = g.host_[p].data();
            d[p] = dev_[p];
        }
        if (cellato_planes_download(needed_bits, h, d, bytes(), nullptr) != CELLATO_OK)
            throw std::runtime_error(std::string("cellato_planes_download: ") + cellato_last_error());
        if (cudaStreamSynchronize(nullptr) != cudaSuccess) throw std::runtime_error("download failed");
        return g;
    }

    std::size_t x_size_original() const { return xw_ * x_word_tile_size; }
    std::size_t y_size_original() const { return yw_ * y_word_tile_size; }
    std::size_t x_size_physical() const { return xw_; }
    std::size_t y_size_physical() const { return yw_; }
    std::size_t bytes() const { return xw_ * yw_ * sizeof(W); }

    storage_tuple_of_pointers data() const {
        storage_tuple_of_pointers r{};
        for (int p = 0; p < needed_bits; ++p) {
            if constexpr (dev == device::CUDA)
                r[p] = dev_[p];
            else
                r[p] = const_cast<W*>(host_[p].data());
        }
        return r;
    }

protected:
    template <template <typename, typename, device> class, typename, typename, device, bool>
    friend class plane_grid;

    storage_tuple_t host_{};
    std::array<W*, needed_bits> dev_{};
    std::size_t xw_ = 0, yw_ = 0;

    std::pair<std::size_t, int> locate(std::size_t x, std::size_t y) const {
        if constexpr (TILED)
            return {(y / y_word_tile_size) * xw_ + x / 8, int((y % y_word_tile_size) * 8 + x % 8)};
        else
            return {y * xw_ + x / word_store_bits, int(x % word_store_bits)};
    }

    void pack(std::size_t y_size, std::size_t x_size, const original_state_t* cells) {
        if (x_size % x_word_tile_size != 0 || y_size % y_word_tile_size != 0)
            throw std::invalid_argument("`x_size` and `y_size` must be multiples of the word tile (" +
                                        std::to_string(x_word_tile_size) + " x " + std::to_string(y_word_tile_size) +
                                        "), but were " + std::to_string(x_size) + " and " + std::to_string(y_size));
        xw_ = x_size / x_word_tile_size;
        yw_ = y_size / y_word_tile_size;
        for (auto& p : host_) p.assign(xw_ * yw_, W(0));
        for (std::size_t y = 0; y < y_size; ++y)
            for (std::size_t x = 0; x < x_size; ++x) {
                const int index = dict::state_to_index(cells[y * x_size + x]);
                const auto [word, bit] = locate(x, y);
                for (int p = 0; p < needed_bits; ++p)
                    if ((index >> p) & 1) host_[p][word] |= W(1) << bit;
            }
    }
};

}  // namespace cellato::memory::grids::detail

#endif
