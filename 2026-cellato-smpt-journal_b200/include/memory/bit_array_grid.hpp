// grids::bit_array::grid<state_dictionary, store_word, device> -- the
// reference's bit_array grid (include/memory/bit_array_grid.hpp:80-322) with
// the same constructors, sizes, cell access, to_cuda / to_cpu / to_standard,
// data() / raw_data() and layout constants.  A cell's bits_per_cell index bits
// sit side by side: cells in row-major order, cells_per_word = bits of
// store_word / bits_per_cell, cell i in word i / cells_per_word at bit
// (i % cells_per_word) * bits_per_cell.  The CUDA side owns its words in one
// device buffer through the C ABI (cellato_planes_alloc / upload / download /
// free with a single "plane").
#ifndef CELLATO_MEMORY_BIT_ARRAY_GRID_HPP
#define CELLATO_MEMORY_BIT_ARRAY_GRID_HPP

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "cellato_b200.h"
#include "./interface.hpp"
#include "./standard_grid.hpp"
#include "./state_dictionary.hpp"

namespace cellato::memory::grids::bit_array {

template <typename store_word_type>
struct cuda_params {
    store_word_type* cuda_data;
    std::size_t x_size;
    std::size_t y_size;
    std::size_t bits_per_cell;
};

// Indexed access to the words, and to one cell's index by its row-major
// position (host memory only).
template <typename states_dict_t, typename store_word_type>
class BitArrayProxy {
public:
    static constexpr int bits_per_cell = states_dict_t::needed_bits;
    static constexpr int cells_per_word = int(sizeof(store_word_type) * 8) / bits_per_cell;
    static constexpr store_word_type cell_mask = (store_word_type(1) << bits_per_cell) - 1;

    explicit BitArrayProxy(store_word_type* data) : data_(data) {}

    store_word_type get_individual_cell_at(std::size_t index) const {
        return (data_[index / cells_per_word] >> ((index % cells_per_word) * bits_per_cell)) & cell_mask;
    }
    store_word_type& operator[](std::size_t word) { return data_[word]; }

private:
    store_word_type* data_;
};

template <typename states_dictionary_t, typename store_word_type = std::uint32_t, device device_type = device::CPU>
class grid {
public:
    using states_dict_t = states_dictionary_t;
    constexpr static bool HAS_OWN_PRINT = false;
    constexpr static int bits_per_cell = states_dict_t::needed_bits;
    constexpr static int cells_per_word = int(sizeof(store_word_type) * 8) / bits_per_cell;
    constexpr static store_word_type cell_mask = (store_word_type(1) << bits_per_cell) - 1;

    using original_state_t = typename states_dict_t::state_t;
    using cell_t = original_state_t;
    using store_type = store_word_type;
    using cuda_params_t = cuda_params<store_word_type>;
    using cell_ptr_t = BitArrayProxy<states_dict_t, store_word_type>;
    using cpu_grid_t = grid<states_dict_t, store_word_type, device::CPU>;
    using cuda_grid_t = grid<states_dict_t, store_word_type, device::CUDA>;

    friend class grid<states_dict_t, store_word_type, device::CPU>;
    friend class grid<states_dict_t, store_word_type, device::CUDA>;

    grid() = default;

    grid(std::size_t y_size, std::size_t x_size) : x_size_(x_size), y_size_(y_size) {
        assert_valid_dimensions(x_size);
        if constexpr (device_type == device::CPU) data_.assign(words(), 0);
    }

    grid(std::size_t y_size, std::size_t x_size, const original_state_t* cells)
        requires(device_type == device::CPU)
        : x_size_(x_size), y_size_(y_size) {
        assert_valid_dimensions(x_size);
        data_.assign(words(), 0);
        for (std::size_t i = 0; i < x_size_ * y_size_; ++i) set_cell_at_index(i, cells[i]);
    }

    grid(const standard::grid<original_state_t>& g)
        requires(device_type == device::CPU)
        : grid(g.y_size_physical(), g.x_size_physical(), g.data()) {}

    grid(cuda_params_t params)
        requires(device_type == device::CUDA)
        : x_size_(params.x_size), y_size_(params.y_size), cuda_data_(params.cuda_data) {
        assert_valid_dimensions(params.x_size);
    }

    void free_cuda_memory() {
        if constexpr (device_type == device::CUDA) {
            void* p[1] = {cuda_data_};
            cellato_planes_free(1, p);
            cuda_data_ = nullptr;
        }
    }

    original_state_t get_cell(std::size_t x, std::size_t y) const
        requires(device_type == device::CPU)
    {
        if (x >= x_size_logical() || y >= y_size_logical()) throw std::out_of_range("Cell coordinates out of range");
        return get_cell_at_index(y * x_size_ + x);
    }

    std::vector<original_state_t> to_original_representation() const
        requires(device_type == device::CPU)
    {
        std::vector<original_state_t> out(x_size_ * y_size_);
        for (std::size_t i = 0; i < out.size(); ++i) out[i] = get_cell_at_index(i);
        return out;
    }

    standard::grid<original_state_t> to_standard() const
        requires(device_type == device::CPU)
    {
        return standard::grid<original_state_t>(to_original_representation(), (int)x_size_, (int)y_size_);
    }

    cuda_grid_t to_cuda() const
        requires(device_type == device::CPU)
    {
        void* d[1] = {nullptr};
        const void* h[1] = {data_.data()};
        if (cellato_planes_alloc(1, bytes(), d) != CELLATO_OK)
            throw std::runtime_error(std::string("cellato_planes_alloc: ") + cellato_last_error());
        if (cellato_planes_upload(1, d, h, bytes(), nullptr) != CELLATO_OK)
            throw std::runtime_error(std::string("cellato_planes_upload: ") + cellato_last_error());
        return cuda_grid_t(cuda_params_t{static_cast<store_word_type*>(d[0]), x_size_, y_size_, bits_per_cell});
    }

    cpu_grid_t to_cpu() const
        requires(device_type == device::CUDA)
    {
        cpu_grid_t g(y_size_, x_size_);
        void* h[1] = {g.data_.data()};
        const void* d[1] = {cuda_data_};
        if (cellato_planes_download(1, h, d, bytes(), nullptr) != CELLATO_OK)
            throw std::runtime_error(std::string("cellato_planes_download: ") + cellato_last_error());
        return g;
    }

    std::size_t x_size_logical() const { return x_size_; }
    std::size_t y_size_logical() const { return y_size_; }
    std::size_t x_size_physical() const { return x_size_ / cells_per_word; }
    std::size_t y_size_physical() const { return y_size_; }

    auto data() { return cell_ptr_t(raw_data()); }
    auto data() const { return cell_ptr_t(raw_data()); }

    store_word_type* raw_data() const {
        if constexpr (device_type == device::CUDA)
            return cuda_data_;
        else
            return const_cast<store_word_type*>(data_.data());
    }

    // words and bytes of the packed grid (the last word may be partly unused)
    std::size_t words() const { return (x_size_ * y_size_ + cells_per_word - 1) / cells_per_word; }
    std::size_t bytes() const { return words() * sizeof(store_word_type); }

private:
    std::vector<store_word_type> data_;
    store_word_type* cuda_data_ = nullptr;
    std::size_t x_size_ = 0, y_size_ = 0;

    void set_cell_at_index(std::size_t i, original_state_t state) {
        const std::size_t w = i / cells_per_word, off = (i % cells_per_word) * bits_per_cell;
        data_[w] &= ~(cell_mask << off);
        data_[w] |= (store_word_type(states_dict_t::state_to_index(state)) & cell_mask) << off;
    }

    original_state_t get_cell_at_index(std::size_t i) const {
        const std::size_t w = i / cells_per_word, off = (i % cells_per_word) * bits_per_cell;
        return states_dict_t::index_to_state(int((data_[w] >> off) & cell_mask));
    }

    static void assert_valid_dimensions(std::size_t x_size) {
        if (x_size % cells_per_word != 0)
            throw std::invalid_argument("Grid x_size must be divisible by cells_per_word. x_size=" +
                                        std::to_string(x_size) + ", cells_per_word=" + std::to_string(cells_per_word) +
                                        " (bits [" + std::to_string(sizeof(store_word_type) * 8) +
                                        "] / bits_per_cell [" + std::to_string(bits_per_cell) + "])");
    }
};

}  // namespace cellato::memory::grids::bit_array

#endif
