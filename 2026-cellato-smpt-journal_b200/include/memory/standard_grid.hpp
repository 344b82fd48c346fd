// One-state-per-cell host grid, interface of the reference
// include/memory/standard_grid.hpp:26-213 (constructors, data(), sizes,
// to_standard(), print(), the 4x4 tile-sum get_checksum()).  Host only: in this
// library the device path is bit planes, so the CUDA members of the reference
// standard grid (its to_cuda/to_cpu for the out-of-scope standard CUDA
// evaluator) are not provided.
#ifndef CELLATO_MEMORY_STANDARD_GRID_HPP
#define CELLATO_MEMORY_STANDARD_GRID_HPP

#include <algorithm>
#include <cstdint>
#include <iostream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "./interface.hpp"

namespace cellato::memory::grids::standard {

template <typename cell_type>
class print_config {
public:
    print_config& with(cell_type state, const std::string& symbol) {
        symbols_[state] = symbol;
        return *this;
    }
    std::string get_str(cell_type state) const {
        auto it = symbols_.find(state);
        return it != symbols_.end() ? it->second : std::to_string(static_cast<int>(state));
    }
    static print_config<cell_type> empty() { return print_config<cell_type>(); }

private:
    std::map<cell_type, std::string> symbols_;
};

template <typename cell_type, device device_type = device::CPU>
class grid {
    static_assert(device_type == device::CPU, "the standard grid is host-only in this library");

public:
    using store_type = cell_type;
    constexpr static bool HAS_OWN_PRINT = true;

    grid() = default;
    grid(int x_size, int y_size) : props_{x_size, y_size}, data_(std::size_t(x_size) * y_size) {}
    grid(std::vector<cell_type>&& data, int x_size, int y_size) : props_{x_size, y_size}, data_(std::move(data)) {
        if (data_.size() != std::size_t(x_size) * y_size)
            throw std::invalid_argument("Data size does not match grid dimensions");
    }
    grid(const grids::properties& properties, std::vector<cell_type> data)
        : props_(properties), data_(std::move(data)) {}

    cell_type* data() { return data_.data(); }
    cell_type* data() const { return const_cast<cell_type*>(data_.data()); }
    int x_size_physical() const { return props_.x_size; }
    int y_size_physical() const { return props_.y_size; }
    int x_size_logical() const { return props_.x_size; }
    int y_size_logical() const { return props_.y_size; }
    grid<cell_type> to_standard() const { return *this; }

    void print(std::ostream& os, print_config<cell_type> config = print_config<cell_type>()) const {
        for (int y = 0; y < props_.y_size; ++y) {
            for (int x = 0; x < props_.x_size; ++x) {
                os << config.get_str(data_[props_.idx(x, y)]) << " ";
                if ((x + 1) % 8 == 0) os << " ";
            }
            os << "\n";
            if ((y + 1) % 8 == 0) os << "\n";
        }
    }

    // Sums of the state values over a 4 x 4 partition into tiles of
    // ceil(X/4) x ceil(Y/4) cells, joined by '-'.
    std::string get_checksum() const {
        constexpr int dims = 4;
        const int tw = (props_.x_size + dims - 1) / dims, th = (props_.y_size + dims - 1) / dims;
        std::ostringstream out;
        for (int ty = 0; ty < dims; ++ty)
            for (int tx = 0; tx < dims; ++tx) {
                std::uint64_t sum = 0;
                for (int y = ty * th; y < std::min(ty * th + th, props_.y_size); ++y)
                    for (int x = tx * tw; x < std::min(tx * tw + tw, props_.x_size); ++x)
                        sum += static_cast<std::uint64_t>(data_[props_.idx(x, y)]);
                if (tx || ty) out << "-";
                out << sum;
            }
        return out.str();
    }

private:
    grids::properties props_{};
    std::vector<cell_type> data_;
};

}  // namespace cellato::memory::grids::standard

#endif  // CELLATO_MEMORY_STANDARD_GRID_HPP
