// Index type of grid coordinates (reference include/memory/idx_type.hpp:8).
#ifndef IDX_TYPE_HPP
#define IDX_TYPE_HPP

#include <cstdint>

namespace cellato::memory {
using idx_type = std::int32_t;
}  // namespace cellato::memory

#endif  // IDX_TYPE_HPP
