// Core types of the nsparse C++ API, as in the reference (nsparse/types.h:18-41).
#ifndef NSPARSE_B200_TYPES_H
#define NSPARSE_B200_TYPES_H

#include <cstdint>

namespace nsparse {

using idx_t = int32_t;
using term_t = uint16_t;
using weight_t = float;

// Accepted for compatibility with Index::read_csr / read_index(kUseMmap); the
// engine always copies the index into device memory.
enum class Residency : uint8_t {
    kInMemory,
    kMmap,
};

namespace detail {
constexpr idx_t INVALID_IDX = -1;
}

}  // namespace nsparse

#endif
