// The native CSR layout reader (csr_layout.cpp) behind
// SeismicIndex::read_csr(path, Residency::kMmap).
#ifndef NSP_CSR_LAYOUT_READ_H
#define NSP_CSR_LAYOUT_READ_H

#include <vector>

#include "nsparse/types.h"

namespace nsparse::detail {

struct NativeCsr {
    idx_t rows = 0;
    std::vector<idx_t> indptr;
    std::vector<term_t> indices;
    std::vector<float> values;
};

// Reads and checks a native-layout file for an index of `dimension` terms;
// throws as the reference's mapped reader does.
NativeCsr read_native_csr(const char* path, int dimension);

}  // namespace nsparse::detail

#endif  // NSP_CSR_LAYOUT_READ_H
