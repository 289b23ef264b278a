// The two on-disk CSR layouts Index::read_csr takes, with the reference's
// names (nsparse/utils/csr_layout.h:19-67 in the reference), so a caller that
// converts files for the mapped residency keeps its code.
//
// Both start with three int64 values {rows, cols, nnz}. Then:
//   interchange (what scipy writes):  int64 indptr[rows + 1], int32 indices[nnz],
//                                     float values[nnz]
//   native (".mcsr"):                 idx_t indptr[rows + 1], term_t indices[nnz],
//                                     zero bytes up to a 4-byte boundary,
//                                     float values[nnz]
// SeismicIndex::read_csr(path, Residency::kMmap) reads the native layout;
// Residency::kInMemory (and every other index type) the interchange one. The
// engine copies either into device memory.
#ifndef NSPARSE_B200_CSR_LAYOUT_H
#define NSPARSE_B200_CSR_LAYOUT_H

#include <cstddef>
#include <cstdint>
#include <string>

#include "nsparse/types.h"

namespace nsparse::csr_layout {

constexpr size_t kHeaderBytes = 3 * sizeof(int64_t);

inline constexpr const char* kNativeSuffix = ".mcsr";

// Zero bytes that bring file position `pos` to the values' float alignment.
constexpr size_t padding(size_t pos) {
    return (sizeof(float) - pos % sizeof(float)) % sizeof(float);
}

constexpr size_t interchange_file_size(size_t indptr_size, size_t nnz) {
    return kHeaderBytes + indptr_size * sizeof(int64_t) + nnz * (sizeof(int32_t) + sizeof(float));
}

constexpr size_t native_values_offset(size_t indptr_size, size_t nnz) {
    return kHeaderBytes + indptr_size * sizeof(idx_t) + nnz * sizeof(term_t) +
           padding(kHeaderBytes + indptr_size * sizeof(idx_t) + nnz * sizeof(term_t));
}

constexpr size_t native_file_size(size_t indptr_size, size_t nnz) {
    return native_values_offset(indptr_size, nnz) + nnz * sizeof(float);
}

// `path` with the native suffix appended.
std::string native_path(const std::string& path);

// Writes the interchange file at `interchange_path` in the native layout at
// `native_path`, streaming the nonzeros in fixed-size chunks. Throws
// std::invalid_argument for a missing or malformed source (bad header, size
// of another layout, indptr not running from 0 to nnz, a term >= cols or a
// value that does not fit its narrower native type) and std::runtime_error
// for IO failures.
void convert(const std::string& interchange_path, const std::string& native_path);

}  // namespace nsparse::csr_layout

#endif  // NSPARSE_B200_CSR_LAYOUT_H
