// CSR file layouts (include/nsparse/utils/csr_layout.h): conversion from the
// interchange layout to the native one, and the native-layout reader behind
// SeismicIndex::read_csr(path, Residency::kMmap). Host code only; the rows
// reach the device through the index's forward-index upload.
#include "nsparse/utils/csr_layout.h"

#include <algorithm>
#include <array>
#include <filesystem>
#include <fstream>
#include <limits>
#include <stdexcept>
#include <vector>

#include "csr_layout_read.h"

namespace nsparse::csr_layout {
namespace {

constexpr size_t kChunk = size_t{1} << 16;  // elements per streamed chunk

// Checks that every value fits the narrower native type.
template <class Narrow, class Wide>
void check_fits(const std::vector<Wide>& v, size_t n, const char* what, const std::string& path) {
    for (size_t i = 0; i < n; ++i)
        if (v[i] < 0 || static_cast<uint64_t>(v[i]) >
                            static_cast<uint64_t>(std::numeric_limits<Narrow>::max()))
            throw std::invalid_argument(std::string(what) +
                                        " does not fit the native CSR width in: " + path);
}

void write_bytes(std::ofstream& f, const void* src, size_t n, const std::string& path) {
    f.write(static_cast<const char*>(src), static_cast<std::streamsize>(n));
    if (!f) throw std::runtime_error("Failed writing CSR file: " + path);
}

void read_bytes(std::ifstream& f, void* dst, size_t n, const std::string& path) {
    f.read(static_cast<char*>(dst), static_cast<std::streamsize>(n));
    if (!f) throw std::runtime_error("Truncated CSR file: " + path);
}

}  // namespace

std::string native_path(const std::string& path) { return path + kNativeSuffix; }

void convert(const std::string& src, const std::string& dst) {
    if (!std::filesystem::exists(src)) throw std::invalid_argument("CSR file does not exist: " + src);
    std::ifstream in(src, std::ios::binary);
    if (!in.is_open()) throw std::runtime_error("Cannot open CSR file: " + src);
    std::array<int64_t, 3> header{};
    read_bytes(in, header.data(), sizeof(header), src);
    const int64_t rows = header[0], cols = header[1], nnz = header[2];
    if (rows <= 0 || cols <= 0 || nnz < 0)
        throw std::invalid_argument("Invalid CSR header in: " + src);
    const size_t np = static_cast<size_t>(rows) + 1, nz = static_cast<size_t>(nnz);
    if (std::filesystem::file_size(src) != interchange_file_size(np, nz))
        throw std::invalid_argument("CSR file is not in the interchange layout: " + src);
    std::ofstream out(dst, std::ios::binary | std::ios::trunc);
    if (!out.is_open()) throw std::runtime_error("Cannot open CSR file for writing: " + dst);
    write_bytes(out, header.data(), sizeof(header), dst);

    std::vector<int64_t> ip(np);
    read_bytes(in, ip.data(), np * sizeof(int64_t), src);
    if (ip.front() != 0 || ip.back() != nnz)
        throw std::invalid_argument("Inconsistent CSR indptr in: " + src);
    check_fits<idx_t>(ip, np, "indptr", src);
    const std::vector<idx_t> ip32(ip.begin(), ip.end());
    write_bytes(out, ip32.data(), np * sizeof(idx_t), dst);

    std::vector<int32_t> wide(std::min(kChunk, std::max<size_t>(nz, 1)));
    std::vector<term_t> narrow(wide.size());
    for (size_t done = 0; done < nz;) {
        const size_t n = std::min(kChunk, nz - done);
        read_bytes(in, wide.data(), n * sizeof(int32_t), src);
        for (size_t i = 0; i < n; ++i)
            if (wide[i] >= cols) throw std::invalid_argument("CSR term out of range in: " + src);
        check_fits<term_t>(wide, n, "term", src);
        for (size_t i = 0; i < n; ++i) narrow[i] = static_cast<term_t>(wide[i]);
        write_bytes(out, narrow.data(), n * sizeof(term_t), dst);
        done += n;
    }
    const std::array<char, sizeof(float)> zeros{};
    const size_t pad = padding(kHeaderBytes + np * sizeof(idx_t) + nz * sizeof(term_t));
    if (pad > 0) write_bytes(out, zeros.data(), pad, dst);
    std::vector<float> vals(wide.size());
    for (size_t done = 0; done < nz;) {
        const size_t n = std::min(kChunk, nz - done);
        read_bytes(in, vals.data(), n * sizeof(float), src);
        write_bytes(out, vals.data(), n * sizeof(float), dst);
        done += n;
    }
    out.flush();
    if (!out) throw std::runtime_error("Failed writing CSR file: " + dst);
}

}  // namespace nsparse::csr_layout

namespace nsparse::detail {

// The checks of the reference's mapped reader (mmap_index.h:72-131 and
// SparseVectors::map_vectors, sparse_vectors.cpp:28-83), on a copy: header,
// 32-bit limits, columns within the index dimension, the exact native file
// size, and an indptr that starts at 0, never decreases and ends at nnz.
// Terms are not scanned, as there; a term >= the dimension is rejected
// before the GPU sees it, by build() and search().
NativeCsr read_native_csr(const char* path, int dimension) {
    if (path == nullptr) throw std::invalid_argument("file_path must not be null");
    if (!std::filesystem::exists(path))
        throw std::invalid_argument(std::string("CSR file does not exist: ") + path);
    const std::string p(path);
    std::ifstream in(p, std::ios::binary);
    if (!in.is_open()) throw std::runtime_error("Cannot open CSR file: " + p);
    std::array<int64_t, 3> header{};
    csr_layout::read_bytes(in, header.data(), sizeof(header), p);
    const int64_t rows = header[0], cols = header[1], nnz = header[2];
    if (rows <= 0 || cols <= 0 || nnz < 0) throw std::invalid_argument("Invalid CSR header in: " + p);
    if (rows > std::numeric_limits<idx_t>::max() || nnz > std::numeric_limits<idx_t>::max())
        throw std::invalid_argument("CSR file too large for 32-bit offsets: " + p);
    if (cols > dimension)
        throw std::invalid_argument("CSR column count exceeds index dimension: " + p);
    const size_t np = static_cast<size_t>(rows) + 1, nz = static_cast<size_t>(nnz);
    if (std::filesystem::file_size(p) != csr_layout::native_file_size(np, nz))
        throw std::invalid_argument(
            "CSR file is not in the native layout (convert it with csr_layout::convert): " + p);
    NativeCsr c;
    c.rows = static_cast<idx_t>(rows);
    c.indptr.resize(np);
    c.indices.resize(nz);
    c.values.resize(nz);
    csr_layout::read_bytes(in, c.indptr.data(), np * sizeof(idx_t), p);
    csr_layout::read_bytes(in, c.indices.data(), nz * sizeof(term_t), p);
    in.seekg(static_cast<std::streamoff>(csr_layout::native_values_offset(np, nz)));
    csr_layout::read_bytes(in, c.values.data(), nz * sizeof(float), p);
    if (c.indptr[0] != 0) throw std::invalid_argument("Mapped indptr must start at 0");
    for (size_t i = 1; i < np; ++i)
        if (c.indptr[i] < c.indptr[i - 1])
            throw std::invalid_argument("Mapped indptr is not monotonic");
    if (static_cast<size_t>(c.indptr[np - 1]) != nz)
        throw std::invalid_argument("Mapped indptr does not end at the index count");
    return c;
}

}  // namespace nsparse::detail
