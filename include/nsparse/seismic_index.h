// SEISMIC approximate index (reference: nsparse/seismic_index.h,
// nsparse/seismic_common.h). build() clusters the posting lists and builds the
// block summaries on the GPU; search() runs the block-pruned traversal on the
// GPU.
#ifndef NSPARSE_B200_SEISMIC_INDEX_H
#define NSPARSE_B200_SEISMIC_INDEX_H

#include <array>
#include <memory>

#include "nsparse/index.h"

namespace nsparse {
class IOReader;
class IOWriter;

// Reference: seismic_common.h:38-47. lambda = posting cap per term (-1:
// max(0.0005 * n_docs, 160)); beta = blocks per list (-1: int(0.1 * lambda));
// alpha = summary mass kept; seed = -1 draws a fresh seed per build.
constexpr int kRandomSeed = -1;
struct SeismicClusterParameters {
    int lambda;
    int beta;
    float alpha;
    int inverted_list_batch_size = 1;
    char* batch_file_output_path = nullptr;
    int seed = kRandomSeed;
};

struct SeismicSearchParameters : public SearchParameters {
    int cut = 10;
    float heap_factor = 1.0F;
    SeismicSearchParameters(int cut, float heap_factor) : cut(cut), heap_factor(heap_factor) {}
    SeismicSearchParameters() = default;
};

namespace detail {
struct SeismicState;
}

class SeismicIndex : public Index {
public:
    static constexpr std::array<char, 4> name = {'S', 'E', 'I', 'S'};
    explicit SeismicIndex(int dim);
    SeismicIndex(int dim, SeismicClusterParameters parameter);
    ~SeismicIndex() override;
    SeismicIndex(const SeismicIndex&) = delete;
    SeismicIndex& operator=(const SeismicIndex&) = delete;
    std::array<char, 4> id() const override { return name; }
    void add(idx_t n, const idx_t* indptr, const term_t* indices, const float* values) override;
    void build() override;
    size_t num_vectors() const override;
    // MmapIndex::read_csr (mmap_index.h:24-36): Residency::kMmap reads the
    // native layout (nsparse/utils/csr_layout.h), into an index that holds no
    // vectors yet; kInMemory the interchange layout (Index::read_csr).
    void read_csr(const char* file_path, Residency residency = Residency::kInMemory) override;

    void write_index(IOWriter* writer);
    void read_index(IOReader* reader, int io_flags = 0);
    detail::SeismicState* state() { return st_.get(); }

protected:
    void search_impl(idx_t n, const idx_t* indptr, const term_t* indices, const float* values,
                     int k, float* distances, idx_t* labels,
                     SearchParameters* search_parameters) override;

private:
    SeismicClusterParameters cluster_parameter_;
    std::unique_ptr<detail::SeismicState> st_;
};

}  // namespace nsparse

#endif
