// SEISMIC over scalar-quantized values (reference:
// nsparse/seismic_scalar_quantized_index.h). Values are stored as 8- or 16-bit
// codes; scores are integer code products summed exactly on the GPU, then
// decoded (utils/scalar_quantizer.h:85-93).
#ifndef NSPARSE_B200_SEISMIC_SQ_INDEX_H
#define NSPARSE_B200_SEISMIC_SQ_INDEX_H

#include <array>
#include <memory>

#include "nsparse/seismic_index.h"
#include "nsparse/utils/scalar_quantizer.h"

namespace nsparse {

struct SeismicSQSearchParameters : public SeismicSearchParameters {
    float vmin;
    float vmax;
    SeismicSQSearchParameters(float vmin, float vmax, int cut, float heap_factor)
        : SeismicSearchParameters(cut, heap_factor), vmin(vmin), vmax(vmax) {}
};

class SeismicScalarQuantizedIndex : public Index {
public:
    static constexpr std::array<char, 4> name = {'S', 'E', 'S', 'Q'};
    explicit SeismicScalarQuantizedIndex(int dim);
    SeismicScalarQuantizedIndex(QuantizerType quantizer_type, float vmin, float vmax,
                                SeismicClusterParameters parameter, int dim);
    ~SeismicScalarQuantizedIndex() override;
    SeismicScalarQuantizedIndex(const SeismicScalarQuantizedIndex&) = delete;
    SeismicScalarQuantizedIndex& operator=(const SeismicScalarQuantizedIndex&) = delete;
    std::array<char, 4> id() const override { return name; }
    void add(idx_t n, const idx_t* indptr, const term_t* indices, const float* values) override;
    void build() override;
    size_t num_vectors() const override;
    const ScalarQuantizer& get_scalar_quantizer() const { return sq_; }
    void read_csr(const char* file_path, Residency residency = Residency::kInMemory) override;

    void write_index(IOWriter* writer);
    void read_index(IOReader* reader, int io_flags = 0);
    detail::SeismicState* state() { return st_.get(); }

protected:
    void search_impl(idx_t n, const idx_t* indptr, const term_t* indices, const float* values,
                     int k, float* distances, idx_t* labels,
                     SearchParameters* search_parameters) override;

private:
    ScalarQuantizer query_quantizer(const SearchParameters* params) const;
    ScalarQuantizer sq_;
    SeismicClusterParameters cluster_parameter_;
    std::unique_ptr<detail::SeismicState> st_;
};

}  // namespace nsparse

#endif
