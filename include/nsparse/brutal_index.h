// Exact brute-force index (reference: nsparse/brutal_index.h). Every document
// is scored on the GPU; zero scores are eligible; id selectors are ignored,
// as in the reference.
#ifndef NSPARSE_B200_BRUTAL_INDEX_H
#define NSPARSE_B200_BRUTAL_INDEX_H

#include <array>
#include <memory>

#include "nsparse/index.h"

namespace nsparse {
namespace detail {
struct ForwardState;
}

class BrutalIndex : public Index {
public:
    explicit BrutalIndex(int dim = 0);
    ~BrutalIndex() override;
    BrutalIndex(const BrutalIndex&) = delete;
    BrutalIndex& operator=(const BrutalIndex&) = delete;
    void add(idx_t n, const idx_t* indptr, const term_t* indices, const float* values) override;
    size_t num_vectors() const override;
    std::array<char, 4> id() const override { return name; }
    static constexpr std::array<char, 4> name = {'B', 'R', 'U', 'T'};

protected:
    void search_impl(idx_t n, const idx_t* indptr, const term_t* indices, const float* values,
                     int k, float* distances, idx_t* labels,
                     SearchParameters* search_parameters) override;

private:
    std::unique_ptr<detail::ForwardState> fwd_;
};

}  // namespace nsparse

#endif
