// Exact inverted index (reference: nsparse/inverted_index.h). Returns the
// exact top-k among documents with a positive score, honouring id selectors.
// The GPU scores every resident document exactly, which for the reference's
// positive-valued inputs is the set its MaxScore traversal ranks.
#ifndef NSPARSE_B200_INVERTED_INDEX_H
#define NSPARSE_B200_INVERTED_INDEX_H

#include <array>
#include <memory>

#include "nsparse/index.h"

namespace nsparse {
class IOReader;
class IOWriter;
namespace detail {
struct ForwardState;
}

class InvertedIndex : public Index {
public:
    explicit InvertedIndex(int dim);
    ~InvertedIndex() override;
    InvertedIndex(const InvertedIndex&) = delete;
    InvertedIndex& operator=(const InvertedIndex&) = delete;
    void add(idx_t n, const idx_t* indptr, const term_t* indices, const float* values) override;
    void build() override;
    size_t num_vectors() const override;
    std::array<char, 4> id() const override { return name; }
    static constexpr std::array<char, 4> name = {'I', 'N', 'V', 'T'};

    void write_index(IOWriter* writer);
    void read_index(IOReader* reader, int io_flags = 0);

protected:
    void search_impl(idx_t n, const idx_t* indptr, const term_t* indices, const float* values,
                     int k, float* distances, idx_t* labels,
                     SearchParameters* search_parameters) override;

private:
    std::unique_ptr<detail::ForwardState> fwd_;
    bool built_ = false;
};

}  // namespace nsparse

#endif
