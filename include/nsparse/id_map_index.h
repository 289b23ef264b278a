// External-id wrapper (reference: nsparse/id_map_index.h:27-110). Owns its
// delegate. Selectors given to search() are expressed in external ids and are
// translated to the delegate's internal ids; returned labels are external.
#ifndef NSPARSE_B200_ID_MAP_INDEX_H
#define NSPARSE_B200_ID_MAP_INDEX_H

#include <array>
#include <memory>
#include <unordered_map>
#include <vector>

#include "nsparse/index.h"

namespace nsparse {
class IOReader;
class IOWriter;

class IDMapIndex : public Index {
public:
    IDMapIndex() = default;
    static constexpr std::array<char, 4> name = {'I', 'D', 'M', 'P'};
    explicit IDMapIndex(Index* delegate);  // takes ownership
    std::array<char, 4> id() const override { return name; }
    void add(idx_t n, const idx_t* indptr, const term_t* indices, const float* values) override;
    void build() override;
    void search(idx_t n, const idx_t* indptr, const term_t* indices, const float* values, int k,
                float* distances, idx_t* labels,
                SearchParameters* search_parameters = nullptr) override;
    size_t num_vectors() const override;
    void add_with_ids(idx_t n, const idx_t* indptr, const term_t* indices, const float* values,
                      const idx_t* ids) override;
    Index* delegate() { return delegate_.get(); }
    const std::vector<idx_t>& internal_to_external() const { return internal_to_external_; }

    void write_index(IOWriter* writer);
    void read_index(IOReader* reader, int io_flags = 0);

protected:
    void search_impl(idx_t, const idx_t*, const term_t*, const float*, int, float*, idx_t*,
                     SearchParameters*) override {}

private:
    std::unique_ptr<Index> delegate_;
    std::vector<idx_t> internal_to_external_;
    std::unordered_map<idx_t, idx_t> external_to_internal_;
};

}  // namespace nsparse

#endif
