// External-id wrapper (reference: nsparse/id_map_index.h:27-110). Owns its
// delegate. Selectors given to search() are expressed in external ids and are
// translated to the delegate's internal ids; returned labels are external.
#ifndef NSPARSE_B200_ID_MAP_INDEX_H
#define NSPARSE_B200_ID_MAP_INDEX_H

#include <array>
#include <cstdint>
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
    // File tag of a map whose external ids need 64 bits (engine extension;
    // maps whose ids all fit 32 bits keep the reference's IDMP layout).
    static constexpr std::array<char, 4> name64 = {'I', 'D', 'M', '8'};
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
    // Extension with no counterpart in the reference (whose idx_t is 32
    // bits): external ids of 64 bits. search() keeps returning 32-bit labels
    // while every external id fits them and raises std::invalid_argument once
    // one does not; search64() returns the ids whatever their width. An
    // id selector given to either names external ids; SetIDSelector64 names
    // 64-bit ones.
    void add_with_ids64(idx_t n, const idx_t* indptr, const term_t* indices, const float* values,
                        const int64_t* ids);
    void search64(idx_t n, const idx_t* indptr, const term_t* indices, const float* values, int k,
                  float* distances, int64_t* labels,
                  SearchParameters* search_parameters = nullptr);
    // Some external id needs more than 32 bits (the file is then written with
    // the name64 tag and 64-bit ids).
    bool wide_ids() const { return wide_; }
    Index* delegate() { return delegate_.get(); }
    const std::vector<int64_t>& internal_to_external() const { return internal_to_external_; }

    void write_index(IOWriter* writer);
    void read_index(IOReader* reader, int io_flags = 0, bool wide = false);

protected:
    void search_impl(idx_t, const idx_t*, const term_t*, const float*, int, float*, idx_t*,
                     SearchParameters*) override {}

private:
    void map_ids(size_t first, idx_t n, const int64_t* ids);
    // The delegate's search with the caller's selector translated to
    // internal ids; labels stay internal.
    void search_internal(idx_t n, const idx_t* indptr, const term_t* indices,
                         const float* values, int k, float* distances, idx_t* labels,
                         SearchParameters* params);

    std::unique_ptr<Index> delegate_;
    std::vector<int64_t> internal_to_external_;
    std::unordered_map<int64_t, idx_t> external_to_internal_;
    bool wide_ = false;
};

}  // namespace nsparse

#endif
