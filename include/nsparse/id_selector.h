// Document filters (reference: nsparse/id_selector.h:22-86). Each selector can
// also fill a bitmap over document ids; the engine turns the selector of a
// search into such a bitmap in device memory and tests one bit per scored
// document instead of a hash lookup.
#ifndef NSPARSE_B200_ID_SELECTOR_H
#define NSPARSE_B200_ID_SELECTOR_H

#include <algorithm>
#include <climits>
#include <cstddef>
#include <cstdint>
#include <unordered_set>
#include <vector>

#include "nsparse/types.h"

namespace nsparse {

class IDSelector {
public:
    virtual ~IDSelector() = default;
    virtual bool is_member(idx_t id) const = 0;
    // Extension: membership of a 64-bit id (an IDMapIndex's external ids).
    // The default answers is_member for ids that fit 32 bits and false
    // otherwise.
    virtual bool is_member64(int64_t id) const {
        return id >= INT32_MIN && id <= INT32_MAX && is_member(static_cast<idx_t>(id));
    }
    bool operator()(idx_t id) const { return is_member(id); }
    // Sets bit d of `bits` (n_docs bits, zero on entry) for every member d in
    // [0, n_docs). The default asks is_member for every id.
    virtual void fill_bitmap(uint64_t* bits, int64_t n_docs) const;
};

class IDSelectorEnumerable : public IDSelector {
public:
    ~IDSelectorEnumerable() override = default;
    virtual std::vector<idx_t> ids() const = 0;
    virtual std::vector<idx_t> ordered_ids() const {
        auto v = ids();
        std::sort(v.begin(), v.end());
        return v;
    }
    virtual size_t size() const = 0;
    // Extension: the ids at 64 bits (the default widens ids()).
    virtual std::vector<int64_t> ids64() const {
        const std::vector<idx_t> v = ids();
        return {v.begin(), v.end()};
    }
    void fill_bitmap(uint64_t* bits, int64_t n_docs) const override;
};

class SetIDSelector : public IDSelectorEnumerable {
public:
    SetIDSelector(size_t n, const idx_t* indices) : ids_(indices, indices + n) {}
    bool is_member(idx_t id) const override { return ids_.count(id) != 0; }
    std::vector<idx_t> ids() const override { return {ids_.begin(), ids_.end()}; }
    size_t size() const override { return ids_.size(); }

private:
    std::unordered_set<idx_t> ids_;
};

class ArrayIDSelector : public IDSelectorEnumerable {
public:
    ArrayIDSelector(size_t n, const idx_t* indices) : ids_(indices, indices + n) {}
    bool is_member(idx_t id) const override {
        return std::find(ids_.begin(), ids_.end(), id) != ids_.end();
    }
    std::vector<idx_t> ids() const override { return ids_; }
    size_t size() const override { return ids_.size(); }

private:
    std::vector<idx_t> ids_;
};

// Not owning: `selector` must outlive this object (as in the reference).
class NotIDSelector : public IDSelector {
public:
    explicit NotIDSelector(IDSelector* selector) : delegate_(selector) {}
    bool is_member(idx_t id) const override { return !delegate_->is_member(id); }
    void fill_bitmap(uint64_t* bits, int64_t n_docs) const override;
    const IDSelector* delegate() const { return delegate_; }

private:
    IDSelector* delegate_;
};

// Extension: a set of 64-bit ids, for an IDMapIndex whose external ids need
// them. ids() lists the members that fit 32 bits; size() counts them all.
class SetIDSelector64 : public IDSelectorEnumerable {
public:
    SetIDSelector64(size_t n, const int64_t* indices) : ids_(indices, indices + n) {}
    bool is_member(idx_t id) const override { return ids_.count(id) != 0; }
    bool is_member64(int64_t id) const override { return ids_.count(id) != 0; }
    std::vector<idx_t> ids() const override {
        std::vector<idx_t> out;
        for (int64_t v : ids_)
            if (v >= INT32_MIN && v <= INT32_MAX) out.push_back(static_cast<idx_t>(v));
        return out;
    }
    std::vector<int64_t> ids64() const override { return {ids_.begin(), ids_.end()}; }
    size_t size() const override { return ids_.size(); }

private:
    std::unordered_set<int64_t> ids_;
};

// Extension: a ready-made membership bitmap over ids [0, n_bits) (bit d of
// word d/64). Ids outside the range are not members. The bits are copied.
class BitmapIDSelector : public IDSelector {
public:
    BitmapIDSelector(int64_t n_bits, const uint64_t* bits);
    bool is_member(idx_t id) const override;
    void fill_bitmap(uint64_t* bits, int64_t n_docs) const override;

private:
    int64_t n_bits_;
    std::vector<uint64_t> bits_;
};

}  // namespace nsparse

#endif
