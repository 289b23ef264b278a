// Index persistence in the reference's on-disk layout, so files move both
// ways between this engine and the reference:
//   header              u32 fourcc + i32 dimension        io/index_io.cpp:88-116
//   SparseVectors       sparse_vectors.cpp:206-231
//   InvertedListClusters cluster/inverted_list_clusters.cpp:333-363
//   SEISMIC lists       io/seismic_invlists_writer.h:36-43
//   SQ quantizer header seismic_scalar_quantized_index.cpp:421-438
//   IDMap               id_map_index.cpp:81-109
//   Inverted            inverted_index.cpp:367-447
// Arrays are padded to their element alignment against the absolute stream
// position (io/align.h:43-104). Loading validates every offset and id the
// kernels will dereference, so a corrupt file is rejected on the host.
#include <algorithm>
#include <array>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "index_state.h"
#include "nsparse/brutal_index.h"
#include "nsparse/id_map_index.h"
#include "nsparse/inverted_index.h"
#include "nsparse/io/index_io.h"
#include "nsparse/seismic_index.h"
#include "nsparse/seismic_scalar_quantized_index.h"

namespace nsparse {

namespace {

constexpr uint32_t fourcc(const std::array<char, 4>& id) {
    return static_cast<uint32_t>(static_cast<uint8_t>(id[0])) |
           static_cast<uint32_t>(static_cast<uint8_t>(id[1])) << 8 |
           static_cast<uint32_t>(static_cast<uint8_t>(id[2])) << 16 |
           static_cast<uint32_t>(static_cast<uint8_t>(id[3])) << 24;
}

class FileWriter : public IOWriter {
public:
    explicit FileWriter(const char* name) {
        f_ = std::fopen(name, "wb");
        if (f_ == nullptr) throw std::runtime_error("Failed to open file for writing");
    }
    ~FileWriter() override {
        if (f_ != nullptr) std::fclose(f_);
    }
    void write(const void* p, size_t size, size_t n) override {
        if (n == 0 || size == 0) return;
        if (std::fwrite(p, size, n, f_) != n) throw std::runtime_error("Failed to write to file");
        pos_ += size * n;
    }
    size_t pos() const override { return pos_; }
    void close() override {
        if (f_ != nullptr) {
            const int rc = std::fclose(f_);
            f_ = nullptr;
            if (rc != 0) throw std::runtime_error("Failed to close file");
        }
    }

private:
    FILE* f_ = nullptr;
    size_t pos_ = 0;
};

class FileReader : public IOReader {
public:
    explicit FileReader(const char* name) {
        f_ = std::fopen(name, "rb");
        if (f_ == nullptr) throw std::runtime_error("Failed to open file for reading");
        std::fseek(f_, 0, SEEK_END);
        size_ = static_cast<size_t>(std::ftell(f_));
        std::fseek(f_, 0, SEEK_SET);
    }
    ~FileReader() override {
        if (f_ != nullptr) std::fclose(f_);
    }
    size_t read(void* p, size_t size, size_t n) override {
        const size_t got = n == 0 ? 0 : std::fread(p, size, n, f_);
        pos_ += got * size;
        return got;
    }
    size_t pos() const override { return pos_; }
    size_t remaining() const { return size_ - pos_; }
    void close() override {
        if (f_ != nullptr) {
            std::fclose(f_);
            f_ = nullptr;
        }
    }

private:
    FILE* f_ = nullptr;
    size_t pos_ = 0;
    size_t size_ = 0;
};

// --------------------------------------------------------------- writing --

void pad_to(IOWriter* w, size_t align) {
    static const uint8_t zeros[8] = {};
    const size_t n = (align - w->pos() % align) % align;
    if (n > 0) w->write(zeros, 1, n);
}

template <class T>
void write_scalar(IOWriter* w, T v) {
    w->write(&v, sizeof(T), 1);
}

template <class T>
void write_padded(IOWriter* w, const T* p, size_t n, size_t align = alignof(T)) {
    pad_to(w, align);
    if (n > 0) w->write(p, sizeof(T), n);
}

void write_sparse_vectors(IOWriter* w, const nsp::HostCsr& h, int dim) {
    const size_t count = static_cast<size_t>(h.n());
    write_scalar<size_t>(w, count);
    if (count == 0) return;
    write_scalar<size_t>(w, static_cast<size_t>(dim));
    write_scalar<size_t>(w, static_cast<size_t>(h.esz));
    write_padded(w, h.indptr.data(), count + 1);
    const size_t nnz = static_cast<size_t>(h.nnz());
    write_padded(w, h.indices.data(), nnz);
    write_padded(w, h.values.data(), nnz * h.esz, static_cast<size_t>(h.esz));
}

void write_lists(IOWriter* w, const nsp::SeismicHost& L, const std::vector<uint8_t>& list_esz) {
    const size_t n_lists = static_cast<size_t>(L.n_lists());
    write_scalar<size_t>(w, n_lists);
    for (size_t t = 0; t < n_lists; ++t) {
        const int64_t b0 = L.lbp[t], b1 = L.lbp[t + 1];
        const int64_t nb = b1 - b0;
        const int64_t d0 = L.bdp[b0], d1 = L.bdp[b1];
        write_scalar<size_t>(w, static_cast<size_t>(d1 - d0));
        write_padded(w, L.docs.data() + d0, static_cast<size_t>(d1 - d0));
        std::vector<int32_t> offsets;
        if (nb > 0) {
            offsets.resize(static_cast<size_t>(nb) + 1);
            for (int64_t b = b0; b <= b1; ++b) offsets[b - b0] = static_cast<int32_t>(L.bdp[b] - d0);
        }
        write_scalar<size_t>(w, offsets.size());
        write_padded(w, offsets.data(), offsets.size());
        const size_t esz = t < list_esz.size() ? list_esz[t] : static_cast<size_t>(L.esz);
        write_scalar<size_t>(w, static_cast<size_t>(nb));
        write_scalar<size_t>(w, esz);
        const int64_t c0 = L.ltp[t], c1 = L.ltp[t + 1];
        write_scalar<size_t>(w, static_cast<size_t>(c1 - c0));
        if (c1 > c0) {
            write_padded(w, L.sterm.data() + c0, static_cast<size_t>(c1 - c0));
            std::vector<int32_t> tp(static_cast<size_t>(c1 - c0) + 1);
            for (int64_t c = c0; c <= c1; ++c) tp[c - c0] = static_cast<int32_t>(L.srun[c] - L.srun[c0]);
            write_padded(w, tp.data(), tp.size());
        }
        const int64_t e0 = L.srun[c0], e1 = L.srun[c1];
        write_scalar<size_t>(w, static_cast<size_t>(e1 - e0));
        write_padded(w, L.sblk.data() + e0, static_cast<size_t>(e1 - e0));
        write_padded(w, L.sval.data() + e0 * L.esz, static_cast<size_t>(e1 - e0) * L.esz, esz);
    }
}

// --------------------------------------------------------------- reading --

[[noreturn]] void corrupt(const char* what) {
    throw std::runtime_error(std::string("corrupt index file: ") + what);
}

template <class T>
T read_scalar(IOReader* r) {
    T v{};
    if (r->read(&v, sizeof(T), 1) != 1) throw std::runtime_error("Truncated index file");
    return v;
}

void skip_padding(IOReader* r, size_t align) {
    uint8_t buf[8];
    const size_t n = (align - r->pos() % align) % align;
    if (n > 0 && r->read(buf, 1, n) != n) throw std::runtime_error("Truncated index file");
}

template <class T>
std::vector<T> read_padded(IOReader* r, size_t n, size_t align = alignof(T)) {
    skip_padding(r, align);
    if (auto* fr = dynamic_cast<FileReader*>(r)) {
        if (n > fr->remaining() / sizeof(T)) throw std::runtime_error("Truncated array in index file");
    }
    std::vector<T> v(n);
    if (n > 0 && r->read(v.data(), sizeof(T), n) != n)
        throw std::runtime_error("Truncated array in index file");
    return v;
}

// Returns the CSR; esz_expected = 0 accepts any width.
nsp::HostCsr read_sparse_vectors(IOReader* r, int dim) {
    nsp::HostCsr h;
    h.dim = dim;
    const size_t count = read_scalar<size_t>(r);
    if (count == 0) return h;
    if (count > static_cast<size_t>(std::numeric_limits<int32_t>::max()))
        corrupt("implausible vector count");
    (void)read_scalar<size_t>(r);  // dimension recorded with the vectors
    const size_t esz = read_scalar<size_t>(r);
    if (esz != 1 && esz != 2 && esz != 4) corrupt("unsupported element size");
    h.esz = static_cast<int>(esz);
    h.indptr = read_padded<int32_t>(r, count + 1);
    if (h.indptr[0] != 0) corrupt("indptr must start at 0");
    for (size_t i = 1; i <= count; ++i)
        if (h.indptr[i] < h.indptr[i - 1]) corrupt("indptr is not monotonic");
    const size_t nnz = static_cast<size_t>(h.indptr[count]);
    h.indices = read_padded<uint16_t>(r, nnz);
    for (uint16_t t : h.indices)
        if (t >= dim) corrupt("term out of range");
    h.values = read_padded<uint8_t>(r, nnz * esz, esz);
    return h;
}

void read_lists(IOReader* r, nsp::SeismicHost& L, std::vector<uint8_t>& list_esz, int esz,
                int dim, int64_t n_docs) {
    const size_t n_lists = read_scalar<size_t>(r);
    if (n_lists > 65536) corrupt("implausible list count");
    L = nsp::SeismicHost();
    L.esz = esz;
    list_esz.assign(n_lists, static_cast<uint8_t>(esz));
    for (size_t t = 0; t < n_lists; ++t) {
        const size_t n_ldocs = read_scalar<size_t>(r);
        std::vector<int32_t> docs = read_padded<int32_t>(r, n_ldocs);
        const size_t n_off = read_scalar<size_t>(r);
        std::vector<int32_t> off = read_padded<int32_t>(r, n_off);
        const size_t n_clusters = read_scalar<size_t>(r);
        const size_t lesz = read_scalar<size_t>(r);
        const size_t n_terms = read_scalar<size_t>(r);
        std::vector<uint16_t> terms;
        std::vector<int32_t> tp;
        if (n_terms > 0) {
            terms = read_padded<uint16_t>(r, n_terms);
            tp = read_padded<int32_t>(r, n_terms + 1);
        }
        const size_t nnz = read_scalar<size_t>(r);
        std::vector<uint16_t> cl = read_padded<uint16_t>(r, nnz);
        if (lesz != 1 && lesz != 2 && lesz != 4) corrupt("unsupported summary element size");
        std::vector<uint8_t> vals = read_padded<uint8_t>(r, nnz * lesz, lesz);
        list_esz[t] = static_cast<uint8_t>(lesz);
        // validation: every offset and id a kernel will follow
        const size_t nb = n_off > 0 ? n_off - 1 : 0;
        if (n_off > 0 && (off[0] != 0 || static_cast<size_t>(off[nb]) != n_ldocs))
            corrupt("cluster offsets do not cover the docs");
        if (n_off == 0 && n_ldocs != 0) corrupt("docs without cluster offsets");
        for (size_t b = 1; b < n_off; ++b)
            if (off[b] < off[b - 1]) corrupt("cluster offsets not monotonic");
        for (int32_t d : docs)
            if (d < 0 || d >= n_docs) corrupt("doc id out of range");
        if (n_clusters > nb) corrupt("more summaries than clusters");
        for (size_t c = 0; c < n_terms; ++c) {
            if (terms[c] >= dim) corrupt("summary term out of range");
            if (c > 0 && terms[c] <= terms[c - 1]) corrupt("summary terms not ascending");
        }
        if (n_terms > 0) {
            if (tp[0] != 0 || static_cast<size_t>(tp[n_terms]) != nnz) corrupt("summary offsets");
            for (size_t c = 1; c <= n_terms; ++c)
                if (tp[c] < tp[c - 1]) corrupt("summary offsets not monotonic");
        } else if (nnz != 0) {
            corrupt("summary entries without terms");
        }
        for (uint16_t b : cl)
            if (b >= nb) corrupt("summary block id out of range");
        if (nnz > 0 && static_cast<int>(lesz) != esz)
            corrupt("summary element size disagrees with the index");
        // append
        const int64_t dbase = static_cast<int64_t>(L.docs.size());
        L.docs.insert(L.docs.end(), docs.begin(), docs.end());
        for (size_t b = 1; b < n_off; ++b) L.bdp.push_back(dbase + off[b]);
        L.lbp.push_back(L.lbp.back() + static_cast<int64_t>(nb));
        const int64_t ebase = L.srun.back();
        L.sterm.insert(L.sterm.end(), terms.begin(), terms.end());
        for (size_t c = 1; c <= n_terms; ++c) L.srun.push_back(ebase + tp[c]);
        L.ltp.push_back(L.ltp.back() + static_cast<int64_t>(n_terms));
        L.sblk.insert(L.sblk.end(), cl.begin(), cl.end());
        L.sval.insert(L.sval.end(), vals.begin(), vals.end());
    }
}

}  // namespace

// ---------------------------------------------------------- per-class IO --

void SeismicIndex::write_index(IOWriter* w) {
    write_sparse_vectors(w, st_->vectors.host, dimension_);
    if (st_->host_valid || st_->dev_valid) {
        write_lists(w, st_->host_lists(), st_->list_esz);
    } else {
        write_scalar<size_t>(w, 0);
    }
}

void SeismicIndex::read_index(IOReader* r, int) {
    nsp::HostCsr h = read_sparse_vectors(r, dimension_);
    if (h.n() > 0 && h.esz != 4) throw std::runtime_error("index file's element size is not the seismic index's");
    h.esz = 4;
    read_lists(r, st_->lists, st_->list_esz, 4, dimension_, h.n());
    st_->vectors.host = std::move(h);
    st_->vectors.host.dim = dimension_;
    st_->vectors.dirty = true;
    st_->host_valid = true;
    st_->dev_valid = false;
}

void SeismicScalarQuantizedIndex::write_index(IOWriter* w) {
    write_scalar<uint8_t>(w, static_cast<uint8_t>(sq_.get_quantizer_type()));
    write_scalar<float>(w, sq_.get_min());
    write_scalar<float>(w, sq_.get_max());
    write_sparse_vectors(w, st_->vectors.host, dimension_);
    if (st_->host_valid || st_->dev_valid) {
        write_lists(w, st_->host_lists(), st_->list_esz);
    } else {
        write_scalar<size_t>(w, 0);
    }
}

void SeismicScalarQuantizedIndex::read_index(IOReader* r, int) {
    const uint8_t qt = read_scalar<uint8_t>(r);
    const float vmin = read_scalar<float>(r);
    const float vmax = read_scalar<float>(r);
    if (qt != static_cast<uint8_t>(QuantizerType::QT_8bit) &&
        qt != static_cast<uint8_t>(QuantizerType::QT_16bit))
        throw std::runtime_error("index file declares an unknown quantizer type");
    sq_ = ScalarQuantizer(static_cast<QuantizerType>(qt), vmin, vmax);
    const int esz = static_cast<int>(sq_.bytes_per_value());
    nsp::HostCsr h = read_sparse_vectors(r, dimension_);
    if (h.n() > 0 && h.esz != esz)
        throw std::runtime_error("index file's element size disagrees with its quantizer type");
    h.esz = esz;
    st_->lists.esz = esz;
    read_lists(r, st_->lists, st_->list_esz, esz, dimension_, h.n());
    st_->vectors.host = std::move(h);
    st_->vectors.host.dim = dimension_;
    st_->vectors.dirty = true;
    st_->host_valid = true;
    st_->dev_valid = false;
}

void InvertedIndex::write_index(IOWriter* w) {
    const nsp::HostCsr& h = fwd_->host;
    write_scalar<size_t>(w, static_cast<size_t>(h.n()));
    const size_t n_terms = built_ ? static_cast<size_t>(dimension_) : 0;
    write_scalar<size_t>(w, n_terms);
    write_scalar<size_t>(w, 4);
    if (n_terms > 0) {
        // posting lists, doc ascending (invlists/inverted_lists.cpp:159-180)
        std::vector<int64_t> cnt(n_terms + 1, 0);
        for (uint16_t t : h.indices) cnt[t + 1]++;
        for (size_t t = 0; t < n_terms; ++t) cnt[t + 1] += cnt[t];
        std::vector<int32_t> pdoc(h.indices.size());
        std::vector<float> pval(h.indices.size());
        std::vector<int64_t> cur(cnt.begin(), cnt.end() - 1);
        const float* vals = reinterpret_cast<const float*>(h.values.data());
        for (int64_t d = 0; d < h.n(); ++d) {
            for (int32_t j = h.indptr[d]; j < h.indptr[d + 1]; ++j) {
                const int64_t p = cur[h.indices[j]]++;
                pdoc[p] = static_cast<int32_t>(d);
                pval[p] = vals[j];
            }
        }
        std::vector<float> maxv(n_terms, 0.0F);
        for (size_t t = 0; t < n_terms; ++t) {
            const size_t len = static_cast<size_t>(cnt[t + 1] - cnt[t]);
            write_scalar<size_t>(w, len);
            if (len > 0) {
                w->write(pdoc.data() + cnt[t], sizeof(int32_t), len);
                w->write(pval.data() + cnt[t], sizeof(float), len);
                for (size_t i = 0; i < len; ++i) maxv[t] = std::max(maxv[t], pval[cnt[t] + i]);
            }
        }
        write_scalar<size_t>(w, n_terms);
        w->write(maxv.data(), sizeof(float), n_terms);
    } else {
        write_scalar<size_t>(w, 0);
    }
}

void InvertedIndex::read_index(IOReader* r, int) {
    const size_t n_docs = read_scalar<size_t>(r);
    const size_t n_terms = read_scalar<size_t>(r);
    const size_t esz = read_scalar<size_t>(r);
    if (esz != 4) throw std::runtime_error("inverted index file declares an unsupported element width");
    if (n_docs > static_cast<size_t>(std::numeric_limits<int32_t>::max())) corrupt("document count");
    if (n_terms > 65536) corrupt("implausible term count");
    std::vector<std::vector<std::pair<uint16_t, float>>> rows(n_docs);
    for (size_t t = 0; t < n_terms; ++t) {
        const size_t len = read_scalar<size_t>(r);
        if (len == 0) continue;
        std::vector<int32_t> docs = read_padded<int32_t>(r, len, 1);
        std::vector<float> vals = read_padded<float>(r, len, 1);
        for (size_t i = 0; i < len; ++i) {
            if (docs[i] < 0 || static_cast<size_t>(docs[i]) >= n_docs) corrupt("doc id out of range");
            rows[docs[i]].emplace_back(static_cast<uint16_t>(t), vals[i]);
        }
    }
    const size_t n_scores = read_scalar<size_t>(r);
    (void)read_padded<float>(r, n_scores, 1);
    nsp::HostCsr h;
    h.dim = dimension_;
    h.esz = 4;
    for (const auto& row : rows) {
        for (const auto& [t, v] : row) {
            h.indices.push_back(t);
            const auto* b = reinterpret_cast<const uint8_t*>(&v);
            h.values.insert(h.values.end(), b, b + 4);
        }
        h.indptr.push_back(static_cast<int32_t>(h.indices.size()));
    }
    fwd_->host = std::move(h);
    fwd_->dirty = true;
    built_ = n_terms > 0;
}

// The reference's IDMP layout (id_map_index.cpp:82-99): the id count, then
// 32-bit ids. A map with ids beyond 32 bits is written under the name64 tag
// with 64-bit ids (engine extension).
void IDMapIndex::write_index(IOWriter* w) {
    write_scalar<size_t>(w, internal_to_external_.size());
    if (wide_) {
        if (!internal_to_external_.empty())
            w->write(internal_to_external_.data(), sizeof(int64_t), internal_to_external_.size());
    } else {
        std::vector<idx_t> narrow(internal_to_external_.begin(), internal_to_external_.end());
        if (!narrow.empty()) w->write(narrow.data(), sizeof(idx_t), narrow.size());
    }
    nsparse::write_index(delegate_.get(), w);
}

namespace detail {
Index* read_index_nested(IOReader* r, int io_flags);
}

void IDMapIndex::read_index(IOReader* r, int io_flags, bool wide) {
    const size_t m = read_scalar<size_t>(r);
    if (wide) {
        internal_to_external_ = read_padded<int64_t>(r, m, 1);
    } else {
        const std::vector<idx_t> narrow = read_padded<idx_t>(r, m, 1);
        internal_to_external_.assign(narrow.begin(), narrow.end());
    }
    delegate_.reset(detail::read_index_nested(r, io_flags));
    external_to_internal_.clear();
    wide_ = false;
    for (size_t i = 0; i < m; ++i) {
        const int64_t e = internal_to_external_[i];
        external_to_internal_[e] = static_cast<idx_t>(i);
        wide_ = wide_ || e < INT32_MIN || e > INT32_MAX;
    }
}

// ------------------------------------------------------------ free API --

void write_index(Index* index, IOWriter* w) {
    if (index == nullptr) throw std::invalid_argument("unexpected nullptr");
    const uint32_t id = fourcc(index->id());
    auto header = [&] {
        write_scalar<uint32_t>(w, id);
        write_scalar<int32_t>(w, index->get_dimension());
    };
    if (auto* s = dynamic_cast<SeismicIndex*>(index)) {
        header();
        s->write_index(w);
    } else if (auto* q = dynamic_cast<SeismicScalarQuantizedIndex*>(index)) {
        header();
        q->write_index(w);
    } else if (auto* m = dynamic_cast<IDMapIndex*>(index)) {
        write_scalar<uint32_t>(w, m->wide_ids() ? fourcc(IDMapIndex::name64) : id);
        write_scalar<int32_t>(w, index->get_dimension());
        m->write_index(w);
    } else if (auto* v = dynamic_cast<InvertedIndex*>(index)) {
        header();
        v->write_index(w);
    } else {
        throw std::runtime_error("Index does not support serialization");
    }
}

void write_index(Index* index, const char* file_name) {
    if (file_name == nullptr) throw std::invalid_argument("unexpected nullptr");
    if (index == nullptr) throw std::invalid_argument("unexpected nullptr");
    if (dynamic_cast<SeismicIndex*>(index) == nullptr &&
        dynamic_cast<SeismicScalarQuantizedIndex*>(index) == nullptr &&
        dynamic_cast<IDMapIndex*>(index) == nullptr && dynamic_cast<InvertedIndex*>(index) == nullptr)
        throw std::runtime_error("Index does not support serialization");
    FileWriter w(file_name);
    write_index(index, &w);
    w.close();
}

namespace detail {
Index* read_index_nested(IOReader* r, int io_flags) {
    const uint32_t id = read_scalar<uint32_t>(r);
    const int32_t dim = read_scalar<int32_t>(r);
    if (dim < 0 || dim > 65536) corrupt("dimension");
    std::unique_ptr<Index> idx;
    if (id == fourcc(SeismicIndex::name)) {
        auto* p = new SeismicIndex(dim);
        idx.reset(p);
        p->read_index(r, io_flags);
    } else if (id == fourcc(SeismicScalarQuantizedIndex::name)) {
        auto* p = new SeismicScalarQuantizedIndex(dim);
        idx.reset(p);
        p->read_index(r, io_flags);
    } else if (id == fourcc(IDMapIndex::name) || id == fourcc(IDMapIndex::name64)) {
        auto* p = new IDMapIndex();
        idx.reset(p);
        p->read_index(r, io_flags, id == fourcc(IDMapIndex::name64));
    } else if (id == fourcc(InvertedIndex::name)) {
        auto* p = new InvertedIndex(dim);
        idx.reset(p);
        p->read_index(r, io_flags);
    } else if (id == fourcc(BrutalIndex::name)) {
        throw std::runtime_error("Index does not support serialization");
    } else {
        throw std::runtime_error("Unknown index type");
    }
    return idx.release();
}
}  // namespace detail

Index* read_index(IOReader* r, int io_flags) { return detail::read_index_nested(r, io_flags); }

Index* read_index(const char* file_name, int io_flags) {
    if (file_name == nullptr) throw std::invalid_argument("unexpected nullptr");
    FileReader r(file_name);
    Index* idx = read_index(&r, io_flags);
    r.close();
    return idx;
}

}  // namespace nsparse
