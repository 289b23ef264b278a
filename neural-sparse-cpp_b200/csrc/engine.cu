// Host-side engine: device buffers, workspaces, index uploads and the search
// drivers. See engine.h.
#include "engine.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <string>
#include <utility>

#include "scan.h"

namespace nsp {

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        throw std::runtime_error(std::string("CUDA error in ") + what + ": " +
                                 cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
    }
}

int device_sm_count() {
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    int sms = 0;
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev),
               "cudaDeviceGetAttribute");
    return sms;
}

static int max_smem_optin() {
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    int v = 0;
    cuda_check(cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev),
               "cudaDeviceGetAttribute");
    return v;
}

// ------------------------------------------------------------ workspace --

Workspace::Workspace() {
    cuda_check(cudaGetDevice(&device_), "cudaGetDevice");
    cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
}

Workspace::~Workspace() {
    // Runs at thread exit; the CUDA context may already be gone at process
    // exit, so failures here are ignored.
    for (int i = 0; i < kNumSlots; ++i) {
        if (dptr_[i] != nullptr) cudaFree(dptr_[i]);
        if (hptr_[i] != nullptr) cudaFreeHost(hptr_[i]);
    }
    if (stream_ != nullptr) cudaStreamDestroy(stream_);
}

Workspace& Workspace::get() {
    thread_local std::unique_ptr<Workspace> ws;
    if (!ws) ws.reset(new Workspace());
    return *ws;
}

void* Workspace::dev(int s, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (dcap_[s] < bytes) {
        cuda_check(cudaStreamSynchronize(stream_), "workspace sync");
        if (dptr_[s] != nullptr) cudaFree(dptr_[s]);
        dptr_[s] = nullptr;
        const size_t cap = bytes + bytes / 2;
        cuda_check(cudaMalloc(&dptr_[s], cap), "workspace cudaMalloc");
        dcap_[s] = cap;
    }
    return dptr_[s];
}

void* Workspace::pinned(Slot s, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (hcap_[s] < bytes) {
        cuda_check(cudaStreamSynchronize(stream_), "workspace sync");
        if (hptr_[s] != nullptr) cudaFreeHost(hptr_[s]);
        hptr_[s] = nullptr;
        const size_t cap = bytes + bytes / 2;
        cuda_check(cudaHostAlloc(&hptr_[s], cap, cudaHostAllocDefault), "cudaHostAlloc");
        hcap_[s] = cap;
    }
    return hptr_[s];
}

// ------------------------------------------------------------- host CSR --

void HostCsr::append(int32_t n, const int32_t* ip, const uint16_t* idx, const uint8_t* vals) {
    if (n <= 0) return;
    const int64_t add = static_cast<int64_t>(ip[n]) - ip[0];
    const int64_t base = nnz();
    if (base + add > INT32_MAX) throw std::invalid_argument("too many non-zeros for int32 offsets");
    indices.insert(indices.end(), idx + ip[0], idx + ip[0] + add);
    values.insert(values.end(), vals + static_cast<size_t>(ip[0]) * esz,
                  vals + static_cast<size_t>(ip[0] + add) * esz);
    indptr.reserve(indptr.size() + n);
    for (int32_t i = 1; i <= n; ++i)
        indptr.push_back(static_cast<int32_t>(base + (ip[i] - ip[0])));
}

// -------------------------------------------------------- forward index --

namespace {

__global__ void row_units_kernel(const int32_t* indptr, int32_t n, int64_t* units) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t len = indptr[i + 1] - indptr[i];
        units[i] = (len + kRowAlign - 1) / kRowAlign;
    }
}

// One warp per row: copy ids and value bytes to the padded position, zero
// the padding.
__global__ void pad_rows_kernel(const int32_t* indptr, const uint16_t* idx, const uint8_t* val,
                                int32_t n, int esz, const int64_t* off16, uint2* rowinfo,
                                uint16_t* pidx, uint8_t* pval) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    for (int64_t r = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) >> 5; r < n;
         r += warps) {
        const int64_t s = indptr[r];
        const int64_t len = indptr[r + 1] - s;
        const int64_t dst = off16[r] * kRowAlign;
        const int64_t plen = ((len + kRowAlign - 1) / kRowAlign) * kRowAlign;
        for (int64_t j = lane; j < plen; j += 32) {
            pidx[dst + j] = j < len ? idx[s + j] : static_cast<uint16_t>(0);
        }
        for (int64_t j = lane; j < plen * esz; j += 32) {
            pval[dst * esz + j] = j < len * esz ? val[s * esz + j] : static_cast<uint8_t>(0);
        }
        if (lane == 0) rowinfo[r] = make_uint2(static_cast<uint32_t>(off16[r]),
                                               static_cast<uint32_t>(len));
    }
}

}  // namespace

void ForwardDevice::upload(const HostCsr& h) {
    cudaStream_t s = Workspace::get().stream();
    static std::atomic<uint64_t> uploads{0};
    generation_ = ++uploads;
    n_docs_ = static_cast<int32_t>(h.n());
    dim_ = h.dim;
    esz_ = h.esz;
    if (n_docs_ == 0) {
        rowinfo_.reset();
        idx_.reset();
        val_.reset();
        return;
    }
    const int64_t nnz = h.nnz();
    DevArray<int32_t> d_indptr;
    DevArray<uint16_t> d_idx;
    DevArray<uint8_t> d_val;
    d_indptr.upload(h.indptr.data(), h.indptr.size(), s);
    d_idx.upload(h.indices.data(), static_cast<size_t>(nnz), s);
    d_val.upload(h.values.data(), static_cast<size_t>(nnz) * esz_, s);
    DevArray<int64_t> units(static_cast<size_t>(n_docs_) + 1);
    row_units_kernel<<<std::min<int64_t>((n_docs_ + 255) / 256, 148 * 16), 256, 0, s>>>(
        d_indptr.data(), n_docs_, units.data());
    cuda_check(cudaGetLastError(), "row_units_kernel");
    // exclusive scan in place over n+1 entries (last entry = total units)
    cuda_check(cudaMemsetAsync(units.data() + n_docs_, 0, sizeof(int64_t), s), "memset");
    exclusive_scan_i64(units.data(), units.data(), static_cast<int64_t>(n_docs_) + 1, s);
    int64_t total_units = 0;
    cuda_check(cudaMemcpyAsync(&total_units, units.data() + n_docs_, sizeof(int64_t),
                               cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaStreamSynchronize(s), "sync");
    if (total_units > static_cast<int64_t>(UINT32_MAX))
        throw std::invalid_argument("forward index too large for 32-bit row offsets");
    const size_t padded = static_cast<size_t>(total_units) * kRowAlign;
    rowinfo_.resize(static_cast<size_t>(n_docs_));
    idx_.resize(std::max<size_t>(padded, 16));
    val_.resize(std::max<size_t>(padded * esz_, 16));
    pad_rows_kernel<<<148 * 16, 256, 0, s>>>(d_indptr.data(), d_idx.data(), d_val.data(), n_docs_,
                                             esz_, units.data(), rowinfo_.data(), idx_.data(),
                                             val_.data());
    cuda_check(cudaGetLastError(), "pad_rows_kernel");
    cuda_check(cudaStreamSynchronize(s), "sync");
}

FwdView ForwardDevice::view() const {
    FwdView v;
    v.n_docs = n_docs_;
    v.dim = dim_;
    v.rowinfo = rowinfo_.data();
    v.idx = idx_.data();
    v.val = val_.data();
    return v;
}

size_t ForwardDevice::device_bytes() const {
    return rowinfo_.size() * sizeof(uint2) + idx_.size() * 2 + val_.size();
}

// --------------------------------------------------------- SEISMIC lists --

namespace {

// One CTA per list: the list's summary-term bitmap and per-word prefix.
__global__ void list_meta_kernel(const int64_t* ltp, const uint16_t* sterm, int32_t n_lists,
                                 int words, uint2* lmeta) {
    extern __shared__ uint32_t bits[];
    __shared__ int warp_sums[32];
    for (int32_t t = blockIdx.x; t < n_lists; t += gridDim.x) {
        for (int w = threadIdx.x; w < words; w += blockDim.x) bits[w] = 0u;
        __syncthreads();
        for (int64_t c = ltp[t] + threadIdx.x; c < ltp[t + 1]; c += blockDim.x) {
            const uint32_t term = sterm[c];
            atomicOr(&bits[term >> 5], 1u << (term & 31));
        }
        __syncthreads();
        // exclusive scan of popcounts over `words` entries, chunked per thread
        const int per = (words + blockDim.x - 1) / blockDim.x;
        const int w0 = threadIdx.x * per;
        const int w1 = min(words, w0 + per);
        int local = 0;
        for (int w = w0; w < w1; ++w) local += __popc(bits[w]);
        const int lane = threadIdx.x & 31;
        const int wid = threadIdx.x >> 5;
        int incl = local;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) warp_sums[wid] = incl;
        __syncthreads();
        if (wid == 0) {
            const int nw = blockDim.x >> 5;
            int v = lane < nw ? warp_sums[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, v, o);
                if (lane >= o) v += y;
            }
            if (lane < nw) warp_sums[lane] = v;  // inclusive
        }
        __syncthreads();
        int run = incl - local + (wid > 0 ? warp_sums[wid - 1] : 0);
        uint2* row = lmeta + static_cast<size_t>(t) * words;
        for (int w = w0; w < w1; ++w) {
            row[w] = make_uint2(bits[w], static_cast<uint32_t>(run));
            run += __popc(bits[w]);
        }
        __syncthreads();
    }
}

}  // namespace

namespace {
std::atomic<uint64_t> g_list_generation{0};
}  // namespace

void SeismicDevice::upload(const SeismicHost& h, int dim) {
    cudaStream_t s = Workspace::get().stream();
    generation_ = ++g_list_generation;
    drow_.reset();
    drow_gen_ = 0;
    n_lists_ = h.n_lists();
    words_ = (dim + 31) / 32;
    max_blocks_ = 0;
    for (int32_t t = 0; t < n_lists_; ++t)
        max_blocks_ = std::max<int32_t>(max_blocks_, static_cast<int32_t>(h.lbp[t + 1] - h.lbp[t]));
    lbp_.upload(h.lbp.data(), h.lbp.size(), s);
    bdp_.upload(h.bdp.data(), h.bdp.size(), s);
    docs_.upload(h.docs.data(), h.docs.size(), s);
    ltp_.upload(h.ltp.data(), h.ltp.size(), s);
    srun_.upload(h.srun.data(), h.srun.size(), s);
    esz_ = h.esz;
    sterm_.upload(h.sterm.data(), h.sterm.size(), s);
    sblk_.upload(h.sblk.data(), h.sblk.size(), s);
    sval_.upload(h.sval.data(), h.sval.size(), s);
    if (n_lists_ > 0) {
        lmeta_.resize(static_cast<size_t>(n_lists_) * words_);
        list_meta_kernel<<<std::min(n_lists_, 148 * 8), 256, static_cast<size_t>(words_) * 4, s>>>(
            ltp_.data(), sterm_.data(), n_lists_, words_, lmeta_.data());
        cuda_check(cudaGetLastError(), "list_meta_kernel");
    }
    cuda_check(cudaStreamSynchronize(s), "sync");
}

void SeismicDevice::adopt(const std::vector<int64_t>& lbp, const std::vector<int64_t>& bdp,
                          const std::vector<int64_t>& ltp, int esz, int dim,
                          DevArray<int32_t>&& docs, DevArray<uint16_t>&& sterm,
                          DevArray<int64_t>&& srun, DevArray<uint16_t>&& sblk,
                          DevArray<uint8_t>&& sval) {
    cudaStream_t s = Workspace::get().stream();
    generation_ = ++g_list_generation;
    drow_.reset();
    drow_gen_ = 0;
    n_lists_ = static_cast<int32_t>(lbp.size()) - 1;
    words_ = (dim + 31) / 32;
    max_blocks_ = 0;
    for (int32_t t = 0; t < n_lists_; ++t)
        max_blocks_ = std::max<int32_t>(max_blocks_, static_cast<int32_t>(lbp[t + 1] - lbp[t]));
    esz_ = esz;
    lbp_.upload(lbp.data(), lbp.size(), s);
    bdp_.upload(bdp.data(), bdp.size(), s);
    ltp_.upload(ltp.data(), ltp.size(), s);
    docs_ = std::move(docs);
    sterm_ = std::move(sterm);
    srun_ = std::move(srun);
    sblk_ = std::move(sblk);
    sval_ = std::move(sval);
    if (n_lists_ > 0) {
        lmeta_.resize(static_cast<size_t>(n_lists_) * words_);
        list_meta_kernel<<<std::min(n_lists_, 148 * 8), 256, static_cast<size_t>(words_) * 4, s>>>(
            ltp_.data(), sterm_.data(), n_lists_, words_, lmeta_.data());
        cuda_check(cudaGetLastError(), "list_meta_kernel");
    }
    cuda_check(cudaStreamSynchronize(s), "sync");
}

void SeismicDevice::download(SeismicHost& h) const {
    cudaStream_t s = Workspace::get().stream();
    h.esz = esz_;
    auto get64 = [&](const DevArray<int64_t>& d, std::vector<int64_t>& v, size_t n) {
        v.resize(n);
        d.download(v.data(), n, s);
    };
    const size_t nl = static_cast<size_t>(n_lists_) + 1;
    get64(lbp_, h.lbp, nl);
    cuda_check(cudaStreamSynchronize(s), "sync");
    const size_t nb = static_cast<size_t>(h.lbp.back()) + 1;
    get64(bdp_, h.bdp, nb);
    get64(ltp_, h.ltp, nl);
    cuda_check(cudaStreamSynchronize(s), "sync");
    const size_t nd = static_cast<size_t>(h.bdp.back());
    const size_t nc = static_cast<size_t>(h.ltp.back());
    h.docs.resize(nd);
    docs_.download(h.docs.data(), nd, s);
    h.sterm.resize(nc);
    sterm_.download(h.sterm.data(), nc, s);
    get64(srun_, h.srun, nc + 1);
    cuda_check(cudaStreamSynchronize(s), "sync");
    const size_t ne = static_cast<size_t>(h.srun.back());
    h.sblk.resize(ne);
    sblk_.download(h.sblk.data(), ne, s);
    h.sval.resize(ne * static_cast<size_t>(esz_));
    sval_.download(h.sval.data(), ne * static_cast<size_t>(esz_), s);
    cuda_check(cudaStreamSynchronize(s), "sync");
}

namespace {
__global__ void posting_rows_kernel(const int32_t* docs, int64_t n, const uint2* rowinfo,
                                    int32_t n_docs, uint2* drow) {
    for (int64_t j = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; j < n;
         j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t d = docs[j];
        drow[j] = (d >= 0 && d < n_docs) ? rowinfo[d] : make_uint2(0u, 0u);
    }
}
}  // namespace

void SeismicDevice::bind_rows(const ForwardDevice& fwd, cudaStream_t s) {
    if (fwd.generation() == drow_gen_ && drow_.size() == docs_.size()) return;
    generation_ = ++g_list_generation;
    const int64_t n = static_cast<int64_t>(docs_.size());
    if (n == 0 || fwd.empty()) {
        drow_.reset();
        drow_gen_ = fwd.generation();
        return;
    }
    if (drow_.size() != docs_.size()) drow_.resize(docs_.size());
    posting_rows_kernel<<<device_sm_count() * 8, 256, 0, s>>>(docs_.data(), n, fwd.view().rowinfo,
                                                              fwd.n_docs(), drow_.data());
    cuda_check(cudaGetLastError(), "posting_rows_kernel");
    cuda_check(cudaStreamSynchronize(s), "sync");
    drow_gen_ = fwd.generation();
}

SeismicView SeismicDevice::view() const {
    SeismicView v;
    v.n_lists = n_lists_;
    v.words = words_;
    v.max_blocks = std::max(max_blocks_, 1);
    v.lbp = lbp_.data();
    v.bdp = bdp_.data();
    v.docs = docs_.data();
    v.lmeta = lmeta_.data();
    v.ltp = ltp_.data();
    v.srun = srun_.data();
    v.sblk = sblk_.data();
    v.sval = sval_.data();
    v.drow = (drow_.size() == docs_.size() && drow_.size() > 0) ? drow_.data() : nullptr;
    return v;
}

size_t SeismicDevice::device_bytes() const {
    return (lbp_.size() + bdp_.size() + ltp_.size() + srun_.size()) * 8 + docs_.size() * 4 +
           lmeta_.size() * 8 + sblk_.size() * 2 + sterm_.size() * 2 + sval_.size() +
           drow_.size() * 8;
}

// -------------------------------------------------------------- queries --

QueryBatch canonicalize(int32_t n, const int32_t* indptr, const uint16_t* idx, const float* val,
                        int dim) {
    QueryBatch q;
    q.n = n;
    bool canonical = indptr[0] == 0;
    int32_t max_nnz = 0;
    for (int32_t i = 0; i < n; ++i) {
        const int32_t s = indptr[i], e = indptr[i + 1];
        if (e < s) throw std::invalid_argument("query indptr is not monotonic");
        max_nnz = std::max(max_nnz, e - s);
        for (int32_t j = s; j < e; ++j) {
            if (idx[j] >= dim) throw std::invalid_argument("query term out of range");
            if (j > s && idx[j] <= idx[j - 1]) canonical = false;
        }
    }
    q.max_nnz = max_nnz;
    if (canonical) {
        q.ip = indptr;
        q.ix = idx;
        q.vv = val;
        return q;
    }
    q.indptr.assign(1, 0);
    q.indptr.reserve(n + 1);
    std::vector<std::pair<uint16_t, int32_t>> row;
    max_nnz = 0;
    for (int32_t i = 0; i < n; ++i) {
        const int32_t s = indptr[i], e = indptr[i + 1];
        row.clear();
        for (int32_t j = s; j < e; ++j) row.emplace_back(idx[j], j);
        std::sort(row.begin(), row.end());
        int32_t kept = 0;
        for (size_t r = 0; r < row.size(); ++r) {
            // keep the last occurrence of a repeated term
            if (r + 1 < row.size() && row[r + 1].first == row[r].first) continue;
            q.idx.push_back(row[r].first);
            q.val.push_back(val[row[r].second]);
            ++kept;
        }
        max_nnz = std::max(max_nnz, kept);
        q.indptr.push_back(static_cast<int32_t>(q.idx.size()));
    }
    q.max_nnz = max_nnz;
    q.ip = q.indptr.data();
    q.ix = q.idx.data();
    q.vv = q.val.data();
    return q;
}

// ----------------------------------------------------------- search ------

namespace {

struct Uploaded {
    int32_t* indptr;
    uint16_t* idx;
    float* val;
    int64_t nnz;
};

Uploaded upload_queries(Workspace& ws, const QueryBatch& q) {
    cudaStream_t s = ws.stream();
    const int64_t nnz = q.ip[q.n] - q.ip[0];
    Uploaded u;
    u.nnz = nnz;
    auto* hi = static_cast<int32_t*>(ws.pinned(Workspace::kQIndptr, (q.n + 1) * sizeof(int32_t)));
    auto* hx = static_cast<uint16_t*>(ws.pinned(Workspace::kQIdx, nnz * sizeof(uint16_t)));
    auto* hv = static_cast<float*>(ws.pinned(Workspace::kQVal, nnz * sizeof(float)));
    const int32_t base = q.ip[0];
    for (int32_t i = 0; i <= q.n; ++i) hi[i] = q.ip[i] - base;
    std::memcpy(hx, q.ix + base, nnz * sizeof(uint16_t));
    std::memcpy(hv, q.vv + base, nnz * sizeof(float));
    u.indptr = static_cast<int32_t*>(ws.dev(Workspace::kQIndptr, (q.n + 1) * sizeof(int32_t)));
    u.idx = static_cast<uint16_t*>(ws.dev(Workspace::kQIdx, nnz * sizeof(uint16_t) + 16));
    u.val = static_cast<float*>(ws.dev(Workspace::kQVal, nnz * sizeof(float) + 16));
    cuda_check(cudaMemcpyAsync(u.indptr, hi, (q.n + 1) * sizeof(int32_t), cudaMemcpyHostToDevice, s),
               "H2D queries");
    cuda_check(cudaMemcpyAsync(u.idx, hx, nnz * sizeof(uint16_t), cudaMemcpyHostToDevice, s),
               "H2D queries");
    cuda_check(cudaMemcpyAsync(u.val, hv, nnz * sizeof(float), cudaMemcpyHostToDevice, s),
               "H2D queries");
    return u;
}

const uint64_t* upload_sel(Workspace& ws, const std::vector<uint64_t>* sel) {
    if (sel == nullptr) return nullptr;
    const size_t bytes = sel->size() * sizeof(uint64_t);
    auto* h = static_cast<uint64_t*>(ws.pinned(Workspace::kSel, bytes));
    std::memcpy(h, sel->data(), bytes);
    auto* d = static_cast<uint64_t*>(ws.dev(Workspace::kSel, bytes));
    cuda_check(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, ws.stream()), "H2D selector");
    return d;
}

void download_results(Workspace& ws, int32_t n, int k, const float* dd, const int32_t* dl,
                      float* out_d, int32_t* out_l) {
    cudaStream_t s = ws.stream();
    const size_t cnt = static_cast<size_t>(n) * k;
    auto* hd = static_cast<float*>(ws.pinned(Workspace::kOutD, cnt * sizeof(float)));
    auto* hl = static_cast<int32_t*>(ws.pinned(Workspace::kOutL, cnt * sizeof(int32_t)));
    cuda_check(cudaMemcpyAsync(hd, dd, cnt * sizeof(float), cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaMemcpyAsync(hl, dl, cnt * sizeof(int32_t), cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaStreamSynchronize(s), "search sync");
    std::memcpy(out_d, hd, cnt * sizeof(float));
    std::memcpy(out_l, hl, cnt * sizeof(int32_t));
}

int val_kind_of(int qbits) { return qbits == 0 ? kF32 : (qbits == 8 ? kU8 : kU16); }

struct SeismicPlan {
    int wpb;
    int blocks;
    size_t smem_per_warp;
    int variant;
    int stage_bytes;
    int bcap;
    int batch_docs;   // variants 2-5
    size_t smem_cta;  // variants 2-5
    int group_lanes;  // variants 2-5: lanes per scored doc
    int cluster;      // variants 2-5: CTAs per query
    int seg_cap;      // variants 2-5: block segments per batch
};

}  // namespace

int auto_cluster(int n_queries) {
    const int sms = device_sm_count();
    int c = 1;
    while (c < 8 && static_cast<long long>(std::max(n_queries, 1)) * (c * 2) <= sms) c *= 2;
    return c;
}

namespace {

// Variants 2-5 (one CTA per query). Warps per CTA: 8 when the batch has
// queries enough to give every SM four CTAs; fewer queries get bigger CTAs
// (16 or 32 warps, up to a whole SM per query), which shortens each query's
// sequence of candidate batches -- the latency of small batches and of the
// one-query-per-launch path -- and, below half a query per SM, a cluster of
// 2-8 such CTAs per query (auto_cluster). Candidate docs per batch: 64 per
// warp and CTA unless asked otherwise; the batch shrinks if shared memory is
// short.
SeismicPlan plan_seismic_cta(int kind, int dim, int qcap, int k, int n_queries,
                             const SeismicSearchArgs& args, bool single) {
    SeismicPlan p{};
    p.variant = args.variant;
    int warps = args.warps_per_block;
    if (warps <= 0) {
        const int sms = device_sm_count();
        const int per = single ? 1 : std::max(n_queries, 1);
        warps = 8;
        if (per * 2 <= sms) warps = 32;
        else if (per <= 2 * sms) warps = 16;
    }
    warps = std::min(std::max(warps, 1), 32);
    const size_t limit = static_cast<size_t>(max_smem_optin());
    int cl = args.cluster > 0 ? args.cluster : auto_cluster(single ? 1 : n_queries);
    int seg_cap = 0, batch = 0;
    for (;;) {
        seg_cap = seismic_cta_seg_cap(cl);
        batch = args.batch_docs > 0 ? args.batch_docs : 64 * warps * cl;
        batch = std::min(std::max((batch + 31) & ~31, 32), 8192);
        while (batch > 32 && seismic_cta_smem(kind, dim, qcap, k, batch, seg_cap) > limit)
            batch >>= 1;
        p.smem_cta = seismic_cta_smem(kind, dim, qcap, k, batch, seg_cap);
        // a cluster's larger segment table must not cost the engine's own
        // choice a query it could run on one CTA
        if (p.smem_cta <= limit || args.cluster > 0 || cl == 1) break;
        cl = 1;
    }
    if (p.smem_cta > limit)
        throw std::invalid_argument("query too long or k too large for the device search kernel");
    p.batch_docs = batch;
    p.wpb = warps;
    p.group_lanes = 1 << std::min(std::max(args.variant - 2, 0), 3);  // 2..5 -> 1..8
    p.cluster = cl;
    p.seg_cap = seg_cap;
    int per_sm = seismic_cta_max_blocks_per_sm(kind, qcap, p.group_lanes, warps, p.smem_cta);
    if (per_sm < 1) per_sm = 1;
    // whole clusters; a persistent grid of at most one resident wave
    const int slots = std::max(1, device_sm_count() * per_sm / cl);
    p.blocks = single ? cl : std::max(1, std::min(n_queries, slots)) * cl;
    if (args.max_ctas > 0 && !single)
        p.blocks = std::max(cl, std::min(p.blocks, args.max_ctas / cl * cl));
    return p;
}

// Launch shape of the warp-per-query kernel (variants 0 and 1). The direct
// variant keeps ~2.5x more warps resident, which measured faster at 1M docs
// than the staged variant's larger bytes in flight per warp; the staged variant's
// buffers are 8 KB unless asked otherwise, and its block scores stay in shared
// memory for lists of up to 4096 blocks.
SeismicPlan plan_seismic(int kind, int words, int qcap, int k, int n_queries,
                         const SeismicSearchArgs& args, int max_blocks) {
    SeismicPlan p;
    p.variant = args.variant < 0 ? 0 : args.variant;
    p.stage_bytes = 0;
    p.bcap = 0;
    if (p.variant == 1) {
        p.stage_bytes = args.stage_bytes > 0 ? args.stage_bytes : 8192;
        p.stage_bytes = (p.stage_bytes + 127) & ~127;
        p.bcap = max_blocks <= 4096 ? std::max(max_blocks, 1) : 0;
    }
    p.smem_per_warp = seismic_smem_per_warp(kind, words, qcap, k, p.bcap, p.stage_bytes);
    const size_t limit = static_cast<size_t>(max_smem_optin());
    if (p.smem_per_warp > limit)
        throw std::invalid_argument("query too long or k too large for the device search kernel");
    int wpb = args.warps_per_block > 0 ? std::min(args.warps_per_block, 8)
                                       : (p.variant == 1 ? 2 : 4);
    while (wpb > 1 && p.smem_per_warp * wpb > limit) wpb >>= 1;
    p.wpb = wpb;
    int per_sm = seismic_max_blocks_per_sm(kind, p.variant, wpb, p.smem_per_warp * wpb);
    if (per_sm < 1) per_sm = 1;
    const int want = (n_queries + wpb - 1) / wpb;
    p.blocks = std::max(1, std::min(want, device_sm_count() * per_sm));
    if (args.max_ctas > 0) p.blocks = std::min(p.blocks, args.max_ctas);
    return p;
}

// The engine's choice of kernel: one CTA per query with four lanes per doc
// (variant 4) measured fastest at 1M docs (2.9x variant 0).
constexpr int kDefaultVariant = 4;
// Batched launches with at least this many queries per CTA claim them longest
// row first.
constexpr int kOrderedClaimsPerCta = 4;

}  // namespace

void run_seismic(const ForwardDevice& fwd, const SeismicDevice& ix, int32_t n,
                 const int32_t* d_indptr, const uint16_t* d_idx, const void* d_vals, int32_t qcap,
                 const SeismicSearchArgs& args_in, const uint64_t* d_sel, float* d_out,
                 int32_t* d_lab, cudaStream_t s, Scratch& ws, SearchStats* stats) {
    SeismicSearchArgs args = args_in;
    if (args.variant < 0) args.variant = kDefaultVariant;
    if (args.d_sel_q != nullptr && args.variant < 2)
        throw std::invalid_argument("per-query selectors need a one-CTA-per-query kernel variant");
    const int kind = val_kind_of(args.qbits);
    SeismicLaunch a{};
    a.fwd = fwd.view();
    a.ix = ix.view();
    // The query bitmap spans the vocabulary even when no lists exist (an
    // unbuilt index), so its width comes from the forward index.
    a.ix.words = (a.fwd.dim + 31) / 32;
    if (ix.view().words != 0 && ix.view().words != a.ix.words)
        throw std::runtime_error("SEISMIC lists and forward index disagree on the dimension");
    a.q.n = n;
    a.q.indptr = d_indptr;
    a.q.idx = d_idx;
    a.q.val = d_vals;
    a.k = args.k;
    a.cut = args.cut;
    a.heap_factor = args.heap_factor;
    a.decode_scale = args.decode_scale;
    a.sel_bits = d_sel;
    a.out_d = d_out;
    a.out_l = d_lab;
    a.qcap = std::max(qcap, 1);
    a.nnz_cap = args.nnz_cap;
    auto* st = static_cast<unsigned long long*>(
        ws.dev(Workspace::kStats, kStatCount * sizeof(unsigned long long)));
    cuda_check(cudaMemsetAsync(st, 0, kStatCount * sizeof(unsigned long long), s), "memset");
    a.stats = st;
    // The kernel's own time, only when asked for: an event recorded inside a
    // stream capture would outlive this call in the graph.
    const bool timed = stats != nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (timed) {
        cuda_check(cudaEventCreate(&e0), "event");
        cuda_check(cudaEventCreate(&e1), "event");
    }
    auto mark = [&](cudaEvent_t e) {
        if (timed) cuda_check(cudaEventRecord(e, s), "event");
    };
    int launches = 0;
    auto* err = static_cast<int32_t*>(ws.dev(Workspace::kErr, sizeof(int32_t)));
    cuda_check(cudaMemsetAsync(err, 0, sizeof(int32_t), s), "memset");
    a.err = err;
    if (args.count_unique && (args.variant < 2 || args.plain))
        throw std::invalid_argument("unique-row counting runs on the batched one-CTA-per-query "
                                    "kernels");
    a.visit = nullptr;
    if (args.variant >= 2) {
        SeismicSearchArgs pa = args;
        if (args.count_unique) {
            // one stamp per doc per CTA: a grid of one CTA per SM, one query each
            pa.cluster = 1;
            pa.max_ctas = device_sm_count();
        }
        const SeismicPlan p = plan_seismic_cta(kind, a.fwd.dim, a.qcap, a.k, n, pa, args.plain);
        if (args.count_unique) {
            const size_t stamps = static_cast<size_t>(p.blocks) *
                                  static_cast<size_t>(std::max(a.fwd.n_docs, 1));
            a.visit = static_cast<uint32_t*>(ws.dev(Workspace::kVisit, stamps * sizeof(uint32_t)));
            cuda_check(cudaMemsetAsync(a.visit, 0, stamps * sizeof(uint32_t), s), "memset");
        }
        const int maxb = std::max(ix.max_blocks(), 1);
        a.variant = args.variant;
        a.batch_docs = p.batch_docs;
        a.group_lanes = p.group_lanes;
        a.cluster = p.cluster;
        a.seg_cap = p.seg_cap;
        a.sel_q = args.d_sel_q;
        a.done = args.d_done;
        a.bscore = static_cast<float*>(ws.dev(
            Workspace::kBScore, static_cast<size_t>(p.blocks) * p.wpb * maxb * sizeof(float)));
        a.order_stride = (maxb + 7) & ~7;
        a.order = static_cast<uint16_t*>(ws.dev(
            Workspace::kOrder, static_cast<size_t>(p.blocks) * a.order_stride * sizeof(uint16_t)));
        int p2 = 1;
        while (p2 < maxb) p2 <<= 1;
        a.sortkeys = nullptr;
        a.sort_stride = 0;
        if (p2 > 2 * p.batch_docs) {
            a.sort_stride = p2;
            a.sortkeys = static_cast<unsigned long long*>(
                ws.dev(Workspace::kSortKeys,
                       static_cast<size_t>(p.blocks) * p2 * sizeof(unsigned long long)));
        }
        if (!args.plain) {
            a.work_counter = static_cast<int32_t*>(ws.dev(Workspace::kCounter, sizeof(int32_t)));
            cuda_check(cudaMemsetAsync(a.work_counter, 0, sizeof(int32_t), s), "memset");
            a.first_query = 0;
            // several queries per CTA: the longest rows are claimed first, so
            // the launch does not end on a long query claimed last (16,384
            // SQ queries at 8.8M docs: -1.0%; by a cost estimate from the
            // cut lists' lengths: -1.1%)
            if (n >= kOrderedClaimsPerCta * p.blocks) {
                auto* ord = static_cast<int32_t*>(
                    ws.dev(Workspace::kQOrder, static_cast<size_t>(n) * sizeof(int32_t)));
                cuda_check(launch_order_by_length(d_indptr, n, ord, s), "claim order launch");
                a.qorder = ord;
            }
            mark(e0);
            cuda_check(launch_seismic_cta(kind, a, p.wpb, p.blocks, s), "seismic search launch");
            mark(e1);
            launches = 1;
        } else {
            // one launch per query, one CTA
            a.work_counter = nullptr;
            mark(e0);
            for (int32_t q = 0; q < n; ++q) {
                a.first_query = q;
                a.q.n = q + 1;
                cuda_check(launch_seismic_cta(kind, a, p.wpb, p.blocks, s),
                           "seismic search launch");
            }
            mark(e1);
            launches = n;
        }
    } else if (!args.plain) {
        const SeismicPlan p = plan_seismic(kind, a.ix.words, a.qcap, a.k, n, args, ix.max_blocks());
        a.variant = p.variant;
        a.stage_bytes = p.stage_bytes;
        a.bcap = p.bcap;
        const size_t warps = static_cast<size_t>(p.blocks) * p.wpb;
        a.bscore = static_cast<float*>(
            ws.dev(Workspace::kBScore, warps * one_warp_slot(a.ix.max_blocks) * sizeof(float)));
        a.work_counter = static_cast<int32_t*>(ws.dev(Workspace::kCounter, sizeof(int32_t)));
        cuda_check(cudaMemsetAsync(a.work_counter, 0, sizeof(int32_t), s), "memset");
        a.first_query = 0;
        mark(e0);
        cuda_check(launch_seismic(kind, a, p.wpb, p.blocks, s), "seismic search launch");
        mark(e1);
        launches = 1;
    } else {
        // One launch per query: a single warp walks the query (the per-query
        // path the batched launch is measured against).
        SeismicSearchArgs one = args;
        one.warps_per_block = 1;
        const SeismicPlan p = plan_seismic(kind, a.ix.words, a.qcap, a.k, 1, one, ix.max_blocks());
        a.variant = p.variant;
        a.stage_bytes = p.stage_bytes;
        a.bcap = p.bcap;
        a.bscore = static_cast<float*>(
            ws.dev(Workspace::kBScore, one_warp_slot(a.ix.max_blocks) * sizeof(float)));
        a.work_counter = nullptr;
        mark(e0);
        for (int32_t q = 0; q < n; ++q) {
            a.first_query = q;
            a.q.n = q + 1;
            cuda_check(launch_seismic(kind, a, 1, 1, s), "seismic search launch");
        }
        mark(e1);
        launches = n;
    }
    if (stats != nullptr) {
        unsigned long long h[kStatCount];
        cuda_check(cudaMemcpyAsync(h, st, sizeof(h), cudaMemcpyDeviceToHost, s), "D2H stats");
        cuda_check(cudaStreamSynchronize(s), "sync");
        float ms = 0.0f;
        cuda_check(cudaEventElapsedTime(&ms, e0, e1), "event time");
        stats->docs_scored = h[kStatDocsScored];
        stats->blocks_visited = h[kStatBlocksVisited];
        stats->bytes = h[kStatBytes];
        stats->lists_probed = h[kStatListsProbed];
        stats->kernel_ms = ms;
        stats->launches = launches;
        stats->row_bytes = h[kStatRowBytes];
        stats->unique_docs = h[kStatUniqueDocs];
        stats->unique_row_bytes = h[kStatUniqueRowBytes];
    }
    if (timed) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
}

SeismicScratchNeed seismic_scratch_need(const ForwardDevice& fwd, const SeismicDevice& ix,
                                        int32_t n, int32_t max_nnz,
                                        const SeismicSearchArgs& args_in) {
    SeismicSearchArgs args = args_in;
    if (args.variant < 0) args.variant = kDefaultVariant;
    if (args.plain) throw std::invalid_argument("scratch of a batched search only");
    const int kind = val_kind_of(args.qbits);
    const int qcap = std::max(max_nnz, 1);
    const int maxb = std::max(ix.max_blocks(), 1);
    SeismicScratchNeed need;
    // stats, error word, work counter (run_seismic asks for each), and the
    // claim order of a batched launch of the one-CTA-per-query kernels
    need.fixed = kStatCount * sizeof(unsigned long long) + 2 * sizeof(int32_t);
    if (args.variant >= 2) need.fixed += static_cast<size_t>(n) * sizeof(int32_t);
    if (args.variant >= 2) {
        const SeismicPlan p = plan_seismic_cta(kind, fwd.view().dim, qcap, args.k, n, args, false);
        int p2 = 1;
        while (p2 < maxb) p2 <<= 1;
        need.per_cta = static_cast<size_t>(p.wpb) * maxb * sizeof(float) +
                       static_cast<size_t>((maxb + 7) & ~7) * sizeof(uint16_t) +
                       (p2 > 2 * p.batch_docs ? static_cast<size_t>(p2) * 8 : 0);
        need.ctas = p.blocks;
        need.cluster = p.cluster;
    } else {
        const int words = (fwd.view().dim + 31) / 32;
        const SeismicPlan p = plan_seismic(kind, words, qcap, args.k, n, args, ix.max_blocks());
        need.per_cta = static_cast<size_t>(p.wpb) * one_warp_slot(ix.max_blocks()) * sizeof(float);
        need.ctas = p.blocks;
        need.cluster = 1;
    }
    return need;
}

void reserve_seismic_scratch(const ForwardDevice& fwd, const SeismicDevice& ix, int32_t n,
                             int32_t max_nnz, const SeismicSearchArgs& args_in) {
    if (n <= 0) return;
    SeismicSearchArgs args = args_in;
    if (args.variant < 0) args.variant = kDefaultVariant;
    Workspace& ws = Workspace::get();
    const size_t nq = static_cast<size_t>(n);
    const size_t nnz = nq * static_cast<size_t>(std::max(max_nnz, 1));
    const size_t cnt = nq * static_cast<size_t>(args.k);
    // the sizes upload_queries, download_results and run_seismic ask for
    ws.pinned(Workspace::kQIndptr, (nq + 1) * sizeof(int32_t));
    ws.pinned(Workspace::kQIdx, nnz * sizeof(uint16_t));
    ws.pinned(Workspace::kQVal, nnz * sizeof(float));
    ws.pinned(Workspace::kOutD, cnt * sizeof(float));
    ws.pinned(Workspace::kOutL, cnt * sizeof(int32_t));
    ws.dev(Workspace::kQIndptr, (nq + 1) * sizeof(int32_t));
    ws.dev(Workspace::kQIdx, nnz * sizeof(uint16_t) + 16);
    ws.dev(Workspace::kQVal, nnz * sizeof(float) + 16);
    if (args.qbits != 0) ws.dev(Workspace::kQCode, nnz * 2 + 16);
    ws.dev(Workspace::kOutD, cnt * sizeof(float));
    ws.dev(Workspace::kOutL, cnt * sizeof(int32_t));
    ws.dev(Workspace::kStats, kStatCount * sizeof(unsigned long long));
    ws.dev(Workspace::kErr, sizeof(int32_t));
    ws.dev(Workspace::kCounter, sizeof(int32_t));
    if (args.variant < 2) return;
    const SeismicPlan p = plan_seismic_cta(val_kind_of(args.qbits), fwd.view().dim,
                                           std::max(max_nnz, 1), args.k, n, args, args.plain);
    const int maxb = std::max(ix.max_blocks(), 1);
    const size_t order_stride = static_cast<size_t>((maxb + 7) & ~7);
    ws.dev(Workspace::kBScore, static_cast<size_t>(p.blocks) * p.wpb * maxb * sizeof(float));
    ws.dev(Workspace::kOrder, static_cast<size_t>(p.blocks) * order_stride * sizeof(uint16_t));
    if (!args.plain && n >= kOrderedClaimsPerCta * p.blocks)
        ws.dev(Workspace::kQOrder, static_cast<size_t>(n) * sizeof(int32_t));
    int p2 = 1;
    while (p2 < maxb) p2 <<= 1;
    if (p2 > 2 * p.batch_docs)
        ws.dev(Workspace::kSortKeys,
               static_cast<size_t>(p.blocks) * p2 * sizeof(unsigned long long));
}

namespace {

// Raises if a search kernel on `s` flagged an error (call after sync):
// 1 a bounded wait gave up, 2 a sort buffer was missing, 3 a query longer
// than the launch's query capacity.
void check_kernel_error(Scratch& ws, cudaStream_t s) {
    int32_t h = 0;
    auto* err = static_cast<int32_t*>(ws.dev(Workspace::kErr, sizeof(int32_t)));
    cuda_check(cudaMemcpyAsync(&h, err, sizeof(int32_t), cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaStreamSynchronize(s), "sync");
    if (h == 1) throw std::runtime_error("search kernel gave up waiting for a bulk copy");
    if (h == 2) throw std::runtime_error("search kernel had no buffer to sort a list's blocks");
    if (h == 3) throw std::invalid_argument("a query row is longer than max_nnz");
    if (h != 0) throw std::runtime_error("search kernel reported an error");
}

}  // namespace

void seismic_search(const ForwardDevice& fwd, const SeismicDevice& ix, const QueryBatch& q,
                    const SeismicSearchArgs& args, const std::vector<uint64_t>* sel_bits,
                    float* out_d, int32_t* out_l, SearchStats* stats) {
    Workspace& ws = Workspace::get();
    cudaStream_t s = ws.stream();
    const Uploaded u = upload_queries(ws, q);
    const void* vals = u.val;
    if (args.qbits != 0) {
        void* codes = ws.dev(Workspace::kQCode, static_cast<size_t>(u.nnz) * 2 + 16);
        cuda_check(launch_sq_encode(u.val, codes, u.nnz, args.qbits, args.q_vmin, args.q_scale, s),
                   "query encode");
        vals = codes;
    }
    const uint64_t* d_sel = upload_sel(ws, sel_bits);
    const size_t cnt = static_cast<size_t>(q.n) * args.k;
    auto* dd = static_cast<float*>(ws.dev(Workspace::kOutD, cnt * sizeof(float)));
    auto* dl = static_cast<int32_t*>(ws.dev(Workspace::kOutL, cnt * sizeof(int32_t)));
    run_seismic(fwd, ix, q.n, u.indptr, u.idx, vals, q.max_nnz, args, d_sel, dd, dl, s, ws, stats);
    download_results(ws, q.n, args.k, dd, dl, out_d, out_l);
    check_kernel_error(ws, s);
}

void seismic_search_start(const ForwardDevice& fwd, const SeismicDevice& ix, const QueryBatch& q,
                          const SeismicSearchArgs& args_in, float* out_d, int32_t* out_l,
                          int32_t* done) {
    SeismicSearchArgs args = args_in;
    if (args.variant < 0) args.variant = kDefaultVariant;
    if (args.plain || args.variant < 2 || done == nullptr)
        throw std::invalid_argument("per-query completion needs a batched one-CTA-per-query "
                                    "kernel variant and a flag per query");
    args.d_done = done;
    Workspace& ws = Workspace::get();
    cudaStream_t s = ws.stream();
    const Uploaded u = upload_queries(ws, q);
    const void* vals = u.val;
    if (args.qbits != 0) {
        void* codes = ws.dev(Workspace::kQCode, static_cast<size_t>(u.nnz) * 2 + 16);
        cuda_check(launch_sq_encode(u.val, codes, u.nnz, args.qbits, args.q_vmin, args.q_scale, s),
                   "query encode");
        vals = codes;
    }
    run_seismic(fwd, ix, q.n, u.indptr, u.idx, vals, q.max_nnz, args, nullptr, out_d, out_l, s,
                ws, nullptr);
}

void seismic_search_wait() {
    Workspace& ws = Workspace::get();
    check_kernel_error(ws, ws.stream());
}

void seismic_search_device(const ForwardDevice& fwd, const SeismicDevice& ix, int32_t n,
                           const int32_t* d_indptr, const uint16_t* d_idx, const void* d_val,
                           int32_t max_nnz, const SeismicSearchArgs& args, const uint64_t* d_sel,
                           float* d_out, int32_t* d_lab, cudaStream_t s, SearchStats* stats) {
    Workspace& ws = Workspace::get();
    run_seismic(fwd, ix, n, d_indptr, d_idx, d_val, max_nnz, args, d_sel, d_out, d_lab, s, ws,
                stats);
}

void exact_search(const ForwardDevice& fwd, const PostingsDevice* post, const QueryBatch& q, int k,
                  int mode, const std::vector<uint64_t>* sel_bits, float* out_d, int32_t* out_l,
                  SearchStats* stats) {
    Workspace& ws = Workspace::get();
    cudaStream_t s = ws.stream();
    const Uploaded u = upload_queries(ws, q);
    const uint64_t* d_sel = upload_sel(ws, sel_bits);
    const size_t cnt = static_cast<size_t>(q.n) * k;
    auto* dd = static_cast<float*>(ws.dev(Workspace::kOutD, cnt * sizeof(float)));
    auto* dl = static_cast<int32_t*>(ws.dev(Workspace::kOutL, cnt * sizeof(int32_t)));

    ExactLaunch a{};
    a.fwd = fwd.view();
    a.q.n = q.n;
    a.q.indptr = u.indptr;
    a.q.idx = u.idx;
    a.q.val = u.val;
    a.k = k;
    a.mode = mode;
    a.sel_bits = d_sel;
    a.qcap = std::max(q.max_nnz, 1);
    a.out_d = dd;
    a.out_l = dl;
    const bool taat = post != nullptr && post->usable() &&
                      post->generation() == fwd.generation() && k <= kTaatMaxK;
    const int words = (fwd.view().dim + 31) / 32;
    const size_t limit = static_cast<size_t>(max_smem_optin());
    const bool values_global = exact_smem(words, a.qcap) > limit;
    if (!taat && exact_smem(words, 0) > limit)
        throw std::invalid_argument("vocabulary too large for the exact search kernel");
    const int groups = (q.n + 31) / 32;
    const int sms = device_sm_count();
    int tiles = std::max(1, (2 * sms + groups - 1) / groups);
    const int32_t nd = std::max(fwd.n_docs(), 1);
    tiles = std::min(tiles, std::max(1, nd / 64));
    a.docs_per_tile = (nd + tiles - 1) / tiles;
    tiles = (nd + a.docs_per_tile - 1) / a.docs_per_tile;
    if (taat) {
        // term at a time: candidates per (query, doc chunk), no per-lane lists
        a.post = post->view();
        const size_t cands = static_cast<size_t>(q.n) * a.post.n_chunks * k;
        a.cand_d = static_cast<float*>(ws.dev(Workspace::kCandD, cands * sizeof(float)));
        a.cand_l = static_cast<int32_t*>(ws.dev(Workspace::kCandL, cands * sizeof(int32_t)));
    } else {
        const size_t lanes = static_cast<size_t>(groups) * tiles * 8 * 32;
        a.heap_d = static_cast<float*>(ws.dev(Workspace::kHeapD, lanes * k * sizeof(float)));
        a.heap_l = static_cast<int32_t*>(ws.dev(Workspace::kHeapL, lanes * k * sizeof(int32_t)));
        const size_t cands = static_cast<size_t>(groups) * 32 * tiles * k;
        a.cand_d = static_cast<float*>(ws.dev(Workspace::kCandD, cands * sizeof(float)));
        a.cand_l = static_cast<int32_t*>(ws.dev(Workspace::kCandL, cands * sizeof(int32_t)));
        a.qval_global = values_global
                            ? static_cast<float*>(ws.dev(Workspace::kQValG,
                                                         static_cast<size_t>(groups) * tiles * 32 *
                                                             a.qcap * sizeof(float)))
                            : nullptr;
    }
    auto* st = static_cast<unsigned long long*>(
        ws.dev(Workspace::kStats, kStatCount * sizeof(unsigned long long)));
    cuda_check(cudaMemsetAsync(st, 0, kStatCount * sizeof(unsigned long long), s), "memset");
    a.stats = st;
    cudaEvent_t e0, e1;
    cuda_check(cudaEventCreate(&e0), "event");
    cuda_check(cudaEventCreate(&e1), "event");
    cuda_check(cudaEventRecord(e0, s), "event");
    if (fwd.n_docs() > 0) {
        cuda_check(taat ? launch_exact_taat(a, s) : launch_exact(a, tiles, s),
                   "exact search launch");
    } else {
        cuda_check(cudaMemsetAsync(dd, 0, cnt * sizeof(float), s), "memset");
    }
    cuda_check(cudaEventRecord(e1, s), "event");
    if (fwd.n_docs() == 0) {
        // nothing indexed: every slot is padding
        cuda_check(cudaStreamSynchronize(s), "sync");
        for (size_t i = 0; i < cnt; ++i) {
            out_d[i] = -1.0f;
            out_l[i] = -1;
        }
    } else {
        download_results(ws, q.n, k, dd, dl, out_d, out_l);
    }
    if (stats != nullptr) {
        unsigned long long h[kStatCount];
        cuda_check(cudaMemcpyAsync(h, st, sizeof(h), cudaMemcpyDeviceToHost, s), "D2H stats");
        cuda_check(cudaStreamSynchronize(s), "sync");
        float ms = 0.0f;
        cuda_check(cudaEventElapsedTime(&ms, e0, e1), "event time");
        stats->bytes = h[kStatBytes];
        stats->kernel_ms = ms;
        stats->launches = 2;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}

void exact_list_search(const ForwardDevice& fwd, const QueryBatch& q, const SeismicSearchArgs& args,
                       const std::vector<int32_t>& ids, float* out_d, int32_t* out_l) {
    Workspace& ws = Workspace::get();
    cudaStream_t s = ws.stream();
    const Uploaded u = upload_queries(ws, q);
    const void* vals = u.val;
    if (args.qbits != 0) {
        void* codes = ws.dev(Workspace::kQCode, static_cast<size_t>(u.nnz) * 2 + 16);
        cuda_check(launch_sq_encode(u.val, codes, u.nnz, args.qbits, args.q_vmin, args.q_scale, s),
                   "query encode");
        vals = codes;
    }
    auto* hid = static_cast<int32_t*>(ws.pinned(Workspace::kIds, ids.size() * sizeof(int32_t) + 4));
    std::memcpy(hid, ids.data(), ids.size() * sizeof(int32_t));
    auto* did = static_cast<int32_t*>(ws.dev(Workspace::kIds, ids.size() * sizeof(int32_t) + 4));
    cuda_check(cudaMemcpyAsync(did, hid, ids.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s),
               "H2D ids");
    const size_t cnt = static_cast<size_t>(q.n) * args.k;
    auto* dd = static_cast<float*>(ws.dev(Workspace::kOutD, cnt * sizeof(float)));
    auto* dl = static_cast<int32_t*>(ws.dev(Workspace::kOutL, cnt * sizeof(int32_t)));
    QueryView qv;
    qv.n = q.n;
    qv.indptr = u.indptr;
    qv.idx = u.idx;
    qv.val = vals;
    cuda_check(launch_exact_list(val_kind_of(args.qbits), fwd.view(), qv, did,
                                 static_cast<int>(ids.size()), args.k, args.decode_scale,
                                 std::max(q.max_nnz, 1), dd, dl, s),
               "exact list launch");
    download_results(ws, q.n, args.k, dd, dl, out_d, out_l);
}

}  // namespace nsp
