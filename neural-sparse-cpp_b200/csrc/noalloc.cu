// SEISMIC search that allocates nothing, for callers that cannot allocate
// device memory per call: an engine embedded in a host whose allocator
// accounts for every device byte against a fixed budget (a JVM plugin, a
// serving process with admission control), or a latency-critical loop that
// cannot afford cudaMalloc/cudaFree, which can synchronize the whole device.
//
// The search kernel's scratch (its work counter, the encoded query codes of a
// quantized index, and the per-warp block-score rows) lives in the file-scope
// device array below instead of the engine's per-thread workspace. Every GPU
// that loads the library reserves kNoAllocScratchBytes for it until exit.
#include <cuda_runtime.h>

#include <mutex>
#include <stdexcept>
#include <string>

#include "engine.h"
#include "index_state.h"
#include "nsp_device.h"
#include "nsparse/seismic_index.h"
#include "nsparse/seismic_scalar_quantized_index.h"
#include "nsparse_c.h"

namespace {

constexpr size_t kNoAllocScratchBytes = size_t{32} << 20;  // NSP_NOALLOC_SCRATCH_BYTES
static_assert(kNoAllocScratchBytes == NSP_NOALLOC_SCRATCH_BYTES, "header and library disagree");

// Shared by every call on a device; contents persist between calls.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device. In host code the
// symbol names a host-side stand-in, so the address is looked up once per
// device (with that device current) and cached.
void* scratch_on_current_device() {
    int dev = 0;
    nsp::cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) throw std::runtime_error("device ordinal out of range");
    std::lock_guard<std::mutex> g(g_mu);
    if (g_scratch_ptr[dev] == nullptr) {
        void* p = nullptr;
        nsp::cuda_check(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress");
        g_scratch_ptr[dev] = p;
    }
    return g_scratch_ptr[dev];
}

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

namespace nsp {
void set_last_error(const char* msg);  // capi.cpp
}

extern "C" nsp_status_t nsp_index_search_device_noalloc(
    nsp_index_t* index, int32_t n, const int32_t* d_indptr, const uint16_t* d_indices,
    const float* d_values, int32_t nnz, int32_t max_row_nnz, int k, float* d_distances,
    int32_t* d_labels, const nsp_search_params_t* params, void* cuda_stream) {
    using namespace nsparse;
    try {
        if (index == nullptr || d_indptr == nullptr || d_indices == nullptr ||
            d_values == nullptr || d_distances == nullptr || d_labels == nullptr)
            throw std::invalid_argument("unexpected nullptr");
        if (n <= 0 || k <= 0) throw std::invalid_argument("value must be positive");
        if (nnz < 0 || max_row_nnz < 0) throw std::invalid_argument("nnz must not be negative");
        auto* base = reinterpret_cast<Index*>(index);
        const auto* sp = reinterpret_cast<const SearchParameters*>(params);
        if (sp != nullptr && sp->get_id_selector() != nullptr)
            throw std::invalid_argument("the no-allocation search takes no id selector");
        if (sp != nullptr && sp->engine.plain)
            throw std::invalid_argument("the no-allocation search runs batched only");
        const auto* ssp = dynamic_cast<const SeismicSearchParameters*>(sp);
        const SeismicSearchParameters defaults;
        if (ssp == nullptr) ssp = &defaults;
        if (ssp->cut <= 0) throw std::invalid_argument("value must be positive");

        detail::SeismicState* st = nullptr;
        int val_kind = nsp::kF32;
        int qbits = 0;
        float q_vmin = 0.0F, q_scale = 0.0F, decode = 0.0F;
        if (auto* si = dynamic_cast<SeismicIndex*>(base)) {
            st = si->state();
        } else if (auto* qi = dynamic_cast<SeismicScalarQuantizedIndex*>(base)) {
            st = qi->state();
            const ScalarQuantizer& isq = qi->get_scalar_quantizer();
            const auto* sqp = dynamic_cast<const SeismicSQSearchParameters*>(sp);
            const ScalarQuantizer qsq =
                sqp == nullptr ? isq : ScalarQuantizer(isq.get_quantizer_type(), sqp->vmin, sqp->vmax);
            qbits = isq.bits();
            val_kind = qbits == 8 ? nsp::kU8 : nsp::kU16;
            q_vmin = qsq.get_min();
            q_scale = qsq.encode_scale();
            decode = isq.decode_scale(qsq);
        } else {
            throw std::invalid_argument("the no-allocation search supports seismic indexes");
        }
        // Uploading the index allocates; it must already be resident (any
        // earlier search or build leaves it so).
        if (st->vectors.dirty || st->vectors.dev.empty() || !st->dev_valid)
            throw std::invalid_argument(
                "index is not resident on the GPU: run one ordinary search first");

        nsp::SeismicLaunch a{};
        a.fwd = st->vectors.dev.view();
        a.ix = st->lists_dev.view();
        a.ix.words = (a.fwd.dim + 31) / 32;
        a.q.n = n;
        a.q.indptr = d_indptr;
        a.q.idx = d_indices;
        a.k = k;
        a.cut = ssp->cut;
        a.heap_factor = ssp->heap_factor;
        a.decode_scale = decode;
        a.out_d = d_distances;
        a.out_l = d_labels;
        a.qcap = max_row_nnz > 0 ? max_row_nnz : 1;
        a.stats = nullptr;
        a.first_query = 0;

        // scratch layout: [counter | query codes | block-score rows]
        auto* scratch = static_cast<unsigned char*>(scratch_on_current_device());
        const size_t codes_bytes = qbits == 0 ? 0 : align256(static_cast<size_t>(nnz) * 2 + 16);
        const size_t head = 256 + codes_bytes;
        if (head >= kNoAllocScratchBytes)
            throw std::invalid_argument("query batch too large for the no-allocation scratch (" +
                                        std::to_string(kNoAllocScratchBytes) + " bytes)");
        const size_t row_bytes = static_cast<size_t>(a.ix.max_blocks) * sizeof(float);
        const size_t rows = (kNoAllocScratchBytes - head) / row_bytes;
        if (rows < 1)
            throw std::invalid_argument("posting lists have too many blocks for the no-allocation "
                                        "scratch");
        const size_t per_warp = nsp::seismic_smem_per_warp(val_kind, a.ix.words, a.qcap, k);
        int wpb = 4;
        while (wpb > 1 && static_cast<size_t>(wpb) > rows) wpb >>= 1;
        int per_sm = nsp::seismic_max_blocks_per_sm(val_kind, wpb, per_warp * wpb);
        if (per_sm < 1) per_sm = 1;
        long long blocks_ll = std::min<long long>((n + wpb - 1) / wpb,
                                                  static_cast<long long>(nsp::device_sm_count()) * per_sm);
        blocks_ll = std::min<long long>(blocks_ll, static_cast<long long>(rows / wpb));
        int blocks = static_cast<int>(blocks_ll);
        if (blocks < 1) blocks = 1;

        auto* stream = static_cast<cudaStream_t>(cuda_stream);
        a.work_counter = reinterpret_cast<int32_t*>(scratch);
        nsp::cuda_check(cudaMemsetAsync(a.work_counter, 0, sizeof(int32_t), stream), "memset");
        a.q.val = d_values;
        if (qbits != 0) {
            void* codes = scratch + 256;
            nsp::cuda_check(nsp::launch_sq_encode(d_values, codes, nnz, qbits, q_vmin, q_scale, stream),
                            "query encode");
            a.q.val = codes;
        }
        a.bscore = reinterpret_cast<float*>(scratch + head);
        nsp::cuda_check(nsp::launch_seismic(val_kind, a, wpb, blocks, stream), "seismic search");
        return NSP_OK;
    } catch (const std::invalid_argument& e) {
        nsp::set_last_error(e.what());
        return NSP_ERR_INVALID_ARGUMENT;
    } catch (const std::exception& e) {
        nsp::set_last_error(e.what());
        return NSP_ERR_RUNTIME;
    }
}
