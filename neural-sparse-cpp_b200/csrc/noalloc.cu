// SEISMIC search that allocates nothing, for callers that cannot allocate
// device memory per call: an engine embedded in a host whose allocator
// accounts for every device byte against a fixed budget (a JVM plugin, a
// serving process with admission control), or a latency-critical loop that
// cannot afford cudaMalloc/cudaFree, which can synchronize the whole device.
//
// The search is the engine's ordinary batched search (run_seismic: the
// one-CTA-per-query kernel unless the parameters ask for another, the
// index's autotuned launch shape when they leave the choice to the engine),
// with every scratch buffer it asks for -- work counter, counters, block-score
// rows, visiting orders, sort keys, the encoded query codes of a quantized
// index -- carved from the file-scope device array below instead of the
// per-thread workspace. The grid is capped to the CTAs whose block-score rows
// fit the array. Every GPU that loads the library reserves
// kNoAllocScratchBytes for it until exit.
#include <cuda_runtime.h>

#include <algorithm>
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

// Hands out 256-byte aligned regions of one fixed device range in the order a
// search asks for its scratch slots; a slot asked for again gets its region
// back. The error slot is the caller's status word when one is given. Nothing
// is allocated: a request beyond the range is refused.
class FixedScratch final : public nsp::Scratch {
public:
    FixedScratch(unsigned char* base, size_t cap, int32_t* status)
        : base_(base), cap_(cap), status_(status) {}
    void* dev(int slot, size_t bytes) override {
        if (slot == nsp::Workspace::kErr && status_ != nullptr) return status_;
        if (slot < 0 || slot >= nsp::Workspace::kNumSlots)
            throw std::runtime_error("unknown scratch slot");
        if (ptr_[slot] != nullptr) {
            if (bytes <= size_[slot]) return ptr_[slot];
            throw std::runtime_error("scratch slot asked for more than its first request");
        }
        const size_t at = align256(used_);
        if (at > cap_ || bytes > cap_ - at)
            throw std::invalid_argument("query batch too large for the no-allocation scratch (" +
                                        std::to_string(cap_) + " bytes)");
        ptr_[slot] = base_ + at;
        size_[slot] = bytes;
        used_ = at + bytes;
        return ptr_[slot];
    }

private:
    unsigned char* base_;
    size_t cap_;
    int32_t* status_;
    size_t used_ = 0;
    void* ptr_[nsp::Workspace::kNumSlots] = {};
    size_t size_[nsp::Workspace::kNumSlots] = {};
};

}  // namespace

namespace nsp {
void set_last_error(const char* msg);  // capi.cpp
}

extern "C" nsp_status_t nsp_index_search_device_noalloc(
    nsp_index_t* index, int32_t n, const int32_t* d_indptr, const uint16_t* d_indices,
    const float* d_values, int32_t nnz, int32_t max_row_nnz, int k, float* d_distances,
    int32_t* d_labels, const nsp_search_params_t* params, void* cuda_stream, int32_t* d_status) {
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
        nsp::SeismicSearchArgs a;
        a.k = k;
        a.cut = ssp->cut;
        a.heap_factor = ssp->heap_factor;
        if (sp != nullptr) {
            a.variant = sp->engine.variant;
            a.warps_per_block = sp->engine.warps_per_block;
            a.stage_bytes = sp->engine.stage_bytes;
            a.batch_docs = sp->engine.batch_docs;
            a.cluster = sp->engine.ctas_per_query;
        }
        if (auto* si = dynamic_cast<SeismicIndex*>(base)) {
            st = si->state();
        } else if (auto* qi = dynamic_cast<SeismicScalarQuantizedIndex*>(base)) {
            st = qi->state();
            const ScalarQuantizer& isq = qi->get_scalar_quantizer();
            const auto* sqp = dynamic_cast<const SeismicSQSearchParameters*>(sp);
            const ScalarQuantizer qsq =
                sqp == nullptr ? isq : ScalarQuantizer(isq.get_quantizer_type(), sqp->vmin, sqp->vmax);
            a.qbits = isq.bits();
            a.q_vmin = qsq.get_min();
            a.q_scale = qsq.encode_scale();
            a.decode_scale = isq.decode_scale(qsq);
        } else {
            throw std::invalid_argument("the no-allocation search supports seismic indexes");
        }
        // Uploading the index allocates; it must already be resident (any
        // earlier search or build leaves it so).
        if (st->vectors.dirty || st->vectors.dev.empty() || !st->dev_valid)
            throw std::invalid_argument(
                "index is not resident on the GPU: run one ordinary search first");
        detail::apply_tuned(*st, a, n);
        // every row must end within the nnz entries the caller declared
        a.nnz_cap = nnz;

        auto* scratch = static_cast<unsigned char*>(scratch_on_current_device());
        size_t head = 0;
        const void* vals = d_values;
        auto* stream = static_cast<cudaStream_t>(cuda_stream);
        // the encoded query codes of a quantized index come first
        const size_t codes_bytes =
            a.qbits == 0 ? 0 : align256(static_cast<size_t>(nnz) * 2 + 16);
        if (codes_bytes + 4096 > kNoAllocScratchBytes)
            throw std::invalid_argument("query batch too large for the no-allocation scratch (" +
                                        std::to_string(kNoAllocScratchBytes) + " bytes)");
        head = codes_bytes;
        const size_t avail = kNoAllocScratchBytes - head;
        // The grid: as many CTAs as the engine would launch, capped to what
        // the rest of the array holds (one slack region of 256 bytes per
        // scratch slot for alignment).
        nsp::SeismicScratchNeed need = nsp::seismic_scratch_need(
            st->vectors.dev, st->lists_dev, n, max_row_nnz, a);
        const size_t slack = 8 * 256;
        auto fits = [&](const nsp::SeismicScratchNeed& nd) -> long long {
            if (nd.fixed + slack >= avail || nd.per_cta == 0) return 0;
            return static_cast<long long>((avail - nd.fixed - slack) / nd.per_cta);
        };
        long long room = fits(need);
        if (room < need.cluster && need.cluster > 1 && a.cluster <= 0) {
            // the engine's cluster does not fit: one CTA per query
            a.cluster = 1;
            need = nsp::seismic_scratch_need(st->vectors.dev, st->lists_dev, n, max_row_nnz, a);
            room = fits(need);
        }
        if (room < need.cluster)
            throw std::invalid_argument("posting lists have too many blocks for the no-allocation "
                                        "scratch (" + std::to_string(kNoAllocScratchBytes) +
                                        " bytes)");
        a.max_ctas = static_cast<int>(std::min<long long>(room, need.ctas));

        FixedScratch fixed(scratch + head, avail, d_status);
        if (a.qbits != 0) {
            void* codes = scratch;
            nsp::cuda_check(
                nsp::launch_sq_encode(d_values, codes, nnz, a.qbits, a.q_vmin, a.q_scale, stream),
                "query encode");
            vals = codes;
        }
        nsp::run_seismic(st->vectors.dev, st->lists_dev, n, d_indptr, d_indices, vals,
                         max_row_nnz, a, nullptr, d_distances, d_labels, stream, fixed, nullptr);
        return NSP_OK;
    } catch (const std::invalid_argument& e) {
        nsp::set_last_error(e.what());
        return NSP_ERR_INVALID_ARGUMENT;
    } catch (const std::exception& e) {
        nsp::set_last_error(e.what());
        return NSP_ERR_RUNTIME;
    }
}
