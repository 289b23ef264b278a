// Device-wide exclusive prefix sum over int64 (in place allowed). Used by the
// forward-index upload and the SEISMIC device build.
#ifndef NSP_SCAN_H
#define NSP_SCAN_H

#include <cuda_runtime.h>

#include <cstdint>

namespace nsp {

// out[i] = sum(in[0..i)); in and out may alias. Synchronous with respect to
// the host only where it allocates its block-sum scratch.
void exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t n, cudaStream_t s);

}  // namespace nsp

#endif  // NSP_SCAN_H
