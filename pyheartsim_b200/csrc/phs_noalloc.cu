// Allocation-free variant of the FP64 electrogram contraction.
//
// phs_egm_contract_f64 allocates its split-K partial sums on every call.  Some
// callers cannot allocate device memory at the moment they contract: code that
// runs while a stream is being captured in global mode (allocation calls are
// illegal there), hosts whose device memory is entirely owned by another
// allocator (a framework's caching pool that has reserved the free memory), and
// latency-critical loops that cannot afford cudaFree's implicit device-wide
// synchronisation.  phs_egm_contract_f64_noalloc gives them the same result
// with the partial sums in a fixed array that lives in this file for the life
// of the process.
//
// Limits and sharing:
//   * the array holds kNoAllocPartials doubles (16 MiB), so T * n_e must not
//     exceed 2,097,152; larger calls are rejected with PHS_ERR_BAD_ARG;
//   * every GPU that loads the library holds its own copy of the array until the
//     process exits;
//   * all calls share the array: calls that overlap on the GPU (different
//     streams, or host threads racing on one device) corrupt each other's
//     partials; serialise them on one stream;
//   * the array keeps the previous call's contents; nothing in it needs to
//     start at zero, because every partial a call reads is first written by the
//     same call.
// The array's device address is looked up (cudaGetSymbolAddress) with the
// calling device current.  Outside a stream capture the lookup is repeated on
// every call, so the address stays right after a device reset reloads the
// module; during a capture the address cached by the last call made outside a
// capture is used.  Make the first call on each device before any stream
// capture.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <mutex>

#include "../../include/phs.h"
#include "phs_common.cuh"

namespace phs {

int contract_f64_into(int64_t T, int64_t n_v, int64_t n_e, const double* V, int64_t ldv, const double* Mt,
                      double* egm, double* P, int64_t max_partials, cudaStream_t stream);

constexpr int64_t kNoAllocPartials = int64_t(1) << 21;   // 16 MiB of FP64 partial sums

static __device__ __align__(256) double g_noalloc_partials[kNoAllocPartials];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_addr[kMaxDevices] = {};

// Device address of g_noalloc_partials on the current device: looked up again
// when `stream` is not capturing, the cached address while it is.
int noalloc_partials(cudaStream_t stream, double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) { set_last_error("phs_egm_contract_f64_noalloc: cudaGetDevice", e); return PHS_ERR_CUDA; }
    if (dev < 0 || dev >= kMaxDevices) {
        char msg[128];
        snprintf(msg, sizeof(msg), "phs_egm_contract_f64_noalloc: device %d is beyond the %d devices it serves", dev,
                 kMaxDevices);
        set_last_message(msg);
        return PHS_ERR_UNSUPPORTED;
    }
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(stream, &cap);
    if (e != cudaSuccess) { set_last_error("phs_egm_contract_f64_noalloc: cudaStreamIsCapturing", e); return PHS_ERR_CUDA; }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (cap == cudaStreamCaptureStatusNone || !g_noalloc_addr[dev]) {
        if (cap != cudaStreamCaptureStatusNone) {
            set_last_message("phs_egm_contract_f64_noalloc: first call on this device made during a stream capture");
            return PHS_ERR_STATE;
        }
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess) {
            set_last_error("phs_egm_contract_f64_noalloc: cudaGetSymbolAddress", e);
            return PHS_ERR_CUDA;
        }
        g_noalloc_addr[dev] = (double*)p;
    }
    *out = g_noalloc_addr[dev];
    return PHS_OK;
}
}  // namespace

}  // namespace phs

extern "C" {

int64_t phs_egm_noalloc_capacity(void) { return phs::kNoAllocPartials; }

int phs_egm_contract_f64_noalloc(int64_t T, int64_t n_v, int64_t n_e, const double* V, int64_t ldv,
                                 const double* Mt, double* egm, void* stream) {
    if (!V || !Mt || !egm || T <= 0 || n_v <= 0 || n_e <= 0 || ldv < n_v) return PHS_ERR_BAD_ARG;
    if (T > phs::kNoAllocPartials / n_e) {
        char msg[160];
        snprintf(msg, sizeof(msg),
                 "phs_egm_contract_f64_noalloc: T*n_e = %lld exceeds the fixed scratch of %lld doubles",
                 (long long)T * (long long)n_e, (long long)phs::kNoAllocPartials);
        phs::set_last_message(msg);
        return PHS_ERR_BAD_ARG;
    }
    double* partials = nullptr;
    int rc = phs::noalloc_partials((cudaStream_t)stream, &partials);
    if (rc != PHS_OK) return rc;
    return phs::contract_f64_into(T, n_v, n_e, V, ldv, Mt, egm, partials, phs::kNoAllocPartials,
                                  (cudaStream_t)stream);
}

}  // extern "C"
