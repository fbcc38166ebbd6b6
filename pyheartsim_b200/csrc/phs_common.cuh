// Shared definitions of the PyHeartSim B200 kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace phs {

constexpr int kThreads = 256;              // threads per CTA of the step kernel
constexpr int kWarps = kThreads / 32;
constexpr int kMaxRestart = 50;            // GMRES(m) restart bound (reference uses m = 50)
constexpr int kSlots = kMaxRestart + 2;    // FP64 partial sums per tile
constexpr int kPhaseScalars = 4;
constexpr int kPadVoxels = 1024;           // per-voxel engine arrays are padded to a multiple of this

// Record a CUDA error message (host side); defined in phs_capi.cu.
void set_last_error(const char* where, cudaError_t e);
// Record a plain error message for phs_last_error().
void set_last_message(const char* msg);

}  // namespace phs

#define PHS_CUDA_TRY(expr)                                   \
    do {                                                     \
        cudaError_t _e = (expr);                             \
        if (_e != cudaSuccess) {                             \
            ::phs::set_last_error(#expr, _e);                \
            return _e == cudaErrorMemoryAllocation ? PHS_ERR_OOM : PHS_ERR_CUDA; \
        }                                                    \
    } while (0)
