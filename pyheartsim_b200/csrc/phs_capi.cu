// Status strings, version and error bookkeeping of the C ABI.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>
#include <mutex>

#include "../../include/phs.h"
#include "phs_common.cuh"

namespace phs {
namespace {
std::mutex g_err_mu;
char g_err[512] = "";
}  // namespace

void set_last_error(const char* where, cudaError_t e) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    snprintf(g_err, sizeof(g_err), "%s: %s (%s)", where, cudaGetErrorName(e), cudaGetErrorString(e));
}

void set_last_message(const char* msg) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    snprintf(g_err, sizeof(g_err), "%s", msg);
}
}  // namespace phs

extern "C" {

const char* phs_status_string(int s) {
    switch (s) {
        case PHS_OK: return "ok";
        case PHS_ERR_BAD_ARG: return "invalid argument";
        case PHS_ERR_BAD_TABLE: return "neighbour table or coefficient out of range";
        case PHS_WARN_NO_CONVERGE: return "GMRES did not converge within maxiter";
        case PHS_ERR_NONFINITE: return "non-finite value in a solver norm";
        case PHS_ERR_OOM: return "device allocation failed";
        case PHS_ERR_TIMEOUT: return "bounded device-side wait gave up";
        case PHS_ERR_CUDA: return "CUDA runtime error";
        case PHS_ERR_UNSUPPORTED: return "unsupported input";
        case PHS_ERR_STATE: return "call not valid in the current state";
        default: return "unknown status";
    }
}

int phs_version(void) { return 100; }

const char* phs_last_error(void) { return phs::g_err; }

}  // extern "C"
