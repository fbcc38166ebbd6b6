// Unipolar electrogram of the PyHeartSim B200 path: lead-field construction,
// FP64 contraction and normalisation.
//
// The reference (simulation/unipolar_electrogram_gpu.py:21-69) evaluates
//   egm[t,e] = sum_v c_v / l_ve^3 * sum_i (D_v grad V)_i * l_ve,i
// with one atomicAdd per (voxel, electrode, time).  Everything except V is
// independent of time, and the gradient is linear in V
// (simulation/unipolar_electrogram_equation_parts.py:60-103), so the sum is a
// matrix product egm = V M with a lead field M (n_v x n_e).  M is built once in
// FP64 (stored transposed, Mt[e][w], the K-major operand of the contraction)
// and the contraction runs as a GEMM.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <algorithm>
#include <vector>

#include "../../include/phs.h"
#include "phs_common.cuh"

namespace phs {

// Mt[e][w] = sum over incoming gradient terms (v, +-(d+1)) of
//            +-c_v / l^3 * (D_v^T l)_d / (2 Delta),  l = x_v - x_e, |l| clamped to >= 1.
__global__ void leadfield_kernel(int64_t n_v, int64_t n_e, const double* __restrict__ xyz,
                                 const double* __restrict__ exyz, const double* __restrict__ c,
                                 const double* __restrict__ D0, const int32_t* __restrict__ in_ptr,
                                 const int32_t* __restrict__ in_src, const int8_t* __restrict__ in_dir,
                                 double inv2d, double* __restrict__ Mt) {
    const int64_t e = blockIdx.y;
    const double ex = exyz[3 * e], ey = exyz[3 * e + 1], ez = exyz[3 * e + 2];
    for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < n_v;
         w += (int64_t)gridDim.x * blockDim.x) {
        double acc = 0.0;
        const int32_t b0 = in_ptr[w], b1 = in_ptr[w + 1];
        for (int32_t q = b0; q < b1; ++q) {
            const int32_t v = in_src[q];
            const int dd = in_dir[q];
            const int d = (dd > 0 ? dd : -dd) - 1;
            const double lx = xyz[3 * v] - ex, ly = xyz[3 * v + 1] - ey, lz = xyz[3 * v + 2] - ez;
            double l = sqrt(lx * lx + ly * ly + lz * lz);
            if (l < 1.0) l = 1.0;
            double proj;
            if (D0) {
                const double* Dv = D0 + 9 * (int64_t)v;
                proj = Dv[0 + d] * lx + Dv[3 + d] * ly + Dv[6 + d] * lz;
            } else {
                proj = (d == 0) ? lx : (d == 1 ? ly : lz);
            }
            const double g = c[v] / (l * l * l) * proj * inv2d;
            acc += (dd > 0) ? g : -g;
        }
        Mt[e * n_v + w] = acc;
    }
}

// FP64 C[t][e] = sum_k A[t][k] * B[e][k] over one K-split; tile 64x64, K-step 16,
// 256 threads with a 4x4 micro-tile each.  Partials go to P[split][t][e].
constexpr int DG_BM = 64, DG_BN = 64, DG_BK = 16;
__global__ void __launch_bounds__(256)
dgemm_tn_kernel(int64_t M, int64_t N, int64_t K, const double* __restrict__ A, int64_t lda,
                const double* __restrict__ B, int64_t ldb, double* __restrict__ P, int64_t kchunk) {
    __shared__ double As[DG_BK][DG_BM + 1];
    __shared__ double Bs[DG_BK][DG_BN + 1];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int64_t m0 = (int64_t)blockIdx.x * DG_BM, n0 = (int64_t)blockIdx.y * DG_BN;
    const int64_t k_beg = (int64_t)blockIdx.z * kchunk;
    const int64_t k_end = std::min<int64_t>(K, k_beg + kchunk);
    double acc[4][4] = {};
    for (int64_t k0 = k_beg; k0 < k_end; k0 += DG_BK) {
        // 64x16 tiles: 1024 values each, 4 per thread
        for (int i = threadIdx.x; i < DG_BM * DG_BK; i += 256) {
            const int r = i / DG_BK, kk = i % DG_BK;
            const int64_t gm = m0 + r, gk = k0 + kk;
            As[kk][r] = (gm < M && gk < k_end) ? A[gm * lda + gk] : 0.0;
            const int64_t gn = n0 + r;
            Bs[kk][r] = (gn < N && gk < k_end) ? B[gn * ldb + gk] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < DG_BK; ++kk) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
    double* Pz = P + (int64_t)blockIdx.z * M * N;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int64_t gm = m0 + ty + 16 * i;
        if (gm >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int64_t gn = n0 + tx + 16 * j;
            if (gn < N) Pz[gm * N + gn] = acc[i][j];
        }
    }
}

// Sum split-K partials in split order (deterministic).
template <typename TO>
__global__ void splitk_reduce_kernel(int64_t MN, int splits, const double* __restrict__ P, TO* __restrict__ C) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < MN; i += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int z = 0; z < splits; ++z) s += P[(int64_t)z * MN + i];
        C[i] = (TO)s;
    }
}

// ptp[e] = max_t egm[t][e] - min_t egm[t][e]
template <typename T>
__global__ void ptp_kernel(int64_t Tn, int64_t n_e, const T* __restrict__ egm, double* __restrict__ ptp) {
    const int64_t e = blockIdx.x;
    double mx = -INFINITY, mn = INFINITY;
    for (int64_t t = threadIdx.x; t < Tn; t += blockDim.x) {
        double v = (double)egm[t * n_e + e];
        mx = fmax(mx, v);
        mn = fmin(mn, v);
    }
    __shared__ double smx[256], smn[256];
    smx[threadIdx.x] = mx;
    smn[threadIdx.x] = mn;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            smx[threadIdx.x] = fmax(smx[threadIdx.x], smx[threadIdx.x + s]);
            smn[threadIdx.x] = fmin(smn[threadIdx.x], smn[threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) ptp[e] = smx[0] - smn[0];
}

// egm *= 1 / mean_e(ptp); every block recomputes the mean in the same order.
template <typename T>
__global__ void scale_kernel(int64_t total, int64_t n_e, const double* __restrict__ ptp, T* __restrict__ egm) {
    __shared__ double s_scale;
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int64_t e = 0; e < n_e; ++e) s += ptp[e];
        s_scale = 1.0 / (s / (double)n_e);
    }
    __syncthreads();
    const double sc = s_scale;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
        egm[i] = (T)((double)egm[i] * sc);
}

int contract_f64(int64_t T, int64_t n_v, int64_t n_e, const double* V, int64_t ldv, const double* Mt,
                 double* egm, cudaStream_t stream) {
    if (T <= 0 || n_v <= 0 || n_e <= 0 || ldv < n_v) return PHS_ERR_BAD_ARG;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t tm = (T + DG_BM - 1) / DG_BM, tn = (n_e + DG_BN - 1) / DG_BN;
    const int64_t target = 2LL * sms;
    int64_t splits = std::max<int64_t>(1, std::min<int64_t>((target + tm * tn - 1) / (tm * tn), (n_v + 255) / 256));
    int64_t kchunk = (n_v + splits - 1) / splits;
    kchunk = ((kchunk + DG_BK - 1) / DG_BK) * DG_BK;
    splits = (n_v + kchunk - 1) / kchunk;
    double* P = nullptr;
    PHS_CUDA_TRY(cudaMallocAsync((void**)&P, (size_t)splits * T * n_e * sizeof(double), stream));
    dim3 grid((unsigned)tm, (unsigned)tn, (unsigned)splits);
    dgemm_tn_kernel<<<grid, 256, 0, stream>>>(T, n_e, n_v, V, ldv, Mt, n_v, P, kchunk);
    const int64_t MN = T * n_e;
    splitk_reduce_kernel<double><<<(unsigned)std::min<int64_t>((MN + 255) / 256, 4096), 256, 0, stream>>>(
        MN, (int)splits, P, egm);
    cudaError_t e = cudaGetLastError();
    cudaFreeAsync(P, stream);
    if (e != cudaSuccess) { set_last_error("contract_f64", e); return PHS_ERR_CUDA; }
    return PHS_OK;
}

// Launch the split-K FP64 contraction into caller-provided partials
// P[splits][T][n_e] and reduce them into egm (used by the allocation-free entry
// point in phs_noalloc.cu).  `max_partials` bounds splits * T * n_e.
int contract_f64_into(int64_t T, int64_t n_v, int64_t n_e, const double* V, int64_t ldv, const double* Mt,
                      double* egm, double* P, int64_t max_partials, cudaStream_t stream) {
    if (T <= 0 || n_v <= 0 || n_e <= 0 || ldv < n_v || T * n_e > max_partials) return PHS_ERR_BAD_ARG;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t tm = (T + DG_BM - 1) / DG_BM, tn = (n_e + DG_BN - 1) / DG_BN;
    const int64_t target = 2LL * sms;
    int64_t splits = std::max<int64_t>(1, std::min<int64_t>((target + tm * tn - 1) / (tm * tn), (n_v + 255) / 256));
    splits = std::min<int64_t>(splits, max_partials / (T * n_e));
    int64_t kchunk = (n_v + splits - 1) / splits;
    kchunk = ((kchunk + DG_BK - 1) / DG_BK) * DG_BK;
    splits = (n_v + kchunk - 1) / kchunk;
    dim3 grid((unsigned)tm, (unsigned)tn, (unsigned)splits);
    dgemm_tn_kernel<<<grid, 256, 0, stream>>>(T, n_e, n_v, V, ldv, Mt, n_v, P, kchunk);
    const int64_t MN = T * n_e;
    splitk_reduce_kernel<double><<<(unsigned)std::min<int64_t>((MN + 255) / 256, 4096), 256, 0, stream>>>(
        MN, (int)splits, P, egm);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { set_last_error("contract_f64_into", e); return PHS_ERR_CUDA; }
    return PHS_OK;
}

int normalize(int64_t T, int64_t n_e, void* egm, bool is_f64, cudaStream_t stream) {
    double* ptp = nullptr;
    PHS_CUDA_TRY(cudaMallocAsync((void**)&ptp, (size_t)n_e * sizeof(double), stream));
    const int64_t total = T * n_e;
    const unsigned blocks = (unsigned)std::min<int64_t>((total + 255) / 256, 2048);
    if (is_f64) {
        ptp_kernel<double><<<(unsigned)n_e, 256, 0, stream>>>(T, n_e, (const double*)egm, ptp);
        scale_kernel<double><<<blocks, 256, 0, stream>>>(total, n_e, ptp, (double*)egm);
    } else {
        ptp_kernel<float><<<(unsigned)n_e, 256, 0, stream>>>(T, n_e, (const float*)egm, ptp);
        scale_kernel<float><<<blocks, 256, 0, stream>>>(total, n_e, ptp, (float*)egm);
    }
    cudaError_t e = cudaGetLastError();
    cudaFreeAsync(ptp, stream);
    if (e != cudaSuccess) { set_last_error("normalize", e); return PHS_ERR_CUDA; }
    return PHS_OK;
}

// defined in phs_egm_tc.cu
int contract_bf16x3(int64_t T, int64_t n_e, int64_t T_pad, int64_t n_e_pad, int64_t K_pad,
                    const uint16_t* Vhi, const uint16_t* Vlo, const uint16_t* Mhi, const uint16_t* Mlo,
                    float* egm, void* work, cudaStream_t stream, int config);
int bf16x3_config_count();
int64_t bf16x3_workspace(int64_t T_pad, int64_t n_e_pad, int64_t K_pad);
int bf16x3_status(const void* work, cudaStream_t stream);
int split_bf16(int64_t rows, int64_t cols, const void* src, int64_t ld, bool src_f64, uint16_t* hi,
               uint16_t* lo, int64_t rows_out, int64_t ld_out, cudaStream_t stream);

}  // namespace phs

using namespace phs;

extern "C" {

int phs_egm_leadfield_f64(int64_t n_v, int64_t n_e, const double* voxel_xyz, const double* electrode_xyz,
                          const double* c_voxel, const double* D0, const int32_t* in_ptr, const int32_t* in_src,
                          const int8_t* in_dir, double inv_two_delta, double* Mt, void* stream) {
    if (n_v <= 0 || n_e <= 0 || n_e > 65535 || !voxel_xyz || !electrode_xyz || !c_voxel || !in_ptr || !Mt)
        return PHS_ERR_BAD_ARG;
    dim3 grid((unsigned)std::min<int64_t>((n_v + 255) / 256, 1024), (unsigned)n_e);
    leadfield_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(n_v, n_e, voxel_xyz, electrode_xyz, c_voxel, D0,
                                                            in_ptr, in_src, in_dir, inv_two_delta, Mt);
    PHS_CUDA_TRY(cudaGetLastError());
    return PHS_OK;
}

int phs_egm_contract_f64(int64_t T, int64_t n_v, int64_t n_e, const double* V, int64_t ldv, const double* Mt,
                         double* egm, void* stream) {
    if (!V || !Mt || !egm) return PHS_ERR_BAD_ARG;
    return contract_f64(T, n_v, n_e, V, ldv, Mt, egm, (cudaStream_t)stream);
}

int phs_egm_normalize(int64_t T, int64_t n_e, void* egm, int is_f64, void* stream) {
    if (T <= 0 || n_e <= 0 || !egm) return PHS_ERR_BAD_ARG;
    return normalize(T, n_e, egm, is_f64 != 0, (cudaStream_t)stream);
}

int phs_split_bf16(int64_t rows, int64_t cols, const void* src, int64_t ld, int src_is_f64, uint16_t* hi,
                   uint16_t* lo, int64_t rows_out, int64_t ld_out, void* stream) {
    if (rows <= 0 || cols <= 0 || ld < cols || rows_out < rows || ld_out < cols || !src || !hi || !lo)
        return PHS_ERR_BAD_ARG;
    return split_bf16(rows, cols, src, ld, src_is_f64 != 0, hi, lo, rows_out, ld_out, (cudaStream_t)stream);
}

int64_t phs_egm_bf16x3_workspace(int64_t T_pad, int64_t n_e_pad, int64_t K_pad) {
    return bf16x3_workspace(T_pad, n_e_pad, K_pad);
}

int phs_egm_contract_bf16x3(int64_t T, int64_t n_e, int64_t T_pad, int64_t n_e_pad, int64_t K_pad,
                            const uint16_t* Vhi, const uint16_t* Vlo, const uint16_t* Mhi, const uint16_t* Mlo,
                            float* egm, void* work, void* stream) {
    return contract_bf16x3(T, n_e, T_pad, n_e_pad, K_pad, Vhi, Vlo, Mhi, Mlo, egm, work, (cudaStream_t)stream, -1);
}

int phs_egm_contract_bf16x3_cfg(int64_t T, int64_t n_e, int64_t T_pad, int64_t n_e_pad, int64_t K_pad,
                                const uint16_t* Vhi, const uint16_t* Vlo, const uint16_t* Mhi, const uint16_t* Mlo,
                                float* egm, void* work, int config, void* stream) {
    if (config < 0) return PHS_ERR_BAD_ARG;
    return contract_bf16x3(T, n_e, T_pad, n_e_pad, K_pad, Vhi, Vlo, Mhi, Mlo, egm, work, (cudaStream_t)stream,
                           config);
}

int phs_egm_bf16x3_config_count(void) { return bf16x3_config_count(); }

int phs_egm_bf16x3_status(const void* work, void* stream) { return bf16x3_status(work, (cudaStream_t)stream); }

int phs_electrogram(int64_t T, int64_t n_v, int64_t n_e, const double* V, const double* voxel_xyz,
                    const double* electrode_xyz, const double* c_voxel, const double* D0, const int32_t* in_ptr,
                    const int32_t* in_src, const int8_t* in_dir, double delta, int mode, double* egm_out) {
    if (T <= 0 || n_v <= 0 || n_e <= 0 || !V || !voxel_xyz || !electrode_xyz || !c_voxel || !in_ptr ||
        !egm_out || !(delta > 0.0))
        return PHS_ERR_BAD_ARG;
    if (mode != PHS_EGM_F64 && mode != PHS_EGM_BF16X3) return PHS_ERR_BAD_ARG;
    const int32_t nnz = in_ptr[n_v];
    for (int64_t i = 0; i < nnz; ++i)
        if (in_src[i] < 0 || in_src[i] >= n_v || in_dir[i] == 0 || in_dir[i] > 3 || in_dir[i] < -3)
            return PHS_ERR_BAD_TABLE;
    cudaStream_t s = nullptr;
    std::vector<void*> bufs;
    auto alloc = [&](size_t bytes) -> void* {
        void* p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(bytes, 16)) != cudaSuccess) return nullptr;
        bufs.push_back(p);
        return p;
    };
    auto cleanup = [&](int rc) {
        for (void* p : bufs) cudaFree(p);
        return rc;
    };
    double* dV = (double*)alloc((size_t)T * n_v * 8);
    double* dxyz = (double*)alloc((size_t)n_v * 24);
    double* dex = (double*)alloc((size_t)n_e * 24);
    double* dc = (double*)alloc((size_t)n_v * 8);
    double* dD = D0 ? (double*)alloc((size_t)n_v * 72) : nullptr;
    int32_t* dptr = (int32_t*)alloc((size_t)(n_v + 1) * 4);
    int32_t* dsrc = (int32_t*)alloc((size_t)nnz * 4);
    int8_t* ddir = (int8_t*)alloc((size_t)nnz);
    double* dMt = (double*)alloc((size_t)n_e * n_v * 8);
    double* degm = (double*)alloc((size_t)T * n_e * 8);
    if (!dV || !dxyz || !dex || !dc || (D0 && !dD) || !dptr || !dsrc || !ddir || !dMt || !degm)
        return cleanup(PHS_ERR_OOM);
    if (cudaMemcpy(dV, V, (size_t)T * n_v * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dxyz, voxel_xyz, (size_t)n_v * 24, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dex, electrode_xyz, (size_t)n_e * 24, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dc, c_voxel, (size_t)n_v * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
        (D0 && cudaMemcpy(dD, D0, (size_t)n_v * 72, cudaMemcpyHostToDevice) != cudaSuccess) ||
        cudaMemcpy(dptr, in_ptr, (size_t)(n_v + 1) * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        (nnz && cudaMemcpy(dsrc, in_src, (size_t)nnz * 4, cudaMemcpyHostToDevice) != cudaSuccess) ||
        (nnz && cudaMemcpy(ddir, in_dir, (size_t)nnz, cudaMemcpyHostToDevice) != cudaSuccess))
        return cleanup(PHS_ERR_CUDA);
    int rc = phs_egm_leadfield_f64(n_v, n_e, dxyz, dex, dc, dD, dptr, dsrc, ddir, 1.0 / (2.0 * delta), dMt, s);
    if (rc != PHS_OK) return cleanup(rc);
    if (mode == PHS_EGM_F64) {
        rc = contract_f64(T, n_v, n_e, dV, n_v, dMt, degm, s);
        if (rc != PHS_OK) return cleanup(rc);
        rc = normalize(T, n_e, degm, true, s);
    } else {
        const int64_t Tp = (T + 127) / 128 * 128, Ep = (n_e + 255) / 256 * 256, Kp = (n_v + 63) / 64 * 64;
        uint16_t* vh = (uint16_t*)alloc((size_t)Tp * Kp * 2);
        uint16_t* vl = (uint16_t*)alloc((size_t)Tp * Kp * 2);
        uint16_t* mh = (uint16_t*)alloc((size_t)Ep * Kp * 2);
        uint16_t* ml = (uint16_t*)alloc((size_t)Ep * Kp * 2);
        float* e32 = (float*)alloc((size_t)T * n_e * 4);
        void* work = alloc((size_t)std::max<int64_t>(bf16x3_workspace(Tp, Ep, Kp), 16));
        if (!vh || !vl || !mh || !ml || !e32 || !work) return cleanup(PHS_ERR_OOM);
        rc = split_bf16(T, n_v, dV, n_v, true, vh, vl, Tp, Kp, s);
        if (rc == PHS_OK) rc = split_bf16(n_e, n_v, dMt, n_v, true, mh, ml, Ep, Kp, s);
        if (rc == PHS_OK) rc = contract_bf16x3(T, n_e, Tp, Ep, Kp, vh, vl, mh, ml, e32, work, s, -1);
        if (rc == PHS_OK) rc = bf16x3_status(work, s);
        if (rc == PHS_OK) rc = normalize(T, n_e, e32, false, s);
        if (rc == PHS_OK) {
            const int64_t MN = T * n_e;
            // widen to the f64 output buffer
            std::vector<float> h32((size_t)MN);
            if (cudaMemcpy(h32.data(), e32, (size_t)MN * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
                return cleanup(PHS_ERR_CUDA);
            for (int64_t i = 0; i < MN; ++i) egm_out[i] = (double)h32[(size_t)i];
            return cleanup(PHS_OK);
        }
        return cleanup(rc);
    }
    if (rc != PHS_OK) return cleanup(rc);
    cudaError_t ce = cudaMemcpy(egm_out, degm, (size_t)T * n_e * 8, cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) { set_last_error("phs_electrogram", ce); return cleanup(PHS_ERR_CUDA); }
    return cleanup(PHS_OK);
}

}  // extern "C"
