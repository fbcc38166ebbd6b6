// Electrogram analysis on the device: electrode activation times and
// conduction velocity.
//
//   phs_electrode_lat        utility/lat_map.py:20-27 -- per electrode, the
//                            first time index of the largest negative first
//                            difference (numpy argmax semantics, NaN counts as
//                            the largest), shifted so the earliest is 0
//   phs_conduction_velocity  utility/conduction_velocity.py:23-70 -- per
//                            electrode, a least-squares plane lat = a x + b y +
//                            c z + d through the electrodes within the radius
//                            (itself included); the minimum-norm solution, as
//                            numpy.linalg.lstsq gives, from a one-sided Jacobi
//                            SVD of the m x 4 system (one CTA per electrode);
//                            velocity grad/|grad|^2, speed 1/|grad|, NaN with
//                            fewer than 4 points or |grad|^2 <= 1e-8
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <vector>

#include "../../include/phs.h"
#include "phs_common.cuh"

namespace {

constexpr int kAThreads = 128;
constexpr double kEps = 2.220446049250313e-16;   // DBL_EPSILON (numpy's finfo(float64).eps)

unsigned int blocks_for(long long n) {
    long long b = (n + kAThreads - 1) / kAThreads;
    if (b < 1) b = 1;
    if (b > 65535) b = 65535;
    return (unsigned int)b;
}

template <typename T>
__device__ __forceinline__ T neg_diff(T cur, T prev);
template <>
__device__ __forceinline__ float neg_diff<float>(float cur, float prev) { return -__fsub_rn(cur, prev); }
template <>
__device__ __forceinline__ double neg_diff<double>(double cur, double prev) { return -__dsub_rn(cur, prev); }

// One thread per electrode, walking down time (consecutive electrodes are
// adjacent in memory, so each time step is one coalesced row).
template <typename T>
__global__ void lat_kernel(long long nt, long long ne, const T* __restrict__ egm, int32_t* __restrict__ idx) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ne; e += (long long)gridDim.x * blockDim.x) {
        T prev = egm[e];
        T best = T(0);
        int bi = 0;
        bool have = false, best_nan = false;
        for (long long t = 0; t + 1 < nt; ++t) {
            const T cur = egm[(t + 1) * ne + e];
            const T d = neg_diff<T>(cur, prev);
            prev = cur;
            if (best_nan) continue;                     // the first NaN is the argmax
            if (isnan(d)) { best_nan = true; bi = (int)t; have = true; continue; }
            if (!have || d > best) { best = d; bi = (int)t; have = true; }
        }
        idx[e] = bi;
    }
}

__global__ void shift_to_zero(long long ne, int32_t* idx) {
    __shared__ int s[kAThreads];
    int m = INT32_MAX;
    for (long long e = threadIdx.x; e < ne; e += blockDim.x) m = min(m, idx[e]);
    s[threadIdx.x] = m;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] = min(s[threadIdx.x], s[threadIdx.x + o]);
        __syncthreads();
    }
    const int mn = s[0];
    for (long long e = threadIdx.x; e < ne; e += blockDim.x) idx[e] -= mn;
}

// squared distance in the order scipy's cKDTree accumulates it (x, y, z)
__device__ __forceinline__ double dist2(const double* a, const double* b) {
    const double dx = __dsub_rn(a[0], b[0]), dy = __dsub_rn(a[1], b[1]), dz = __dsub_rn(a[2], b[2]);
    return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

__global__ void cv_count(long long ne, const double* __restrict__ xyz, double r2, int32_t* __restrict__ counts) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ne; i += (long long)gridDim.x * blockDim.x) {
        int c = 0;
        for (long long j = 0; j < ne; ++j) c += (dist2(xyz + 3 * i, xyz + 3 * j) <= r2);
        counts[i] = c;
    }
}

// rows of electrode i at [off[i], off[i] + counts[i]) of five planes: x, y, z, 1, lat
__global__ void cv_fill(long long ne, const double* __restrict__ xyz, const double* __restrict__ lat, double r2,
                        const long long* __restrict__ off, const int32_t* __restrict__ counts, long long total,
                        double* __restrict__ ws) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ne; i += (long long)gridDim.x * blockDim.x) {
        long long k = 0;
        const long long o = off[i], cnt = counts[i];
        for (long long j = 0; j < ne && k < cnt; ++j) {
            if (dist2(xyz + 3 * i, xyz + 3 * j) <= r2) {
                const long long r = o + k;
                ws[r] = xyz[3 * j];
                ws[total + r] = xyz[3 * j + 1];
                ws[2 * total + r] = xyz[3 * j + 2];
                ws[3 * total + r] = 1.0;
                ws[4 * total + r] = lat[j];
                ++k;
            }
        }
    }
}

// CTA-wide sum of three values (fixed order: thread slices, then a tree)
__device__ __forceinline__ void block_sum3(double& a, double& b, double& c, double (*s)[kAThreads]) {
    s[0][threadIdx.x] = a;
    s[1][threadIdx.x] = b;
    s[2][threadIdx.x] = c;
    __syncthreads();
    for (int o = kAThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            s[0][threadIdx.x] += s[0][threadIdx.x + o];
            s[1][threadIdx.x] += s[1][threadIdx.x + o];
            s[2][threadIdx.x] += s[2][threadIdx.x + o];
        }
        __syncthreads();
    }
    a = s[0][0];
    b = s[1][0];
    c = s[2][0];
    __syncthreads();
}

__global__ void __launch_bounds__(kAThreads) cv_solve(long long ne, const long long* __restrict__ off,
                                                      const int32_t* __restrict__ counts, long long total,
                                                      double* __restrict__ ws, double* __restrict__ vvec,
                                                      double* __restrict__ vmag) {
    __shared__ double red[3][kAThreads];
    __shared__ double V[4][4];
    __shared__ double rot[2];
    const long long i = blockIdx.x;
    if (i >= ne) return;
    const long long m = counts[i], o = off[i];
    if (m < 4) {
        if (threadIdx.x == 0) {
            vvec[3 * i] = vvec[3 * i + 1] = vvec[3 * i + 2] = nan("");
            vmag[i] = nan("");
        }
        return;
    }
    double* col[4] = {ws + o, ws + total + o, ws + 2 * total + o, ws + 3 * total + o};
    const double* bvec = ws + 4 * total + o;
    if (threadIdx.x < 16) V[threadIdx.x / 4][threadIdx.x % 4] = (threadIdx.x / 4 == threadIdx.x % 4) ? 1.0 : 0.0;
    __syncthreads();
    // one-sided Jacobi: rotate column pairs until they are orthogonal to machine precision
    for (int sweep = 0; sweep < 60; ++sweep) {
        int rotated = 0;
        for (int p = 0; p < 3; ++p) {
            for (int q = p + 1; q < 4; ++q) {
                double al = 0.0, be = 0.0, ga = 0.0;
                for (long long k = threadIdx.x; k < m; k += kAThreads) {
                    const double x = col[p][k], y = col[q][k];
                    al += x * x;
                    be += y * y;
                    ga += x * y;
                }
                block_sum3(al, be, ga, red);
                if (ga == 0.0 || fabs(ga) <= kEps * sqrt(al * be)) continue;
                ++rotated;
                if (threadIdx.x == 0) {
                    const double zeta = (be - al) / (2.0 * ga);
                    const double t = copysign(1.0, zeta) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                    const double c = 1.0 / sqrt(1.0 + t * t);
                    rot[0] = c;
                    rot[1] = c * t;
                }
                __syncthreads();
                const double c = rot[0], s = rot[1];
                for (long long k = threadIdx.x; k < m; k += kAThreads) {
                    const double x = col[p][k], y = col[q][k];
                    col[p][k] = c * x - s * y;
                    col[q][k] = s * x + c * y;
                }
                if (threadIdx.x < 4) {
                    const double x = V[threadIdx.x][p], y = V[threadIdx.x][q];
                    V[threadIdx.x][p] = c * x - s * y;
                    V[threadIdx.x][q] = s * x + c * y;
                }
                __syncthreads();
            }
        }
        if (rotated == 0) break;
    }
    // singular values, projections of b on the rotated columns (u_i sigma_i)
    double sig2[4], ub[4];
    for (int c = 0; c < 4; c += 1) {
        double a2 = 0.0, ab = 0.0, z = 0.0;
        for (long long k = threadIdx.x; k < m; k += kAThreads) {
            const double x = col[c][k];
            a2 += x * x;
            ab += x * bvec[k];
        }
        block_sum3(a2, ab, z, red);
        sig2[c] = a2;
        ub[c] = ab;
    }
    if (threadIdx.x == 0) {
        double smax = 0.0;
        for (int c = 0; c < 4; ++c) smax = fmax(smax, sqrt(sig2[c]));
        const double tol = kEps * (double)(m > 4 ? m : 4) * smax;   // numpy lstsq rcond=None
        double coef[4] = {0.0, 0.0, 0.0, 0.0};
        for (int c = 0; c < 4; ++c) {
            if (!(sqrt(sig2[c]) > tol)) continue;
            const double w = ub[c] / sig2[c];
            for (int r = 0; r < 4; ++r) coef[r] += V[r][c] * w;
        }
        const double g2 = coef[0] * coef[0] + coef[1] * coef[1] + coef[2] * coef[2];
        if (g2 > 1e-8) {
            vvec[3 * i] = coef[0] / g2;
            vvec[3 * i + 1] = coef[1] / g2;
            vvec[3 * i + 2] = coef[2] / g2;
            vmag[i] = 1.0 / sqrt(g2);
        } else {
            vvec[3 * i] = vvec[3 * i + 1] = vvec[3 * i + 2] = nan("");
            vmag[i] = nan("");
        }
    }
}

}  // namespace

using phs::set_last_error;

extern "C" {

int phs_electrode_lat(int64_t nt, int64_t ne, const void* egm, int is_f64, int32_t* lat_out, void* stream) {
    if (nt < 2 || ne <= 0 || nt > INT32_MAX || !egm || !lat_out) return PHS_ERR_BAD_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    if (is_f64)
        lat_kernel<double><<<blocks_for(ne), kAThreads, 0, s>>>(nt, ne, (const double*)egm, lat_out);
    else
        lat_kernel<float><<<blocks_for(ne), kAThreads, 0, s>>>(nt, ne, (const float*)egm, lat_out);
    shift_to_zero<<<1, kAThreads, 0, s>>>(ne, lat_out);
    PHS_CUDA_TRY(cudaGetLastError());
    PHS_CUDA_TRY(cudaStreamSynchronize(s));
    return PHS_OK;
}

int phs_conduction_velocity(int64_t ne, const double* xyz, const double* lat, double radius, double* v_vec,
                            double* v_mag, void* stream) {
    if (ne <= 0 || ne > (1 << 20) || !xyz || !lat || !v_vec || !v_mag || !(radius >= 0.0)) return PHS_ERR_BAD_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const double r2 = radius * radius;
    int32_t* counts = nullptr;
    long long* off = nullptr;
    double* ws = nullptr;
    auto done = [&](int rc) {
        if (ws) cudaFreeAsync(ws, s);
        if (off) cudaFreeAsync(off, s);
        if (counts) cudaFreeAsync(counts, s);
        cudaStreamSynchronize(s);
        return rc;
    };
    cudaError_t e = cudaMallocAsync((void**)&counts, (size_t)ne * sizeof(int32_t), s);
    if (e == cudaSuccess) {
        cv_count<<<blocks_for(ne), kAThreads, 0, s>>>(ne, xyz, r2, counts);
        e = cudaGetLastError();
    }
    std::vector<int32_t> h_counts((size_t)ne);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_counts.data(), counts, (size_t)ne * sizeof(int32_t),
                                              cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { set_last_error("phs_conduction_velocity", e); return done(PHS_ERR_CUDA); }
    std::vector<long long> h_off((size_t)ne);
    long long total = 0;
    for (long long i = 0; i < ne; ++i) {
        h_off[(size_t)i] = total;
        total += h_counts[(size_t)i];
    }
    e = cudaMallocAsync((void**)&off, (size_t)ne * sizeof(long long), s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(off, h_off.data(), (size_t)ne * sizeof(long long),
                                              cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&ws, (size_t)(5 * (total > 0 ? total : 1)) * sizeof(double), s);
    if (e == cudaSuccess) {
        cv_fill<<<blocks_for(ne), kAThreads, 0, s>>>(ne, xyz, lat, r2, off, counts, total, ws);
        cv_solve<<<(unsigned int)ne, kAThreads, 0, s>>>(ne, off, counts, total, ws, v_vec, v_mag);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_last_error("phs_conduction_velocity", e);
        return done(e == cudaErrorMemoryAllocation ? PHS_ERR_OOM : PHS_ERR_CUDA);
    }
    return done(PHS_OK);
}

}  // extern "C"
