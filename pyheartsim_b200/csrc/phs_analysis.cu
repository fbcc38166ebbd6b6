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
//   phs_interpolate_lat      utility/lat_map.py:29-46 -- electrode LAT spread
//                            over the voxels: linear (barycentric) inside a
//                            Delaunay triangulation of the electrodes, nearest
//                            electrode outside its hull; the point location
//                            follows scipy's LinearNDInterpolator rules (the
//                            bounding-box test and the barycentric inside test
//                            with eps = 100 DBL_EPSILON, degenerate simplices
//                            through their neighbours with sqrt(DBL_EPSILON))
//   phs_activation_times     every upward threshold crossing of Vm per voxel in
//                            a [S][n] history (re-entry analysis: the first
//                            crossing is the activation table the step kernel
//                            records; the later ones are the re-activations)
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
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

// One thread per voxel, walking down the history (one coalesced row per
// sample).  A crossing at sample s: u[s] >= thr and u[s-1] < thr, with the
// state before sample 0 counted as below.  The first max_k crossing samples go
// to times[v * max_k + i]; counts[v] is the number of crossings (it may exceed
// max_k).
template <typename T>
__global__ void activation_kernel(long long S, long long n, const T* __restrict__ hist, long long ld, T thr, int max_k,
                                  int32_t* __restrict__ times, int32_t* __restrict__ counts) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        bool above = false;
        int c = 0;
        for (long long s = 0; s < S; ++s) {
            const bool a = hist[s * ld + v] >= thr;
            if (a && !above) {
                if (c < max_k) times[v * max_k + c] = (int32_t)s;
                ++c;
            }
            above = a;
        }
        counts[v] = c;
    }
}

// ---- interpolate_lat --------------------------------------------------------
constexpr double kInterpEps = 100.0 * 2.220446049250313e-16;   // 100 DBL_EPSILON
constexpr double kInterpEpsBroad = 1.4901161193847656e-08;     // sqrt(DBL_EPSILON)
constexpr int kSimplexChunk = 64;

// Barycentric coordinates of x in a simplex with transform tr (the inverse
// vertex matrix [D][D] row-major, then the last vertex [D]): c[i] =
// sum_j tr[D i + j] (x_j - r_j) for i < D, c[D] = 1 - c[0] - ... - c[D-1], each
// an unfused multiply and add in that order (scipy's _barycentric_inside).
template <int D>
__device__ __forceinline__ void barycentric(const double* tr, const double* x, double* c) {
    c[D] = 1.0;
#pragma unroll
    for (int i = 0; i < D; ++i) {
        double a = 0.0;
#pragma unroll
        for (int j = 0; j < D; ++j) a = __dadd_rn(a, __dmul_rn(tr[D * i + j], __dsub_rn(x[j], tr[D * D + j])));
        c[i] = a;
        c[D] = __dsub_rn(c[D], a);
    }
}

template <int D>
__device__ __forceinline__ bool inside_all(const double* c, double eps) {
    bool in = true;
#pragma unroll
    for (int i = 0; i <= D; ++i) in = in && (-eps <= c[i]) && (c[i] <= 1.0 + eps);
    return in;
}

// One thread per voxel: the first simplex (in index order) whose barycentric
// coordinates all lie in [-eps, 1 + eps]; simplices with a NaN transform
// (degenerate) are replaced by the test of their neighbours, with
// sqrt(DBL_EPSILON) of leeway on the coordinate facing the degenerate one.
// Value: sum_j c_j lat[vertex_j] in vertex order, or NaN outside (nearest
// fallback in interp_nearest_kernel).
template <int D>
__global__ void interp_linear_kernel(long long nv, const double* __restrict__ pts, long long ns,
                                     const int32_t* __restrict__ simplices, const double* __restrict__ transform,
                                     const int32_t* __restrict__ neighbors, const double* __restrict__ lo,
                                     const double* __restrict__ hi, const double* __restrict__ values,
                                     double* __restrict__ out) {
    constexpr int TS = D * (D + 1);
    __shared__ double s_tr[kSimplexChunk * TS];
    const long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const bool live = v < nv;
    double x[D];
    bool outside = !live;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        x[d] = live ? pts[v * D + d] : 0.0;
        if (live && (x[d] < lo[d] - kInterpEps || x[d] > hi[d] + kInterpEps)) outside = true;
    }
    long long found = -1;
    double cf[D + 1];
#pragma unroll
    for (int i = 0; i <= D; ++i) cf[i] = 0.0;
    for (long long s0 = 0; s0 < ns; s0 += kSimplexChunk) {
        const int cnt = (int)((ns - s0 < kSimplexChunk) ? ns - s0 : kSimplexChunk);
        __syncthreads();
        for (int i = threadIdx.x; i < cnt * TS; i += blockDim.x) s_tr[i] = transform[s0 * TS + i];
        __syncthreads();
        if (outside || found >= 0) continue;
        for (int q = 0; q < cnt && found < 0; ++q) {
            const double* tr = s_tr + q * TS;
            double c[D + 1];
            if (tr[0] == tr[0]) {
                barycentric<D>(tr, x, c);
                if (inside_all<D>(c, kInterpEps)) {
                    found = s0 + q;
#pragma unroll
                    for (int i = 0; i <= D; ++i) cf[i] = c[i];
                }
            } else {
                const long long is = s0 + q;
                for (int k = 0; k <= D && found < 0; ++k) {
                    const int nbr = neighbors[is * (D + 1) + k];
                    if (nbr < 0) continue;
                    const double* tn = transform + (long long)nbr * TS;
                    if (!(tn[0] == tn[0])) continue;
                    barycentric<D>(tn, x, c);
                    bool in = true;
                    for (int m = 0; m <= D; ++m) {
                        const double e = (neighbors[(long long)nbr * (D + 1) + m] == (int)is) ? kInterpEpsBroad
                                                                                              : kInterpEps;
                        in = in && (-e <= c[m]) && (c[m] <= 1.0 + kInterpEps);
                    }
                    if (in) {
                        found = nbr;
#pragma unroll
                        for (int i = 0; i <= D; ++i) cf[i] = c[i];
                    }
                }
            }
        }
    }
    if (!live) return;
    if (found < 0) {
        out[v] = __longlong_as_double(0x7ff8000000000000ll);   // NaN: outside the hull
        return;
    }
    double acc = 0.0;
#pragma unroll
    for (int j = 0; j <= D; ++j) acc = __dadd_rn(acc, __dmul_rn(cf[j], values[simplices[found * (D + 1) + j]]));
    out[v] = acc;
}

// Nearest electrode of every voxel whose linear value is NaN: the smallest
// squared distance, summed over the dimensions in order; the lowest index on
// an exact tie.
template <int D>
__global__ void interp_nearest_kernel(long long nv, const double* __restrict__ pts, long long ne,
                                      const double* __restrict__ epts, const double* __restrict__ values,
                                      double* __restrict__ out) {
    __shared__ double s_e[kSimplexChunk * D];
    const long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const bool need = v < nv && isnan(out[v]);
    double x[D];
#pragma unroll
    for (int d = 0; d < D; ++d) x[d] = need ? pts[v * D + d] : 0.0;
    double best = 0.0;
    long long bi = -1;
    for (long long e0 = 0; e0 < ne; e0 += kSimplexChunk) {
        const int cnt = (int)((ne - e0 < kSimplexChunk) ? ne - e0 : kSimplexChunk);
        __syncthreads();
        for (int i = threadIdx.x; i < cnt * D; i += blockDim.x) s_e[i] = epts[e0 * D + i];
        __syncthreads();
        if (!need) continue;
        for (int q = 0; q < cnt; ++q) {
            double d2 = 0.0;
#pragma unroll
            for (int d = 0; d < D; ++d) {
                const double t = __dsub_rn(x[d], s_e[q * D + d]);
                d2 = __dadd_rn(d2, __dmul_rn(t, t));
            }
            if (bi < 0 || d2 < best) { best = d2; bi = e0 + q; }
        }
    }
    if (need && bi >= 0) out[v] = values[bi];
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

int phs_interpolate_lat(int64_t n_v, int ndim, const double* voxel, int64_t n_e, const double* electrode,
                        const double* lat_electrode, int64_t n_simplex, const int32_t* simplices,
                        const double* transform, const int32_t* neighbors, const double* min_bound,
                        const double* max_bound, double* lat_voxel, void* stream) {
    if (n_v <= 0 || n_e <= 0 || n_simplex <= 0 || (ndim != 2 && ndim != 3) || !voxel || !electrode ||
        !lat_electrode || !simplices || !transform || !neighbors || !min_bound || !max_bound || !lat_voxel)
        return PHS_ERR_BAD_ARG;
    if (n_v > 65535LL * 128) return PHS_ERR_BAD_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned int blocks = (unsigned int)((n_v + 127) / 128);
    if (ndim == 2) {
        interp_linear_kernel<2><<<blocks, 128, 0, s>>>(n_v, voxel, n_simplex, simplices, transform, neighbors,
                                                       min_bound, max_bound, lat_electrode, lat_voxel);
        interp_nearest_kernel<2><<<blocks, 128, 0, s>>>(n_v, voxel, n_e, electrode, lat_electrode, lat_voxel);
    } else {
        interp_linear_kernel<3><<<blocks, 128, 0, s>>>(n_v, voxel, n_simplex, simplices, transform, neighbors,
                                                       min_bound, max_bound, lat_electrode, lat_voxel);
        interp_nearest_kernel<3><<<blocks, 128, 0, s>>>(n_v, voxel, n_e, electrode, lat_electrode, lat_voxel);
    }
    PHS_CUDA_TRY(cudaGetLastError());
    return PHS_OK;
}

int phs_activation_times(int64_t S, int64_t n, const void* hist, int64_t ld, int is_f64, double threshold,
                         int32_t max_per_voxel, int32_t* times, int32_t* counts, void* stream) {
    if (S <= 0 || n <= 0 || ld < n || S > INT32_MAX || max_per_voxel < 0 || !hist || !counts ||
        (max_per_voxel > 0 && !times))
        return PHS_ERR_BAD_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned int blocks = (unsigned int)std::min<long long>((n + 255) / 256, 65535);
    if (is_f64)
        activation_kernel<double><<<blocks, 256, 0, s>>>(S, n, (const double*)hist, ld, threshold, max_per_voxel,
                                                         times, counts);
    else
        activation_kernel<float><<<blocks, 256, 0, s>>>(S, n, (const float*)hist, ld, (float)threshold,
                                                        max_per_voxel, times, counts);
    PHS_CUDA_TRY(cudaGetLastError());
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
