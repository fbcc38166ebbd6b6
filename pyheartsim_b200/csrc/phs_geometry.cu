// Geometry and operator tables built on the device.
//
// The reference prepares the inputs of the time stepper on the host with
// Python loops: one KDTree query per neighbour (utility/voxelization.py:102-152,
// find_neighbor_voxel_ids), a loop over voxels for P_2d
// (simulation/equation_parts.py:36-114) and one for the CSR Laplacian
// (simulation/simulation_gpu.py:138-225).  Here the same tables come from
// three device passes:
//
//   phs_lattice_neighbors  dense occupancy grid over the bounding box of the
//                          integer lattice coordinates: scatter voxel ids,
//                          gather the 18 neighbours; a scan over the grid in
//                          (z, y, x) order gives the row order of the voxels
//   phs_equation_parts     P_2d, FP64, in the reference's operation order
//                          (no contraction), so it is bit-identical
//   phs_operator_tables    the compacted operator of compile_instance in device
//                          row order: face neighbours and coefficients (face
//                          cross terms folded in), the isotropic row form,
//                          edge pairs, flags and per-voxel parameters
//
// Every index a kernel dereferences is either < n by construction or checked.
#include <cuda_runtime.h>
#include <stdint.h>
#include <limits.h>

#include "../../include/phs.h"
#include "phs_common.cuh"

namespace {

constexpr int kGeoThreads = 256;
constexpr long long kMaxGridCells = 1ll << 31;

// neighbour offsets in the reference's column order (utility/voxelization.py:107-132)
__constant__ int8_t c_off[18][3] = {
    {1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1},
    {1, 1, 0}, {-1, 1, 0}, {1, -1, 0}, {-1, -1, 0},
    {0, 1, 1}, {0, -1, 1}, {0, 1, -1}, {0, -1, -1},
    {1, 0, 1}, {-1, 0, 1}, {1, 0, -1}, {-1, 0, -1}};

// edge cross-term pairs (+ column, - column, P_2d column), simulation_gpu.py:199-206
__constant__ int8_t c_edge[6][3] = {{6, 8, 9}, {9, 7, 10}, {14, 16, 11}, {17, 15, 12}, {10, 12, 13}, {13, 11, 14}};

unsigned int grid_for(long long n) {
    long long b = (n + kGeoThreads - 1) / kGeoThreads;
    if (b < 1) b = 1;
    if (b > 148 * 64) b = 148 * 64;
    return (unsigned int)b;
}

__global__ void bbox_kernel(const int32_t* __restrict__ ijk, long long n, int* mm) {
    int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const int c = ijk[3 * v + d];
            lo[d] = min(lo[d], c);
            hi[d] = max(hi[d], c);
        }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[d] = min(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
            hi[d] = max(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
        }
    }
    if ((threadIdx.x & 31) == 0) {
        for (int d = 0; d < 3; ++d) {
            atomicMin(mm + d, lo[d]);
            atomicMax(mm + 3 + d, hi[d]);
        }
    }
}

struct Box {
    int lo[3];      // minimum coordinate minus one (one empty cell of padding)
    long long sx, sy, sz;
};

__device__ __forceinline__ long long cell_of(const Box& b, int x, int y, int z) {
    return (((long long)z - b.lo[2]) * b.sy + ((long long)y - b.lo[1])) * b.sx + ((long long)x - b.lo[0]);
}

__global__ void fill_i32(int32_t* p, long long n, int32_t v) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        p[i] = v;
}

__global__ void scatter_kernel(const int32_t* __restrict__ ijk, long long n, Box b, int32_t* grid, unsigned int* err) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        const long long c = cell_of(b, ijk[3 * v], ijk[3 * v + 1], ijk[3 * v + 2]);
        if (atomicCAS(grid + c, -1, (int32_t)v) != -1) atomicOr(err, 1u);   // two voxels in one cell
    }
}

__global__ void gather_kernel(const int32_t* __restrict__ ijk, long long n, Box b, const int32_t* __restrict__ grid,
                              int32_t* __restrict__ nb18) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        const int x = ijk[3 * v], y = ijk[3 * v + 1], z = ijk[3 * v + 2];
#pragma unroll
        for (int k = 0; k < 18; ++k)   // the padding keeps every neighbour cell inside the grid
            nb18[18 * v + k] = grid[cell_of(b, x + c_off[k][0], y + c_off[k][1], z + c_off[k][2])];
    }
}

// Row order: rank of a voxel = occupied cells before its cell in (z, y, x)
// order.  Three passes over the grid in chunks of kChunkCells.
constexpr int kChunkCells = kGeoThreads * 4;

__global__ void chunk_count(const int32_t* __restrict__ grid, long long cells, int32_t* counts) {
    __shared__ int s[kGeoThreads / 32];
    const long long base = (long long)blockIdx.x * kChunkCells;
    int c = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const long long q = base + i * kGeoThreads + threadIdx.x;
        if (q < cells && grid[q] >= 0) ++c;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < kGeoThreads / 32; ++w) t += s[w];
        counts[blockIdx.x] = t;
    }
}

// exclusive scan of `m` chunk counts, one CTA (sequential over its threads' slices)
__global__ void scan_counts(int32_t* counts, long long m) {
    __shared__ long long part[kGeoThreads];
    const long long per = (m + kGeoThreads - 1) / kGeoThreads;
    const long long a = threadIdx.x * per, e = min(a + per, m);
    long long s = 0;
    for (long long i = a; i < e; ++i) s += counts[i];
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long run = 0;
        for (int t = 0; t < kGeoThreads; ++t) {
            const long long x = part[t];
            part[t] = run;
            run += x;
        }
    }
    __syncthreads();
    long long run = part[threadIdx.x];
    for (long long i = a; i < e; ++i) {
        const long long x = counts[i];
        counts[i] = (int32_t)run;
        run += x;
    }
}

__global__ void chunk_order(const int32_t* __restrict__ grid, long long cells, const int32_t* __restrict__ offsets,
                            int32_t* __restrict__ order) {
    // cells of the chunk in order: thread t owns cells 4t .. 4t+3
    __shared__ int s[kGeoThreads];
    const long long base = (long long)blockIdx.x * kChunkCells + 4ll * threadIdx.x;
    int32_t g[4];
    int c = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        g[i] = (base + i < cells) ? grid[base + i] : -1;
        c += (g[i] >= 0);
    }
    s[threadIdx.x] = c;
    __syncthreads();
    // exclusive scan over the CTA's threads (Hillis-Steele on shared memory)
    for (int o = 1; o < kGeoThreads; o <<= 1) {
        const int x = (threadIdx.x >= o) ? s[threadIdx.x - o] : 0;
        __syncthreads();
        s[threadIdx.x] += x;
        __syncthreads();
    }
    int r = offsets[blockIdx.x] + s[threadIdx.x] - c;
#pragma unroll
    for (int i = 0; i < 4; ++i)
        if (g[i] >= 0) order[r++] = g[i];
}

// ---- P_2d, simulation/equation_parts.py:36-114 ---------------------------------
__device__ __forceinline__ double dget(const double* D0, long long v, int r, int c) {
    return D0 ? D0[9 * v + 3 * r + c] : (r == c ? 1.0 : 0.0);
}

__global__ void parts_kernel(long long n, const int32_t* __restrict__ nb18, const double* __restrict__ D0,
                             const double* __restrict__ par, double* __restrict__ P) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        double d[18];
        long long q[6];
#pragma unroll
        for (int k = 0; k < 18; ++k) d[k] = (nb18[18 * v + k] >= 0) ? 1.0 : 0.0;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const int32_t t = nb18[18 * v + k];
            q[k] = (t >= 0 && t < n) ? t : 0;          // the reference's -1 -> 0 remap
        }
        double* o = P + 21 * v;
        // columns 0..5: 4 delta_k D_kk (products with the 0/1 deltas are exact)
        o[0] = __dmul_rn(__dmul_rn(4.0, d[0]), dget(D0, v, 0, 0));
        o[1] = __dmul_rn(__dmul_rn(4.0, d[1]), dget(D0, v, 0, 0));
        o[2] = __dmul_rn(__dmul_rn(4.0, d[2]), dget(D0, v, 1, 1));
        o[3] = __dmul_rn(__dmul_rn(4.0, d[3]), dget(D0, v, 1, 1));
        o[4] = __dmul_rn(__dmul_rn(4.0, d[4]), dget(D0, v, 2, 2));
        o[5] = __dmul_rn(__dmul_rn(4.0, d[5]), dget(D0, v, 2, 2));
        // columns 6..8: face cross terms, evaluated left to right as numpy does
#pragma unroll
        for (int col = 0; col < 3; ++col) {
            const double d01 = __dmul_rn(d[0], d[1]), d23 = __dmul_rn(d[2], d[3]), d45 = __dmul_rn(d[4], d[5]);
            const double t0 = __dmul_rn(d01, __dsub_rn(dget(D0, q[0], 0, col), dget(D0, q[1], 0, col)));
            const double t1 = __dmul_rn(d23, __dsub_rn(dget(D0, q[2], 1, col), dget(D0, q[3], 1, col)));
            const double t2 = __dmul_rn(d45, __dsub_rn(dget(D0, q[4], 2, col), dget(D0, q[5], 2, col)));
            const double dd = (col == 0) ? d01 : (col == 1) ? d23 : d45;
            o[6 + col] = __dmul_rn(dd, __dadd_rn(__dadd_rn(t0, t1), t2));
        }
        // columns 9..14: edge cross terms 2 delta_a delta_b D_ij
        o[9] = __dmul_rn(__dmul_rn(__dmul_rn(2.0, d[6]), d[8]), dget(D0, v, 0, 1));
        o[10] = __dmul_rn(__dmul_rn(__dmul_rn(2.0, d[7]), d[9]), dget(D0, v, 0, 1));
        o[11] = __dmul_rn(__dmul_rn(__dmul_rn(2.0, d[14]), d[16]), dget(D0, v, 0, 2));
        o[12] = __dmul_rn(__dmul_rn(__dmul_rn(2.0, d[15]), d[17]), dget(D0, v, 0, 2));
        o[13] = __dmul_rn(__dmul_rn(__dmul_rn(2.0, d[10]), d[12]), dget(D0, v, 1, 2));
        o[14] = __dmul_rn(__dmul_rn(__dmul_rn(2.0, d[11]), d[13]), dget(D0, v, 1, 2));
#pragma unroll
        for (int k = 0; k < 6; ++k) o[15 + k] = par[6 * v + k];
    }
}

// ---- operator tables (compile_instance on the device) --------------------------
__global__ void flags_kernel(long long n, const double* __restrict__ P, unsigned int* fl) {
    unsigned int face = 0, edge = 0, nonuni = 0;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        const double* p = P + 21 * v;
        for (int k = 6; k < 9; ++k) face |= (p[k] != 0.0);
        for (int k = 9; k < 15; ++k) edge |= (p[k] != 0.0);
        for (int k = 15; k < 20; ++k) nonuni |= (p[k] != P[k]);
    }
    if (__any_sync(0xffffffffu, face) && (threadIdx.x & 31) == 0) atomicOr(fl, 1u);
    if (__any_sync(0xffffffffu, edge) && (threadIdx.x & 31) == 0) atomicOr(fl, 2u);
    if (__any_sync(0xffffffffu, nonuni) && (threadIdx.x & 31) == 0) atomicOr(fl, 4u);
}

__global__ void inverse_kernel(long long n, const int32_t* __restrict__ order, int32_t* __restrict__ inv,
                               unsigned int* err) {
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {
        const long long v = order ? order[r] : r;
        if (v < 0 || v >= n) { atomicOr(err, 1u); continue; }
        inv[v] = (int32_t)r;
    }
}

__global__ void tables_kernel(phs_operator_tables_args a, unsigned int face, unsigned int edge, double den,
                              unsigned int* err) {
    const long long n = a.n_voxel;
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {
        const long long v = a.order ? a.order[r] : r;
        if (v < 0 || v >= n) { atomicOr(err, 1u); continue; }
        const double* p = a.P + 21 * v;
        const int32_t nf = a.node_flag ? a.node_flag[v] : 0;
        const double c = (nf == 4) ? 0.0 : p[20];
        const double Dc = __ddiv_rn(c, den);
        double cf[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            cf[k] = __dmul_rn(Dc, p[k]);
            if (face) {
                const double x = __dmul_rn(Dc, p[6 + (k >> 1)]);
                cf[k] = __dadd_rn(cf[k], (k & 1) ? -x : x);
            }
            int32_t t = a.nb18[18 * v + k];
            if (t == -1) t = 0;                      // the reference's -1 -> 0 remap
            if (t < 0 || t >= n) { atomicOr(err, 2u); t = 0; }
            const int32_t rt = a.inv[t];
            if (rt < 0) atomicOr(err, 1u);
            a.nb6[6 * r + k] = rt;
            a.coef6[6 * r + k] = cf[k];
        }
        // isotropic row form: the first non-zero coefficient and a presence mask
        double w = 0.0;
        unsigned int mk = 0;
        for (int k = 5; k >= 0; --k)
            if (cf[k] != 0.0) { w = cf[k]; mk |= 1u << k; }
        bool iso = true;
#pragma unroll
        for (int k = 0; k < 6; ++k) iso = iso && (cf[k] == (((mk >> k) & 1u) ? w : 0.0));
        if (!iso) atomicAnd(a.iso_word, 0u);
        a.cw[r] = w;
        a.mask6[r] = (uint8_t)mk;
        a.vflags[r] = (nf == 3) ? (uint8_t)PHS_VFLAG_TBLOCK : (uint8_t)0;
        if (a.vparams)
            for (int k = 0; k < 5; ++k) a.vparams[5 * r + k] = p[15 + k];
        if (edge) {
            for (int e = 0; e < 6; ++e) {
                for (int s = 0; s < 2; ++s) {
                    int32_t t = a.nb18[18 * v + c_edge[e][s]];
                    if (t == -1) t = 0;
                    if (t < 0 || t >= n) { atomicOr(err, 2u); t = 0; }
                    const int32_t rt = a.inv[t];
                    if (rt < 0) atomicOr(err, 1u);
                    a.nb_edge[12 * r + 2 * e + s] = rt;
                }
                a.coef_edge[6 * r + e] = __dmul_rn(Dc, p[c_edge[e][2]]);
            }
        }
    }
}

// One pacing set per launch: distinct ids touch distinct bytes, and a repeated
// id writes the same value, so the byte update needs no atomic.
__global__ void pacing_bits(const int64_t* __restrict__ ids, long long count, long long n, const int32_t* __restrict__ inv,
                            uint8_t bit, uint8_t* vflags, unsigned int* err) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count; i += (long long)gridDim.x * blockDim.x) {
        const long long v = ids[i];
        if (v < 0 || v >= n) { atomicOr(err, 4u); continue; }
        const int32_t r = inv[v];
        if (r < 0 || r >= n) { atomicOr(err, 1u); continue; }
        vflags[r] = (uint8_t)(vflags[r] | bit);
    }
}

}  // namespace

using phs::set_last_error;
using phs::set_last_message;

extern "C" {

int phs_lattice_neighbors(int64_t n, const int32_t* ijk, int32_t* nb18, int32_t* order, void* stream) {
    if (n <= 0 || n > INT32_MAX || !ijk || !nb18) return PHS_ERR_BAD_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    int h_mm[6] = {INT_MAX, INT_MAX, INT_MAX, INT_MIN, INT_MIN, INT_MIN};
    int* d_mm = nullptr;
    unsigned int* d_err = nullptr;
    int32_t* grid = nullptr;
    int32_t* counts = nullptr;
    int rc = PHS_OK;
    auto cleanup = [&]() {
        if (counts) cudaFreeAsync(counts, s);
        if (grid) cudaFreeAsync(grid, s);
        if (d_err) cudaFreeAsync(d_err, s);
        if (d_mm) cudaFreeAsync(d_mm, s);
        cudaStreamSynchronize(s);
    };
#define GEO_TRY(expr)                                                  \
    do {                                                               \
        cudaError_t _e = (expr);                                       \
        if (_e != cudaSuccess) {                                       \
            set_last_error(#expr, _e);                                 \
            cleanup();                                                 \
            return _e == cudaErrorMemoryAllocation ? PHS_ERR_OOM : PHS_ERR_CUDA; \
        }                                                              \
    } while (0)
    GEO_TRY(cudaMallocAsync((void**)&d_mm, sizeof(h_mm), s));
    GEO_TRY(cudaMallocAsync((void**)&d_err, sizeof(unsigned int), s));
    GEO_TRY(cudaMemcpyAsync(d_mm, h_mm, sizeof(h_mm), cudaMemcpyHostToDevice, s));
    GEO_TRY(cudaMemsetAsync(d_err, 0, sizeof(unsigned int), s));
    bbox_kernel<<<grid_for(n), kGeoThreads, 0, s>>>(ijk, n, d_mm);
    GEO_TRY(cudaGetLastError());
    GEO_TRY(cudaMemcpyAsync(h_mm, d_mm, sizeof(h_mm), cudaMemcpyDeviceToHost, s));
    GEO_TRY(cudaStreamSynchronize(s));
    bool coords_ok = true;   // neighbour coordinates (+-1) and the padding stay inside int
    for (int d = 0; d < 3; ++d) coords_ok = coords_ok && h_mm[d] >= INT_MIN + 2 && h_mm[3 + d] <= INT_MAX - 2;
    Box b;
    long long span[3] = {0, 0, 0};
    for (int d = 0; d < 3 && coords_ok; ++d) {
        b.lo[d] = h_mm[d] - 1;
        span[d] = (long long)h_mm[3 + d] - (long long)h_mm[d] + 3;   // one padding cell on each side
    }
    b.sx = span[0];
    b.sy = span[1];
    b.sz = span[2];
    // cells = sx * sy * sz, checked factor by factor against the bound
    const bool fits = coords_ok && span[0] > 0 && span[1] > 0 && span[2] > 0 && span[0] <= kMaxGridCells &&
                      span[1] <= kMaxGridCells / span[0] && span[2] <= kMaxGridCells / (span[0] * span[1]);
    if (!fits) {
        set_last_message("phs_lattice_neighbors: bounding box of the coordinates exceeds 2^31 cells");
        cleanup();
        return PHS_ERR_UNSUPPORTED;
    }
    const long long cells = span[0] * span[1] * span[2];
    GEO_TRY(cudaMallocAsync((void**)&grid, (size_t)cells * sizeof(int32_t), s));
    fill_i32<<<grid_for(cells), kGeoThreads, 0, s>>>(grid, cells, -1);
    scatter_kernel<<<grid_for(n), kGeoThreads, 0, s>>>(ijk, n, b, grid, d_err);
    gather_kernel<<<grid_for(n), kGeoThreads, 0, s>>>(ijk, n, b, grid, nb18);
    GEO_TRY(cudaGetLastError());
    if (order) {
        const long long chunks = (cells + kChunkCells - 1) / kChunkCells;
        GEO_TRY(cudaMallocAsync((void**)&counts, (size_t)chunks * sizeof(int32_t), s));
        chunk_count<<<(unsigned int)chunks, kGeoThreads, 0, s>>>(grid, cells, counts);
        scan_counts<<<1, kGeoThreads, 0, s>>>(counts, chunks);
        chunk_order<<<(unsigned int)chunks, kGeoThreads, 0, s>>>(grid, cells, counts, order);
        GEO_TRY(cudaGetLastError());
    }
    unsigned int h_err = 0;
    GEO_TRY(cudaMemcpyAsync(&h_err, d_err, sizeof(h_err), cudaMemcpyDeviceToHost, s));
    GEO_TRY(cudaStreamSynchronize(s));
    if (h_err) {
        set_last_message("phs_lattice_neighbors: duplicate voxel coordinates");
        rc = PHS_ERR_BAD_TABLE;
    }
    cleanup();
#undef GEO_TRY
    return rc;
}

int phs_equation_parts(int64_t n, const int32_t* nb18, const double* D0, const double* par, double* P, void* stream) {
    if (n <= 0 || n > INT32_MAX || !nb18 || !par || !P) return PHS_ERR_BAD_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    parts_kernel<<<grid_for(n), kGeoThreads, 0, s>>>(n, nb18, D0, par, P);
    PHS_CUDA_TRY(cudaGetLastError());
    PHS_CUDA_TRY(cudaStreamSynchronize(s));
    return PHS_OK;
}

int phs_operator_flags(int64_t n, const double* P, int32_t* out3, void* stream) {
    if (n <= 0 || !P || !out3) return PHS_ERR_BAD_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    unsigned int* d = nullptr;
    PHS_CUDA_TRY(cudaMallocAsync((void**)&d, sizeof(unsigned int), s));
    unsigned int h = 0;
    cudaError_t e = cudaMemsetAsync(d, 0, sizeof(unsigned int), s);
    if (e == cudaSuccess) {
        flags_kernel<<<grid_for(n), kGeoThreads, 0, s>>>(n, P, d);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(d, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { set_last_error("phs_operator_flags", e); return PHS_ERR_CUDA; }
    out3[0] = (h & 1u) != 0;
    out3[1] = (h & 2u) != 0;
    out3[2] = (h & 4u) == 0;
    return PHS_OK;
}

int phs_operator_tables(phs_operator_tables_args* a) {
    if (!a || a->n_voxel <= 0 || a->n_voxel > INT32_MAX || !a->P || !a->nb18 || !a->inv || !a->nb6 || !a->coef6 ||
        !a->cw || !a->mask6 || !a->vflags || !(a->Delta > 0.0) || !a->iso_word)
        return PHS_ERR_BAD_ARG;
    if (a->edge && (!a->nb_edge || !a->coef_edge)) return PHS_ERR_BAD_ARG;
    cudaStream_t s = (cudaStream_t)a->stream;
    const long long n = a->n_voxel;
    unsigned int* d_err = nullptr;
    PHS_CUDA_TRY(cudaMallocAsync((void**)&d_err, sizeof(unsigned int), s));
    unsigned int h_err = 0, one = 1u;
    cudaError_t e = cudaMemsetAsync(d_err, 0, sizeof(unsigned int), s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(a->iso_word, &one, sizeof(one), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        fill_i32<<<grid_for(n), kGeoThreads, 0, s>>>(a->inv, n, -1);   // entries an order misses stay -1
        inverse_kernel<<<grid_for(n), kGeoThreads, 0, s>>>(n, a->order, a->inv, d_err);
        // 4 Delta^2 as the host computes it: Delta ** 2, then times 4
        const double den = 4.0 * (a->Delta * a->Delta);
        tables_kernel<<<grid_for(n), kGeoThreads, 0, s>>>(*a, a->face_cross ? 1u : 0u, a->edge ? 1u : 0u, den, d_err);
        if (a->s1 && a->n_s1 > 0)
            pacing_bits<<<grid_for(a->n_s1), kGeoThreads, 0, s>>>(a->s1, a->n_s1, n, a->inv, (uint8_t)PHS_VFLAG_S1,
                                                                   a->vflags, d_err);
        if (a->s2 && a->n_s2 > 0)
            pacing_bits<<<grid_for(a->n_s2), kGeoThreads, 0, s>>>(a->s2, a->n_s2, n, a->inv, (uint8_t)PHS_VFLAG_S2,
                                                                   a->vflags, d_err);
        e = cudaGetLastError();
    }
    unsigned int iso = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_err, d_err, sizeof(h_err), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&iso, a->iso_word, sizeof(iso), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(d_err, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { set_last_error("phs_operator_tables", e); return PHS_ERR_CUDA; }
    a->iso = iso != 0;
    if (h_err) {
        set_last_message("phs_operator_tables: an order entry, neighbour or pacing voxel id is outside [0, n)");
        return PHS_ERR_BAD_TABLE;
    }
    return PHS_OK;
}

}  // extern "C"
