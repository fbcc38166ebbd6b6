// Split-BF16 electrogram contraction on the sm_100a tensor cores.
//
//   egm[t][e] = sum_k V[t][k] M[k][e]
//            ~= sum_k (Vhi Mhi + Vhi Mlo + Vlo Mhi)[t][e]      (FP32 accumulation)
//
// with V = Vhi + Vlo and M = Mhi + Mlo split into BF16 pairs.  This replaces the
// per-(voxel, electrode, time) atomicAdd kernel of
// simulation/unipolar_electrogram_gpu.py:21-69 by a dense contraction of the
// lead field (see phs_egm.cu) against the Vm history.
//
// One CTA computes a 128 (t) x BN (e) tile over one K range (split-K):
//   warp 0 lane 0   TMA producer: per stage two 128 x BK BF16 tiles of V (hi,
//                   lo) and two BN x BK tiles of M (hi, lo), 128-byte (BK = 64)
//                   or 64-byte (BK = 32) swizzle, an mbarrier ring of STAGES
//   warp 1 lane 0   MMA issuer: per BK-wide K block, BK/16 K-slices x 3 products
//                   of tcgen05.mma.cta_group::1.kind::f16 (M=128, N=BN, K=16)
//                   into one FP32 accumulator in TMEM (BN columns);
//                   tcgen05.commit frees the stage
//   warps 0..3      epilogue: tcgen05.ld 32x32b.x32 -> FP32 partial tile in HBM
// Tile configurations (kTcConfigs; every one uses 192 KB of shared memory):
// 128 x 128 with 3 stages of BK 64, 128 x 256 with 2 stages of BK 64, 128 x 256
// with 4 stages of BK 32, 128 x 128 with 6 stages of BK 32.  The 256-wide tiles
// read 0.75 of the operand bytes per FLOP of the 128-wide ones (the operands
// stream from L2); the BK-32 rings keep more, smaller stages in flight ahead of
// the MMAs (measured slower: their 64-byte TMA rows move less per request).
// phs_egm_contract_bf16x3 uses kTcDefaultConfig;
// phs_egm_contract_bf16x3_cfg takes a configuration (the autotuner's choice).
// Split-K partials are summed in split order by a second kernel.
//
// Every wait is bounded (kTcWaitNs); on timeout the CTA records an error word,
// drains its own copies and MMAs (bounded), frees TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <algorithm>
#include <mutex>

#include "../../include/phs.h"
#include "phs_common.cuh"

namespace phs {

constexpr int TC_BM = 128;
constexpr int TC_BN_MAX = 256;
constexpr int TC_THREADS = 128;

// Compile-time shape of one tile configuration.
template <int BN, int BK, int STAGES>
struct TcShape {
    static constexpr int A_BYTES = TC_BM * BK * 2;
    static constexpr int B_BYTES = BN * BK * 2;
    static constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
    static constexpr size_t SMEM = (size_t)STAGES * STAGE_BYTES + 1024 /*align*/ + 256 /*barriers*/;
    static constexpr uint32_t SBO = 8u * BK * 2u;            // bytes between 8-row core-matrix groups
    static constexpr uint64_t LAYOUT = BK == 64 ? 2u : 4u;   // SWIZZLE_128B / SWIZZLE_64B
};
constexpr unsigned long long kTcWaitNs = 2000000000ull;  // 2 s
constexpr int64_t kTcHeader = 256;                        // error word at the workspace head

__device__ __forceinline__ unsigned long long tc_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase with the given parity to complete.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    const unsigned long long t0 = tc_ns();
    while (!mbar_try(bar, parity)) {
        if (tc_ns() - t0 > kTcWaitNs) return false;
    }
    return true;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int c0, int c1) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(dst), "l"((uint64_t)map), "r"(bar), "r"(c0), "r"(c1)
        : "memory");
}

// UMMA shared-memory descriptor: K-major, swizzled rows (128 or 64 bytes), 8-row
// groups `sbo` bytes apart.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t sbo, uint64_t layout) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);        // start address
    d |= (uint64_t)1u << 16;                          // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;     // stride byte offset
    d |= (uint64_t)1u << 46;                          // descriptor version (sm_100)
    d |= layout << 61;                                // swizzle mode
    return d;
}

// Instruction descriptor of kind::f16: BF16 x BF16 -> F32, both K-major.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
    return (1u << 4)                    // D format F32
         | (1u << 7)                    // A format BF16
         | (1u << 10)                   // B format BF16
         | ((uint32_t)(N >> 3) << 17)   // N >> 3
         | ((uint32_t)(M >> 4) << 24);  // M >> 4
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld_32x32b_x32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

template <int BN, int BK, int STAGES>
__global__ void __launch_bounds__(TC_THREADS, 1)
egm_bf16x3_kernel(const __grid_constant__ CUtensorMap map_vhi, const __grid_constant__ CUtensorMap map_vlo,
                  const __grid_constant__ CUtensorMap map_mhi, const __grid_constant__ CUtensorMap map_mlo,
                  int nkb_total, int kb_per_split, int T_pad, int part_cols, float* __restrict__ part,
                  int* __restrict__ err) {
    using Sh = TcShape<BN, BK, STAGES>;
    constexpr int TC_BN = BN;
    constexpr int TC_BK = BK;
    constexpr int TC_STAGES = STAGES;
    constexpr int TC_A_BYTES = Sh::A_BYTES;
    constexpr int TC_B_BYTES = Sh::B_BYTES;
    constexpr int TC_STAGE_BYTES = Sh::STAGE_BYTES;
    constexpr int TC_TMEM_COLS = BN;
    extern __shared__ __align__(1024) uint8_t tc_smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)tc_smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* bars = (uint64_t*)(smem + (size_t)TC_STAGES * TC_STAGE_BYTES);
    // bars[0..S) full, bars[S..2S) empty, bars[2S] done;  tmem base after them
    uint32_t* tmem_slot = (uint32_t*)(bars + 2 * TC_STAGES + 1);
    __shared__ int s_fail;

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int t0 = blockIdx.x * TC_BM;
    const int e0 = blockIdx.y * TC_BN;
    const int kb0 = blockIdx.z * kb_per_split;
    const int kb1 = min(nkb_total, kb0 + kb_per_split);
    const int nkb = max(0, kb1 - kb0);

    if (threadIdx.x == 0) {
        s_fail = 0;
        for (int i = 0; i < 2 * TC_STAGES + 1; ++i) mbar_init(smem_u32(&bars[i]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TC_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    const uint32_t done_bar = smem_u32(&bars[2 * TC_STAGES]);

    if (warp == 0 && lane == 0) {
        // ------------------------------------------------ TMA producer
        int issued = 0;
        for (int i = 0; i < nkb; ++i) {
            const int s = i % TC_STAGES;
            const int r = i / TC_STAGES;
            if (r > 0 && !mbar_wait(smem_u32(&bars[TC_STAGES + s]), (uint32_t)((r - 1) & 1))) {
                atomicExch(&s_fail, 1);
                break;
            }
            if (*(volatile int*)&s_fail) break;
            const uint32_t fb = smem_u32(&bars[s]);
            uint8_t* st = smem + (size_t)s * TC_STAGE_BYTES;
            mbar_expect_tx(fb, TC_STAGE_BYTES);
            const int kc = (kb0 + i) * TC_BK;
            tma_load_2d(smem_u32(st), &map_vhi, fb, kc, t0);
            tma_load_2d(smem_u32(st + TC_A_BYTES), &map_vlo, fb, kc, t0);
            tma_load_2d(smem_u32(st + 2 * TC_A_BYTES), &map_mhi, fb, kc, e0);
            tma_load_2d(smem_u32(st + 2 * TC_A_BYTES + TC_B_BYTES), &map_mlo, fb, kc, e0);
            issued = i + 1;
        }
        // drain: every stage that was armed must have landed before the CTA leaves
        if (*(volatile int*)&s_fail) {
            for (int i = max(0, issued - TC_STAGES); i < issued; ++i)
                mbar_wait(smem_u32(&bars[i % TC_STAGES]), (uint32_t)((i / TC_STAGES) & 1));
        }
    } else if (warp == 1 && lane == 0) {
        // ------------------------------------------------ MMA issuer
        const uint32_t idesc = umma_idesc_bf16(TC_BM, TC_BN);
        for (int i = 0; i < nkb; ++i) {
            const int s = i % TC_STAGES;
            const int r = i / TC_STAGES;
            if (!mbar_wait(smem_u32(&bars[s]), (uint32_t)(r & 1))) {
                atomicExch(&s_fail, 1);
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            uint8_t* st = smem + (size_t)s * TC_STAGE_BYTES;
            const uint64_t dAh = umma_desc(smem_u32(st), Sh::SBO, Sh::LAYOUT);
            const uint64_t dAl = umma_desc(smem_u32(st + TC_A_BYTES), Sh::SBO, Sh::LAYOUT);
            const uint64_t dBh = umma_desc(smem_u32(st + 2 * TC_A_BYTES), Sh::SBO, Sh::LAYOUT);
            const uint64_t dBl = umma_desc(smem_u32(st + 2 * TC_A_BYTES + TC_B_BYTES), Sh::SBO, Sh::LAYOUT);
#pragma unroll
            for (int kk = 0; kk < TC_BK / 16; ++kk) {
                const uint64_t adv = (uint64_t)(kk * 32) >> 4;  // 16 bf16 = 32 B along K
                const uint32_t acc0 = (i > 0 || kk > 0) ? 1u : 0u;
                umma_bf16(tmem, dAh + adv, dBh + adv, idesc, acc0);
                umma_bf16(tmem, dAh + adv, dBl + adv, idesc, 1u);
                umma_bf16(tmem, dAl + adv, dBh + adv, idesc, 1u);
            }
            umma_commit(smem_u32(&bars[TC_STAGES + s]));  // stage free once these MMAs finish
        }
        umma_commit(done_bar);  // accumulator complete (also after a failure: drains issued MMAs)
    }
    __syncwarp();

    // ------------------------------------------------ epilogue (all four warps)
    bool ok = mbar_wait(done_bar, 0u);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!ok) atomicExch(&s_fail, 1);
    __syncthreads();
    if (!s_fail && nkb > 0) {
        const int row = t0 + warp * 32 + lane;
        float* out = part + ((size_t)blockIdx.z * T_pad + row) * part_cols + e0;
#pragma unroll 1
        for (int c = 0; c < TC_BN / 32; ++c) {
            uint32_t r[32];
            tmem_ld_32x32b_x32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(c * 32), r);
            float4* o4 = (float4*)(out + c * 32);
#pragma unroll
            for (int q = 0; q < 8; ++q)
                o4[q] = make_float4(__uint_as_float(r[4 * q]), __uint_as_float(r[4 * q + 1]),
                                    __uint_as_float(r[4 * q + 2]), __uint_as_float(r[4 * q + 3]));
        }
    } else if (nkb == 0) {
        const int row = t0 + warp * 32 + lane;
        float* out = part + ((size_t)blockIdx.z * T_pad + row) * part_cols + e0;
        for (int c = 0; c < TC_BN; ++c) out[c] = 0.0f;
    }
    if (s_fail && threadIdx.x == 0) atomicExch(err, 1);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS)
                     : "memory");
    }
}

// egm[t][e] = sum_z part[z][t][e] (split order, FP64), t < T, e < n_e.
__global__ void tc_reduce_kernel(int64_t T, int64_t n_e, int64_t T_pad, int64_t part_cols, int splits,
                                 const float* __restrict__ part, float* __restrict__ egm) {
    const int64_t total = T * n_e;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = i / n_e, e = i % n_e;
        double s = 0.0;
        for (int z = 0; z < splits; ++z) s += (double)part[((size_t)z * T_pad + t) * part_cols + e];
        egm[i] = (float)s;
    }
}

// hi = bf16(x), lo = bf16(x - hi); zero padding up to [rows_out][ld_out].
template <typename S>
__global__ void split_bf16_kernel(int64_t rows, int64_t cols, const S* __restrict__ src, int64_t ld,
                                  __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo, int64_t rows_out,
                                  int64_t ld_out) {
    const int64_t total = rows_out * ld_out;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = i / ld_out, c = i % ld_out;
        double x = (r < rows && c < cols) ? (double)src[r * ld + c] : 0.0;
        __nv_bfloat16 h = __float2bfloat16_rn((float)x);
        __nv_bfloat16 l = __float2bfloat16_rn((float)(x - (double)__bfloat162float(h)));
        hi[i] = h;
        lo[i] = l;
    }
}

namespace {

PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, []() {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    });
    return fn;
}

// Tensor map of a [rows][cols_k] BF16 operand, boxes of box_rows x bk (rows
// past the end read as zeros), swizzled to match the MMA descriptors.
bool make_map(CUtensorMap* m, const void* base, int64_t rows, int64_t cols_k, int box_rows, int bk) {
    auto enc = get_encode();
    if (!enc) return false;
    cuuint64_t dims[2] = {(cuuint64_t)cols_k, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)cols_k * 2};
    cuuint32_t box[2] = {(cuuint32_t)bk, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, bk == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// Split-K: at least ~4 CTAs per SM, and at most kMaxKPerSplit K values
// accumulated in one FP32 TMEM accumulator.  Long FP32 accumulation chains are
// the dominant error of the split-BF16 contraction (the dipole sum cancels), so
// each accumulator is kept short and the slices are summed in FP64.
constexpr int64_t kMaxKPerSplit = 8192;

// The tile configurations: (BN, BK, stages), their kernels and shared memory.
struct TcConfig {
    int bn, bk, stages;
    const void* fn;
    size_t smem;
};
template <int BN, int BK, int ST>
constexpr TcConfig tc_config() {
    return TcConfig{BN, BK, ST, (const void*)egm_bf16x3_kernel<BN, BK, ST>, TcShape<BN, BK, ST>::SMEM};
}
const TcConfig kTcConfigs[] = {tc_config<128, 64, 3>(), tc_config<256, 64, 2>(), tc_config<256, 32, 4>(),
                               tc_config<128, 32, 6>()};
constexpr int kTcNumConfigs = 4;
// 128 x 256 tiles, 2 stages of BK 64: the fastest at 1000 x 519,533 x 2048
// (5.09 ms against 5.78 ms for 128 x 128; the BK-32 rings took 8.7 and 10.7 ms).
constexpr int kTcDefaultConfig = 1;

// Columns of the split-K partial tiles: n_e_pad rounded up to the tile width.
int64_t partial_cols(int64_t E_pad, int bn) { return (E_pad + bn - 1) / bn * bn; }

void splits_for(const TcConfig& c, int64_t T_pad, int64_t E_pad, int64_t K_pad, int* splits, int* kb_per) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t tiles = (T_pad / TC_BM) * (partial_cols(E_pad, c.bn) / c.bn);
    const int64_t nkb = K_pad / c.bk;
    const int64_t max_kb = kMaxKPerSplit / c.bk;
    int64_t s = std::max<int64_t>(1, (4LL * sms + tiles - 1) / tiles);
    s = std::max<int64_t>(s, (nkb + max_kb - 1) / max_kb);
    s = std::min<int64_t>(s, std::max<int64_t>(1, nkb / 8));
    s = std::min<int64_t>(s, 65535);
    int64_t per = (nkb + s - 1) / s;
    s = (nkb + per - 1) / per;
    *splits = (int)s;
    *kb_per = (int)per;
}

int64_t workspace_of(const TcConfig& c, int64_t T_pad, int64_t E_pad, int64_t K_pad) {
    int s = 1, per = 1;
    splits_for(c, T_pad, E_pad, K_pad, &s, &per);
    return kTcHeader + (int64_t)s * T_pad * partial_cols(E_pad, c.bn) * 4;
}

}  // namespace

int bf16x3_config_count() { return kTcNumConfigs; }

int64_t bf16x3_workspace(int64_t T_pad, int64_t n_e_pad, int64_t K_pad) {
    if (T_pad <= 0 || n_e_pad <= 0 || K_pad <= 0) return -1;
    int64_t w = 0;
    for (const TcConfig& c : kTcConfigs) w = std::max(w, workspace_of(c, T_pad, n_e_pad, K_pad));
    return w;
}

int split_bf16(int64_t rows, int64_t cols, const void* src, int64_t ld, bool src_f64, uint16_t* hi, uint16_t* lo,
               int64_t rows_out, int64_t ld_out, cudaStream_t stream) {
    const int64_t total = rows_out * ld_out;
    const unsigned blocks = (unsigned)std::min<int64_t>((total + 255) / 256, 8192);
    if (src_f64)
        split_bf16_kernel<double><<<blocks, 256, 0, stream>>>(rows, cols, (const double*)src, ld, (__nv_bfloat16*)hi,
                                                              (__nv_bfloat16*)lo, rows_out, ld_out);
    else
        split_bf16_kernel<float><<<blocks, 256, 0, stream>>>(rows, cols, (const float*)src, ld, (__nv_bfloat16*)hi,
                                                             (__nv_bfloat16*)lo, rows_out, ld_out);
    PHS_CUDA_TRY(cudaGetLastError());
    return PHS_OK;
}

int contract_bf16x3(int64_t T, int64_t n_e, int64_t T_pad, int64_t E_pad, int64_t K_pad, const uint16_t* Vhi,
                    const uint16_t* Vlo, const uint16_t* Mhi, const uint16_t* Mlo, float* egm, void* work,
                    cudaStream_t stream, int config) {
    if (config < 0) config = kTcDefaultConfig;
    if (config >= kTcNumConfigs) return PHS_ERR_BAD_ARG;
    const TcConfig& c = kTcConfigs[config];
    if (T <= 0 || n_e <= 0 || T > T_pad || n_e > E_pad || T_pad % TC_BM || E_pad % 128 || K_pad % 64 ||
        K_pad <= 0 || !Vhi || !Vlo || !Mhi || !Mlo || !egm || !work)
        return PHS_ERR_BAD_ARG;
    const int64_t Ew = partial_cols(E_pad, c.bn);
    if (T_pad / TC_BM > 65535 || Ew / c.bn > 65535 || K_pad / c.bk > INT32_MAX) return PHS_ERR_BAD_ARG;
    // 16-byte aligned bases and row strides for TMA
    if (((uintptr_t)Vhi | (uintptr_t)Vlo | (uintptr_t)Mhi | (uintptr_t)Mlo) & 15) return PHS_ERR_BAD_ARG;
    CUtensorMap mv_hi, mv_lo, mm_hi, mm_lo;
    if (!make_map(&mv_hi, Vhi, T_pad, K_pad, TC_BM, c.bk) || !make_map(&mv_lo, Vlo, T_pad, K_pad, TC_BM, c.bk) ||
        !make_map(&mm_hi, Mhi, E_pad, K_pad, c.bn, c.bk) || !make_map(&mm_lo, Mlo, E_pad, K_pad, c.bn, c.bk))
        return PHS_ERR_CUDA;
    int splits = 1, per = 1;
    splits_for(c, T_pad, E_pad, K_pad, &splits, &per);
    int* err = (int*)work;
    float* part = (float*)((char*)work + kTcHeader);
    PHS_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), stream));
    // the dynamic shared-memory opt-in is a per-device attribute of each kernel
    {
        static std::mutex mu;
        static bool attr_set[64][kTcNumConfigs] = {};
        int dev = 0;
        PHS_CUDA_TRY(cudaGetDevice(&dev));
        std::lock_guard<std::mutex> lk(mu);
        if (dev < 0 || dev >= 64 || !attr_set[dev][config]) {
            PHS_CUDA_TRY(cudaFuncSetAttribute(c.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c.smem));
            if (dev >= 0 && dev < 64) attr_set[dev][config] = true;
        }
    }
    dim3 grid((unsigned)(T_pad / TC_BM), (unsigned)(Ew / c.bn), (unsigned)splits);
    int nkb_total = (int)(K_pad / c.bk), T_pad_i = (int)T_pad, Ew_i = (int)Ew;
    void* args[] = {(void*)&mv_hi, (void*)&mv_lo, (void*)&mm_hi, (void*)&mm_lo, (void*)&nkb_total, (void*)&per,
                    (void*)&T_pad_i, (void*)&Ew_i, (void*)&part, (void*)&err};
    PHS_CUDA_TRY(cudaLaunchKernel(c.fn, grid, dim3(TC_THREADS), args, c.smem, stream));
    const int64_t total = T * n_e;
    tc_reduce_kernel<<<(unsigned)std::min<int64_t>((total + 255) / 256, 8192), 256, 0, stream>>>(
        T, n_e, T_pad, Ew, splits, part, egm);
    PHS_CUDA_TRY(cudaGetLastError());
    return PHS_OK;
}

// Error word of the last contraction that used `work`, read after `stream`
// has finished it (synchronises the stream).
int bf16x3_status(const void* work, cudaStream_t stream) {
    if (!work) return PHS_ERR_BAD_ARG;
    PHS_CUDA_TRY(cudaStreamSynchronize(stream));
    int herr = 0;
    PHS_CUDA_TRY(cudaMemcpy(&herr, work, sizeof(int), cudaMemcpyDeviceToHost));
    return herr ? PHS_ERR_TIMEOUT : PHS_OK;
}

}  // namespace phs
