// Time-stepping engine of the PyHeartSim B200 path.
//
// One persistent kernel advances every active simulation instance.  Each
// instance is owned by a "team" of CTAs that synchronise with their own bounded
// barrier, so instances of different sizes progress independently inside one
// launch.  Per step and instance:
//
//   RHS phase   RK4 reaction (simulation/simulation_gpu.py:27-43, 71-130) of
//               every voxel, then, after a team barrier, the Crank-Nicolson
//               right-hand side b = u* + dt/2 L u*  (simulation/simulation_gpu.py:245)
//               and the initial residual r0 = b - A x0  (A = I - dt/2 L, :321-322)
//   GMRES       restarted GMRES on A (CuPy semantics of the reference's call at
//               simulation/simulation_gpu.py:253): classical Gram-Schmidt, the
//               Hessenberg least-squares solved by Givens rotations on device,
//               FP64 dot products and norms whatever the storage type
//   update      x += V y, then either the true-residual test of the next cycle
//               (full_cycles = 1, CuPy semantics) or the Givens estimate
//               (full_cycles = 0, early exit)
//
// The Laplacian is applied matrix-free from a compacted table of six neighbour
// indices and six premultiplied coefficients per voxel, which is the CSR matrix
// of simulation/simulation_gpu.py:138-225 without the explicit zeros.
//
// Reductions are deterministic: every tile of kThreads*VPT voxels writes its
// own FP64 partials and the last CTA of the team to arrive at the barrier sums
// the tiles in index order.  The result therefore does not depend on the team
// size, so an instance gives bit-identical results alone and in a batch.
#include <cuda_runtime.h>
#include <cuda/atomic>
#include <climits>
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <algorithm>
#include <vector>
#include <map>

#include "../../include/phs.h"
#include "phs_common.cuh"

namespace phs {

// ------------------------------------------------------------------ device types
struct alignas(128) TeamSync {
    unsigned int count;
    unsigned int gen;
    unsigned int pad[30];
};

enum Action : int {
    ACT_NONE = 0,
    ACT_ZERO_B = 1,      // ||b|| == 0: the solve returns b
    ACT_DONE = 2,        // residual test passed: the solve returns x
    ACT_CYCLE = 3,       // start an Arnoldi cycle (V0 holds r, s[0] = 1/||r||)
    ACT_NEXT_J = 4,      // continue the cycle with column j+1
    ACT_UPDATE_FINAL = 5,// x += V y, solve finished (Givens estimate)
    ACT_UPDATE_CHECK = 6,// x += V y, then the true-residual test
    ACT_FAIL = 7,        // non-finite norm: instance retired with an error
};

enum Phase : int { PH_PLAIN = 0, PH_RHS = 1, PH_DOTS = 2, PH_NORM = 3, PH_CHECK = 4 };

// Phase timer slots (nanoseconds of globaltimer, summed over steps).
enum ProfSlot : int {
    PF_RHS = 0, PF_RHS_WAIT, PF_A, PF_A_WAIT, PF_C, PF_C_WAIT, PF_X, PF_CHECK, PF_CHECK_WAIT,
    PF_COPY, PF_RHS1, PF_STEPS, PF_SOLVE_ITERS, PF_TEAM,
    PF_LEADER,      // time in the leader bodies of the team's barriers (whichever CTA led)
    PF_BARRIERS,    // team barriers passed
    kProfSlots = 16
};

struct Scalars {
    double R[(kMaxRestart + 1) * kMaxRestart];  // column j at R[j*(kMaxRestart+1) + i]
    double cs[kMaxRestart];
    double sn[kMaxRestart];
    double g[kMaxRestart + 1];
    double s[kMaxRestart + 1];      // v_j = s_j * V_j
    double coef[kMaxRestart + 1];   // coefficients published for the next phase
    double bnorm, atol_eff, rnorm, est;
    int action;
    int k;
    int iters_solve;                // Arnoldi steps of the current solve
    int iters_cap;                  // CuPy-style iteration count (restart per cycle)
};

struct InstState {
    long long step;        // steps completed
    int id_save;           // next history slot
    int pending;           // history slot owed for the last completed step (-1: none)
    int status;
    int hbuf;              // current gate buffer
    long long arnoldi;
    long long solves;
    int max_arnoldi;
    int nonconv;
    long long arnoldi_sq;  // sum over solves of (Arnoldi steps)^2
};

template <typename T>
struct InstDev {
    const int32_t* nb;      // [n*6]
    const int16_t* nbr;     // [ldv*4] compact neighbour table (decode_nb), or nullptr
    const int32_t* nbase;   // [ldv/512*4] its base offsets per 512-voxel block
    const T* coef;          // [n*6], or nullptr when every row is isotropic (cw, m6)
    const T* cw;            // [n] common coefficient of row n (isotropic rows)
    const uint8_t* m6;      // [n] neighbour presence bits of row n (isotropic rows)
    const int32_t* enb;     // [n*12] edge pairs (a0,b0,...,a5,b5) of anisotropic rows, or nullptr
    const T* ecf;           // [n*6] edge pair coefficients, or nullptr (D0 = I)
    const uint8_t* vflags;  // [n]
    const T* vparams;       // [n*5] or nullptr
    const uint8_t* stim;    // [n_steps]
    T* u;
    T* h0;
    T* h1;
    T* x;
    T* b;
    T* V;                   // [(m+1)*n]
    T* dx;                  // [n] last diffusion increment (extrapolated initial guess), or nullptr
    T* hist_u;              // [S*n]
    T* hist_h;              // [S*n] or nullptr
    int32_t* lat;           // [n]
    double* part;           // [n_tiles*kSlots]
    double* gpart;          // FP64: [n_groups*kSlots] sums of kGroupTiles consecutive tiles, or nullptr
    unsigned int* gcnt;     // FP64: [n_groups] arrivals of the current phase at each group
    Scalars* sc;
    TeamSync* sync;
    InstState* st;
    unsigned long long* prof;  // [kProfSlots] phase timers (CTA rank 0 of the team), or nullptr
    T params[5];
    T dt, half_dt, jmag;
    double tol, atol;
    long long n;
    long long ldv;          // padded voxel count (multiple of kPadVoxels): stride of V, length of per-voxel arrays
    long long n_steps;
    long long tb_steps;
    int n_tiles;
    int n_groups;           // ceil(n_tiles / kGroupTiles)
    int ps;                 // partial slots per (tile, warp): m + 2
    int model;
    int m;                  // restart length actually used: min(restart, n)
    int maxiter;
    int full_cycles;
    int stride;
    int n_samples;
    int save_h;
};

// ------------------------------------------------------------------ reaction
// Mitchell-Schaeffer / Aliev-Panfilov right-hand sides,
// simulation/simulation_gpu.py:27-43 (P_2d columns 15..19 in p[0..4]).
template <typename T>
__device__ __forceinline__ void reaction(int model, T u, T h, T J, const T* p, T& du, T& dh) {
    if (model == 0) {
        du = (h * (u * u) * (T(1) - u)) / p[2] - u / p[3] + J;
        dh = (u < p[4]) ? (T(1) - h) / p[0] : -h / p[1];
    } else {
        du = -p[0] * u * (u - p[1]) * (u - T(1)) - u * h + J;
        dh = (p[2] + p[3] * h / (u + p[4])) * (-h - p[0] * u * (u - p[1] - T(1)));
    }
}

// FP32 form of the same right-hand sides: the Mitchell-Schaeffer time
// constants enter as precomputed reciprocals (q[0] = 1/tau_open, q[1] =
// 1/tau_close, q[2] = 1/tau_in, q[3] = 1/tau_out, q[4] = v_gate) and the
// Aliev-Panfilov quotient uses the fast division; FP64 keeps the reference's
// divisions exactly.
__device__ __forceinline__ void reaction_fast(int model, float u, float h, float J, const float* q, float& du,
                                              float& dh) {
    if (model == 0) {
        du = h * (u * u) * (1.0f - u) * q[2] - u * q[3] + J;
        dh = (u < q[4]) ? (1.0f - h) * q[0] : -h * q[1];
    } else {
        du = -q[0] * u * (u - q[1]) * (u - 1.0f) - u * h + J;
        dh = (q[2] + q[3] * __fdividef(h, u + q[4])) * (-h - q[0] * u * (u - q[1] - 1.0f));
    }
}

template <typename T>
__device__ __forceinline__ void reaction_any(int model, T u, T h, T J, const T* p, T& du, T& dh) {
    if constexpr (sizeof(T) == 4) reaction_fast(model, u, h, J, p, du, dh);
    else reaction(model, u, h, J, p, du, dh);
}

// Classical RK4 with J held over the step, simulation/simulation_gpu.py:71-130.
// `p` holds P_2d columns 15..19 (FP64) or their FP32 form (see reaction_fast).
template <typename T>
__device__ __forceinline__ void rk4(int model, T u, T h, T J, const T* p, T dt, T& us, T& hs) {
    T k1u, k1h, k2u, k2h, k3u, k3h, k4u, k4h;
    reaction_any(model, u, h, J, p, k1u, k1h);
    T ut = u + T(0.5) * dt * k1u;
    T ht = h + T(0.5) * dt * k1h;
    reaction_any(model, ut, ht, J, p, k2u, k2h);
    ut = u + T(0.5) * dt * k2u;
    ht = h + T(0.5) * dt * k2h;
    reaction_any(model, ut, ht, J, p, k3u, k3h);
    ut = u + dt * k3u;
    ht = h + dt * k3h;
    reaction_any(model, ut, ht, J, p, k4u, k4h);
    us = u + (dt / T(6)) * (k1u + T(2) * k2u + T(2) * k3u + k4u);
    hs = h + (dt / T(6)) * (k1h + T(2) * k2h + T(2) * k3h + k4h);
}

// P_2d columns 15..19 -> the parameter form rk4<T> expects.
template <typename T>
__host__ __device__ __forceinline__ void model_form(int model, const T* p, T* q) {
    if (sizeof(T) == 4 && model == 0) {
        q[0] = T(1) / p[0];
        q[1] = T(1) / p[1];
        q[2] = T(1) / p[2];
        q[3] = T(1) / p[3];
        q[4] = p[4];
    } else {
        for (int i = 0; i < 5; ++i) q[i] = p[i];
    }
}

// ------------------------------------------------------------------ helpers
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bound of every device-side wait: 4 s of wall time or 2^26 polls.
constexpr unsigned long long kWaitNs = 4000000000ull;
constexpr unsigned int kWaitPolls = 1u << 26;

// Bulk L2 prefetch of [p, p + bytes) (p 16-byte aligned, bytes a multiple of 16).
__device__ __forceinline__ void prefetch_l2(const void* p, unsigned int bytes) {
    const unsigned long long g = (unsigned long long)__cvta_generic_to_global(p);
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(g), "r"(bytes) : "memory");
}

// ------------------------------------------------------------------ staging ring
// Staged step kernels (RING > 0) add one producer warp to the 256 consumer
// threads.  For every tile loop of a phase the consumers publish a job (the
// arrays the phase streams and their bytes per voxel); the producer copies
// each of the CTA's tiles' contiguous slices of every array into a stage of a
// shared-memory ring with 1-D cp.async.bulk, signalled on the stage's "full"
// mbarrier, and refills a stage once all consumer warps have arrived on its
// "empty" mbarrier.  Consumers read the tile from shared memory; the stencil's
// neighbour gathers and the scattered accesses stay on global memory.
constexpr int kStageMaxArr = 12;    // arrays per stage
constexpr int kMaxStages = 6;       // ring depth limit
constexpr int kRingHeader = 1024;   // barriers and jobs ahead of the ring in dynamic shared memory

struct StageJob {
    const char* src[kStageMaxArr];  // array base (voxel 0)
    int bytes[kStageMaxArr];        // bytes of one tile's slice
    int off[kStageMaxArr];          // offset of the slice in a stage
    int n_arr;
    int stage_bytes;
    int n_stages;
    int tile0, step, n_tiles;       // the CTA's tiles: tile0, tile0 + step, ... < n_tiles
    int quit;
};
struct RingHeader {
    unsigned long long full[kMaxStages];
    unsigned long long empty[kMaxStages];
    StageJob job[2];
    int stop;                       // a bounded stage wait gave up: later waits return at once
};
static_assert(sizeof(RingHeader) <= kRingHeader, "ring header");

// Consumer-only CTA barrier: __syncthreads without a producer warp, else named
// barrier 1 over the 256 consumer threads.
template <bool ST>
__device__ __forceinline__ void csync() {
    if constexpr (ST) asm volatile("bar.sync 1, %0;" ::"n"(kThreads) : "memory");
    else __syncthreads();
}
// Job hand-over on named barrier 2: consumers arrive, the producer waits.
__device__ __forceinline__ void job_arrive() { asm volatile("bar.arrive 2, %0;" ::"n"(kThreads + 32) : "memory"); }
__device__ __forceinline__ void job_wait() { asm volatile("bar.sync 2, %0;" ::"n"(kThreads + 32) : "memory"); }

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint32_t a, unsigned int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t a) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(a) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t a, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t a, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    return ok != 0u;
}
// Bounded wait for the phase of parity `parity` of the mbarrier at a.  Gives up
// after 4 s or 2^26 polls (sets *stop and the abort word), and at once once
// *stop is set when `heed_stop`; returns whether the phase completed.
__device__ __forceinline__ bool mbar_wait(uint32_t a, uint32_t parity, volatile int* stop, unsigned int* abort_word,
                                          bool heed_stop = true) {
    if (mbar_try(a, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (unsigned int polls = 0;; ++polls) {
        if (mbar_try(a, parity)) return true;
        if (heed_stop && *stop) return false;
        if (polls > kWaitPolls || global_ns() - t0 > kWaitNs) {
            *stop = 1;
            atomicOr(abort_word, 1u);
            return false;
        }
    }
}
// 1-D bulk copy global -> shared (both 16-byte aligned, bytes a multiple of 16),
// completion counted on the mbarrier at mbar.  No multicast.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"((unsigned long long)__cvta_generic_to_global(src)), "r"(bytes), "r"(mbar)
                 : "memory");
}
// Orders this thread's generic-proxy global accesses before later async-proxy
// (bulk copy) ones.
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }

// Consumer side of the staging ring.  A phase lists its arrays with add()
// (every consumer thread makes the same calls, so all agree on the offsets;
// thread 0 writes the job), then publish() hands the job to the producer and
// returns the ring depth, 0 when the phase runs unstaged; acquire() waits for
// the next tile's stage and release() marks the calling warp done with it.
template <int RING, int TILE, typename T>
struct Stager {
    RingHeader* rh;
    unsigned char* ring;
    int job_buf;
    int lay_off, lay_n;
    int nst, sg;          // ring depth of the phase, stage of the current tile
    unsigned int cpar;    // parity to wait for on each full barrier

    __device__ __forceinline__ void begin() {
        lay_off = 0;
        lay_n = 0;
    }
    __device__ __forceinline__ int add(const void* base, int elem) {
        const int o = lay_off;
        if (threadIdx.x == 0 && lay_n < kStageMaxArr) {
            StageJob& J = rh->job[job_buf];
            J.src[lay_n] = static_cast<const char*>(base);
            J.bytes[lay_n] = TILE * elem;
            J.off[lay_n] = o;
        }
        lay_off += TILE * elem;
        ++lay_n;
        return o;
    }
    // basis vectors a phase may stage after its fixed arrays: as many as keep
    // the ring at least two stages deep
    __device__ __forceinline__ int vec_cap() const {
        const int c = (RING / 2 - lay_off) / (TILE * (int)sizeof(T));
        return max(0, min(c, kStageMaxArr - lay_n));
    }
    __device__ __forceinline__ int publish(int rank, int P, int n_tiles) {
        nst = (lay_off > 0 && lay_n <= kStageMaxArr) ? RING / lay_off : 0;
        if (nst > kMaxStages) nst = kMaxStages;
        if (rank >= n_tiles) nst = 0;
        if (nst == 0) return 0;
        if (threadIdx.x == 0) {
            StageJob& J = rh->job[job_buf];
            J.n_arr = lay_n;
            J.stage_bytes = lay_off;
            J.n_stages = nst;
            J.tile0 = rank;
            J.step = P;
            J.n_tiles = n_tiles;
            J.quit = 0;
        }
        fence_proxy_async_global();   // this thread's global writes before the bulk reads
        csync<true>();
        job_arrive();
        job_buf ^= 1;
        sg = -1;
        return nst;
    }
    __device__ __forceinline__ const unsigned char* acquire(unsigned int* abort_word) {
        if (++sg == nst) sg = 0;
        mbar_wait(smem_u32(&rh->full[sg]), (cpar >> sg) & 1u, &rh->stop, abort_word);
        cpar ^= 1u << sg;
        return ring + sg * lay_off;
    }
    __device__ __forceinline__ void release() {
        __syncwarp();
        if ((threadIdx.x & 31) == 0) mbar_arrive(smem_u32(&rh->empty[sg]));
    }
    // hands the producer warp its last job
    __device__ __forceinline__ void quit() {
        if (threadIdx.x == 0) rh->job[job_buf].quit = 1;
        csync<true>();
        job_arrive();
    }
};

struct SharedCtl {
    int last;
    unsigned int gen;
    int action;
    int k;
    int abort;
    double sj;
    double bnorm;
};

// Bounded team barrier.  The last CTA to arrive runs `leader` (whole CTA)
// before releasing the others.  Returns false when the wait gave up or another
// team aborted; the kernel then leaves all loops.
//
// The release word carries, besides a barrier counter (bits 9-31), the
// action (bits 0-2) and cycle length k (bits 3-8) the leader left in `sc`, so
// the waiting CTAs learn them from the load that releases them (ctl.action,
// ctl.k).  Ordering: the arrival is an acq_rel RMW (the CTA's writes, made
// visible to thread 0 by the CTA barrier and the fence, precede it; the
// leader's RMW acquires every earlier arrival); the release is a release store
// and the waiters' polls are acquire loads.
constexpr unsigned int kGenShift = 9;
template <bool ST, typename Leader>
__device__ __forceinline__ bool team_sync(TeamSync* ts, int P, unsigned int* abort_word, SharedCtl& ctl,
                                          const Scalars* sc, unsigned long long* prof, Leader&& leader) {
    csync<ST>();
    if (threadIdx.x == 0) {
        cuda::atomic_ref<unsigned int, cuda::thread_scope_device> gen(ts->gen);
        cuda::atomic_ref<unsigned int, cuda::thread_scope_device> cnt(ts->count);
        unsigned int g = gen.load(cuda::memory_order_relaxed);
        __threadfence();
        unsigned int a = cnt.fetch_add(1u, cuda::memory_order_acq_rel);
        ctl.last = (a == (unsigned int)(P - 1));
        ctl.gen = g;
        ctl.abort = 0;
    }
    csync<ST>();
    if (ctl.last) {
        const unsigned long long tl = (prof && threadIdx.x == 0) ? global_ns() : 0ull;
        leader();
        csync<ST>();
        if (threadIdx.x == 0) {
            if (prof) {
                atomicAdd(prof + PF_LEADER, global_ns() - tl);
                atomicAdd(prof + PF_BARRIERS, 1ull);
            }
            cuda::atomic_ref<unsigned int, cuda::thread_scope_device> gen(ts->gen);
            cuda::atomic_ref<unsigned int, cuda::thread_scope_device> cnt(ts->count);
            const int act = __ldcg(&sc->action), k = __ldcg(&sc->k);
            ctl.action = act;
            ctl.k = k;
            cnt.store(0u, cuda::memory_order_relaxed);
            const unsigned int word = ((((ctl.gen >> kGenShift) + 1u) << kGenShift)) | ((unsigned int)(k & 63) << 3) |
                                      (unsigned int)(act & 7);
            gen.store(word, cuda::memory_order_release);
        }
    } else if (threadIdx.x == 0) {
        cuda::atomic_ref<unsigned int, cuda::thread_scope_device> gen(ts->gen);
        cuda::atomic_ref<unsigned int, cuda::thread_scope_device> ab(*abort_word);
        unsigned long long t0 = global_ns();
        unsigned int polls = 0;
        unsigned int word;
        while ((word = gen.load(cuda::memory_order_acquire)) == ctl.gen) {
            if (ab.load(cuda::memory_order_relaxed) != 0u) { ctl.abort = 1; break; }
            if (++polls > kWaitPolls || global_ns() - t0 > kWaitNs) {
                ab.fetch_or(1u, cuda::memory_order_relaxed);
                ctl.abort = 1;
                break;
            }
            __nanosleep(64);
        }
        ctl.action = (int)(word & 7u);
        ctl.k = (int)((word >> 3) & 63u);
    }
    csync<ST>();
    return ctl.abort == 0;
}

// The six (neighbour, coefficient) pairs of row n, as 8/16-byte vector loads.
__device__ __forceinline__ void load_nb(const int32_t* nb, long long n, int32_t (&q)[6]) {
    const int2* p = reinterpret_cast<const int2*>(nb + 6 * n);
    int2 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
    q[0] = a.x; q[1] = a.y; q[2] = b.x; q[3] = b.y; q[4] = c.x; q[5] = c.y;
}
__device__ __forceinline__ void load_coef(const float* cf, long long n, float (&c)[6]) {
    const float2* p = reinterpret_cast<const float2*>(cf + 6 * n);
    float2 a = __ldg(p), b = __ldg(p + 1), d = __ldg(p + 2);
    c[0] = a.x; c[1] = a.y; c[2] = b.x; c[3] = b.y; c[4] = d.x; c[5] = d.y;
}
__device__ __forceinline__ void load_coef(const double* cf, long long n, double (&c)[6]) {
    const double2* p = reinterpret_cast<const double2*>(cf + 6 * n);
    double2 a = __ldg(p), b = __ldg(p + 1), d = __ldg(p + 2);
    c[0] = a.x; c[1] = a.y; c[2] = b.x; c[3] = b.y; c[4] = d.x; c[5] = d.y;
}

// Compact neighbour table.  In the row order of a lattice (x fastest) the
// present +x and -x neighbours of voxel n are n + 1 and n - 1 (slots 0 and 1
// of the reference's column order), and the other four slots hold offsets that
// change slowly along the rows: base[r] of the voxel's 512-voxel block plus the
// voxel's int16 residual r (slots 2..5).  Exact for every present neighbour
// (checked when the table is built); absent ones decode to unused values.
__device__ __forceinline__ void decode_nb(short4 r, int4 b, long long n, int32_t (&q)[6]) {
    const int32_t nn = (int32_t)n;
    q[0] = nn + 1;
    q[1] = nn - 1;
    q[2] = nn + b.x + r.x;
    q[3] = nn + b.y + r.y;
    q[4] = nn + b.z + r.z;
    q[5] = nn + b.w + r.w;
}

// Coefficients of row n: one common value and a presence mask for isotropic
// rows (D0 = I gives c_n / Delta^2 on every present neighbour), else six values.
template <typename T>
__device__ __forceinline__ void row_coef(const T* coef, const T* cw, const uint8_t* m6, long long n, T (&c)[6]) {
    if (cw) {
        const T w = cw[n];
        const unsigned mk = __ldg(m6 + n);
#pragma unroll
        for (int k = 0; k < 6; ++k) c[k] = ((mk >> k) & 1u) ? w : T(0);
    } else {
        load_coef(coef, n, c);
    }
}

// Matrix-free row of L applied to `vec` at voxel n (coefficients already loaded);
// all six gathers are issued before they are combined.
template <typename T>
__device__ __forceinline__ T lap_row(const T* vec, T vn, const int32_t (&q)[6], const T (&c)[6]) {
    T g[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) g[k] = (c[k] != T(0)) ? vec[q[k]] : vn;
    T acc = T(0);
#pragma unroll
    for (int k = 0; k < 6; ++k) acc += c[k] * (g[k] - vn);
    return acc;
}

// Edge cross terms of an anisotropic row n (simulation/simulation_gpu.py:199-217):
// six antisymmetric pairs ecf[p] * (vec[a_p] - vec[b_p]); all gathers first.
template <typename T>
__device__ __forceinline__ T edge_row(const T* vec, const int32_t* enb, const T* ecf, long long n) {
    const int4* pi = reinterpret_cast<const int4*>(enb + 12 * n);
    const int4 i0 = __ldg(pi), i1 = __ldg(pi + 1), i2 = __ldg(pi + 2);
    const int32_t q[12] = {i0.x, i0.y, i0.z, i0.w, i1.x, i1.y, i1.z, i1.w, i2.x, i2.y, i2.z, i2.w};
    T g[6];
    load_coef(ecf, n, g);
    T va[6], vb[6];
#pragma unroll
    for (int p = 0; p < 6; ++p) {
        va[p] = (g[p] != T(0)) ? vec[q[2 * p]] : T(0);
        vb[p] = (g[p] != T(0)) ? vec[q[2 * p + 1]] : T(0);
    }
    T acc = T(0);
#pragma unroll
    for (int p = 0; p < 6; ++p) acc += g[p] * (va[p] - vb[p]);
    return acc;
}


// Basis vectors whose loads are issued together: FP32 tiles hold four voxels
// per thread (four loads per vector already), FP64 tiles one, and the FP64
// plain form's GMRES(50) cycles pass over up to 50 vectors per phase, so its
// chunks are four times longer to keep as many loads in flight.
template <typename T>
constexpr int kChunkOf = sizeof(T) == 8 ? 16 : 4;
template <typename T>
constexpr bool kWarpParts = sizeof(T) == 4;
// FP64 partial sums are combined in fixed groups of this many consecutive tiles
// by whichever CTA finishes a group's last tile, so the leader reads one
// partial per group (GMRES(50) reduces up to 51 slots per barrier).
constexpr int kGroupTiles = 8;
constexpr int kMaxGroupWalk = 32;   // tiles a CTA counts in per pass

// ------------------------------------------------------------------ the kernel
// EDGE: the launch carries anisotropic instances (edge cross terms); the
// isotropic launches compile without that code.
template <typename T, int VPT, int MINB, bool EDGE, int RING, bool NBC>
__global__ void __launch_bounds__(kThreads + (RING > 0 ? 32 : 0), MINB)
step_kernel(const InstDev<T>* __restrict__ insts, const int4* __restrict__ cta_map,
            long long n_steps_launch, unsigned int* abort_word) {
    constexpr bool ST = RING > 0;   // staged: producer warp + shared-memory ring (FP32 only)
    static_assert(!ST || sizeof(T) == 4, "staged kernels are FP32");
    // NBC: every instance of the launch has a compact neighbour table (decode_nb)
    static_assert(!(ST && NBC), "staged kernels choose the table per instance");
    constexpr int TILE = kThreads * VPT;
    constexpr int kChunk = kChunkOf<T>;
    const int4 cm = cta_map[blockIdx.x];
    const int rank = cm.y;
    const int P = cm.z;

    __shared__ InstDev<T> I;
    __shared__ SharedCtl ctl;
    __shared__ double shc[kMaxRestart + 1];
    __shared__ long long sh_step0;
    __shared__ int sh_id_save, sh_pending, sh_hbuf, sh_status;
    // staged kernels: ring header (mbarriers, jobs) and the ring itself
    extern __shared__ __align__(128) unsigned char dyn_smem[];
    RingHeader* const rh = reinterpret_cast<RingHeader*>(dyn_smem);
    unsigned char* const ring = dyn_smem + kRingHeader;

    if (threadIdx.x == 0) {
        I = insts[cm.x];
        sh_step0 = __ldcg(&I.st->step);
        sh_id_save = __ldcg(&I.st->id_save);
        sh_pending = __ldcg(&I.st->pending);
        sh_hbuf = __ldcg(&I.st->hbuf);
        sh_status = __ldcg(&I.st->status);
        if constexpr (ST) {
            for (int q = 0; q < kMaxStages; ++q) {
                mbar_init(smem_u32(&rh->full[q]), 1u);
                mbar_init(smem_u32(&rh->empty[q]), (unsigned)kWarps);
            }
            rh->stop = 0;
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
    }
    __syncthreads();

    if constexpr (ST) {
        // ---- producer warp: copies the slices of each published job's tiles
        if (threadIdx.x >= kThreads) {
            const int pl = threadIdx.x - kThreads;
            const uint32_t ring_u32 = smem_u32(ring);
            volatile int* stop = &rh->stop;
            unsigned int epar = 0xffffffffu;   // parity to wait for on each empty barrier (fresh: passes)
            unsigned int fpar = 0u;            // fills of each stage, mod 2
            unsigned int used = 0u;
            bool dead = false;                 // an empty-barrier wait gave up: issue nothing more
            int jb = 0;
            for (;;) {
                job_wait();
                const StageJob* J = &rh->job[jb];
                jb ^= 1;
                if (J->quit) break;
                fence_proxy_async_global();
                const int na = J->n_arr, sbytes = J->stage_bytes, nst = J->n_stages;
                const int tstep = J->step, nt = J->n_tiles;
                const char* src = pl < na ? J->src[pl] : nullptr;
                const int bytes = pl < na ? J->bytes[pl] : 0;
                const int off = pl < na ? J->off[pl] : 0;
                int sg = 0;
                for (int tile = J->tile0; tile < nt && !dead; tile += tstep) {
                    const uint32_t fb = smem_u32(&rh->full[sg]);
                    bool ok = true;
                    if (pl == 0) ok = mbar_wait(smem_u32(&rh->empty[sg]), (epar >> sg) & 1u, stop, abort_word);
                    ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
                    if (!ok) {
                        dead = true;
                        break;
                    }
                    epar ^= 1u << sg;
                    if (pl == 0) mbar_expect_tx(fb, (uint32_t)sbytes);
                    __syncwarp();
                    if (pl < na) bulk_g2s(ring_u32 + (uint32_t)(sg * sbytes + off), src + (size_t)tile * bytes, (uint32_t)bytes, fb);
                    fpar ^= 1u << sg;
                    used |= 1u << sg;
                    if (++sg == nst) sg = 0;
                }
            }
            // every copy this CTA issued has landed before it exits
            if (pl == 0)
                for (int q = 0; q < kMaxStages; ++q)
                    if ((used >> q) & 1u) mbar_wait(smem_u32(&rh->full[q]), ((fpar >> q) & 1u) ^ 1u, stop, abort_word, false);
            __syncwarp();
            return;
        }
    }

    const long long N = I.n;
    const int ps = I.ps;
    const bool grouped = !kWarpParts<T> && I.gpart != nullptr;
    const int nparts = kWarpParts<T> ? I.n_tiles * kWarps : (grouped ? I.n_groups : I.n_tiles);
    const double* psum = grouped ? I.gpart : I.part;   // what the leader sums
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    Scalars* sc = I.sc;
    long long step = sh_step0;
    long long step_end = step + n_steps_launch;
    if (step_end > I.n_steps) step_end = I.n_steps;
    int id_save = sh_id_save;
    int pending = sh_pending;
    int hbuf = sh_hbuf;
    bool retired = (sh_status == PHS_ERR_NONFINITE);
    bool aborted = false;
    // optional phase timer: thread 0 of CTA rank 0 of each team
    __shared__ unsigned long long pf[kProfSlots];
    __shared__ unsigned long long pf_t;
    const bool prof_on = (I.prof != nullptr) && rank == 0;
    if (prof_on && threadIdx.x == 0) {
        for (int i = 0; i < kProfSlots; ++i) pf[i] = 0ull;
        pf_t = global_ns();
    }
    auto mark = [&](int slot) {
        if (prof_on && threadIdx.x == 0) {
            unsigned long long t = global_ns();
            pf[slot] += t - pf_t;
            pf_t = t;
        }
    };

    // Partial sums of one tile.  FP32: one entry per (tile, warp), written by
    // lane 0 after a warp reduction.  FP64 (long GMRES(50) cycles): the warps of
    // a tile are first combined in shared memory, one entry per tile, so the
    // leader reads 8x fewer values.  Both orders are fixed.
    __shared__ double red[2][kWarps][kSlots];
    int red_buf = 0;
    auto put = [&](int tile, int slot, double v) {
        if constexpr (kWarpParts<T>) {
            if (lane == 0) I.part[(size_t)(tile * kWarps + warp) * ps + slot] = v;
        } else {
            if (lane == 0) red[red_buf][warp][slot] = v;
        }
    };
    auto tile_done = [&](int tile, int nslot) {
        if constexpr (!kWarpParts<T>) {
            csync<ST>();
            for (int t = threadIdx.x; t < nslot; t += kThreads) {
                double a = 0.0;
#pragma unroll
                for (int w = 0; w < kWarps; ++w) a += red[red_buf][w][t];
                I.part[(size_t)tile * ps + t] = a;
            }
            red_buf ^= 1;
        }
    };
    // After a CTA's tiles of a phase (FP64 with group sums): one fence, then
    // the CTA counts its tiles in at their groups; the CTA whose tile completes
    // a group sums that group's tiles in order.  Every tile of a group arrives
    // once per phase and the next phase's arrivals follow the team barrier, so
    // the completing CTA resets the counter.
    __shared__ int sh_glast[kMaxGroupWalk];
    __shared__ int sh_nlast;
    auto groups_done = [&](int nslot) {
        if constexpr (!kWarpParts<T>) {
            if (I.gpart == nullptr) return;
            for (int base = rank; base < I.n_tiles; base += kMaxGroupWalk * P) {
                csync<ST>();
                if (threadIdx.x == 0) {
                    __threadfence();
                    int nl = 0;
                    for (int q = 0; q < kMaxGroupWalk; ++q) {
                        const int tile = base + q * P;
                        if (tile >= I.n_tiles) break;
                        const int g = tile / kGroupTiles;
                        const int gsz = min(kGroupTiles, I.n_tiles - g * kGroupTiles);
                        if (atomicAdd(I.gcnt + g, 1u) == (unsigned int)(gsz - 1)) sh_glast[nl++] = g;
                    }
                    sh_nlast = nl;
                    __threadfence();
                }
                csync<ST>();
                for (int q = 0; q < sh_nlast; ++q) {
                    const int g = sh_glast[q];
                    const int t0 = g * kGroupTiles;
                    const int t1 = min(t0 + kGroupTiles, I.n_tiles);
                    for (int t = threadIdx.x; t < nslot; t += kThreads) {
                        double a = 0.0;
                        for (int u = t0; u < t1; ++u) a += __ldcg(I.part + (size_t)u * ps + t);
                        I.gpart[(size_t)g * ps + t] = a;
                    }
                    if (threadIdx.x == 0) I.gcnt[g] = 0u;
                }
            }
        }
    };
    auto voxel = [&](int tile, int v) -> long long { return (long long)tile * TILE + v * kThreads + threadIdx.x; };

    // ---- consumer side of the staging ring (ST)
    Stager<RING, TILE, T> stg{rh, ring, 0, 0, 0, 0, 0, 0u};
    // row coefficients of local voxel li from a stage (cw + m6, or coef)
    auto stage_coef = [&](const unsigned char* sb, int o_c, int o_m, int li, T (&c)[6]) {
        if (o_m >= 0) {
            const T w = reinterpret_cast<const T*>(sb + o_c)[li];
            const unsigned mk = sb[o_m + li];
#pragma unroll
            for (int k = 0; k < 6; ++k) c[k] = ((mk >> k) & 1u) ? w : T(0);
        } else {
            const T* cf = reinterpret_cast<const T*>(sb + o_c) + 6 * li;
#pragma unroll
            for (int k = 0; k < 6; ++k) c[k] = cf[k];
        }
    };
    // neighbour indices of voxel n (local li) from a stage's compact table, or
    // the int32 table in global memory when the instance has none
    auto stage_nb = [&](const unsigned char* sb, int o_nb, int li, long long n, int32_t (&q)[6]) {
        if (o_nb >= 0)
            decode_nb(reinterpret_cast<const short4*>(sb + o_nb)[li], __ldg(reinterpret_cast<const int4*>(I.nbase) + (n >> 9)),
                      n, q);
        else
            load_nb(I.nb, n, q);
    };
    // neighbour indices of row n (unstaged loops)
    auto row_nb = [&](long long n, int32_t (&q)[6]) {
        if constexpr (NBC) {
            decode_nb(__ldg(reinterpret_cast<const short4*>(I.nbr) + n), __ldg(reinterpret_cast<const int4*>(I.nbase) + (n >> 9)),
                      n, q);
        } else {
            load_nb(I.nb, n, q);
        }
    };

    // Prefetch into L2 the slice of an array (elem bytes per voxel) that `tile`
    // will read, so that the loads of the CTA's next tile find it there.  Start
    // and end are rounded down to 16 bytes: every prefetched byte lies inside
    // the array (whose allocation starts 256-byte aligned).
    auto pf_slice = [&](const void* arr, int elem, int tile) {
        if (arr == nullptr || tile >= I.n_tiles) return;
        const long long v0 = (long long)tile * TILE;
        const long long v1 = (v0 + TILE < N) ? v0 + TILE : N;
        uintptr_t a = reinterpret_cast<uintptr_t>(arr) + (uintptr_t)(v0 * elem);
        uintptr_t b = reinterpret_cast<uintptr_t>(arr) + (uintptr_t)(v1 * elem);
        a &= ~(uintptr_t)15;
        b &= ~(uintptr_t)15;
        if (b > a) prefetch_l2(reinterpret_cast<const void*>(a), (unsigned int)(b - a));
    };
    // the row tables of the operator (neighbours, coefficients, flags, edges)
    auto pf_rows = [&](int t, int tile) {
        switch (t) {
            case 0: if (NBC) pf_slice(I.nbr, 8, tile); else pf_slice(I.nb, 24, tile); break;
            case 1: pf_slice(I.cw ? (const void*)I.cw : (const void*)I.coef, I.cw ? (int)sizeof(T) : 6 * (int)sizeof(T), tile); break;
            case 2: pf_slice(I.m6, 1, tile); break;
            case 3: pf_slice(I.vflags, 1, tile); break;
            case 4: if (EDGE) pf_slice(I.enb, 48, tile); break;
            case 5: if (EDGE) pf_slice(I.ecf, 6 * (int)sizeof(T), tile); break;
            default: break;
        }
    };
    constexpr int kRowArrays = 6;

    auto params_of = [&](long long n, T* p) {
        if (I.vparams) {
            T raw[5];
#pragma unroll
            for (int q = 0; q < 5; ++q) raw[q] = I.vparams[5 * n + q];
            model_form<T>(I.model, raw, p);
        } else {
#pragma unroll
            for (int q = 0; q < 5; ++q) p[q] = I.params[q];
        }
    };

    // ---- leader bodies ------------------------------------------------------
    // Deterministic sums of partial slots slot0 .. slot0+ns-1 over all partials,
    // by the whole leader CTA; results in bsum_out[0..ns).  The order depends
    // only on the partial count, not on the team size.
    //  FP32 (a partial per tile and warp: many partials, few slots): thread t
    //  adds partials t, t+256, ... in order, four slots per pass with their loads
    //  issued together, then a fixed xor tree per warp.
    //  FP64 (a partial per group of tiles: few partials, up to 51 slots in a
    //  GMRES(50) cycle): lane l of warp w adds slot l (and l + 32) over partials
    //  w, w+8, ... in order, its loads issued together, so one pass of loads
    //  serves every slot.
    //  Both end with the warp results added in warp order.
    __shared__ double bsum_w[kMaxRestart + 1][kWarps];
    __shared__ double bsum_out[kMaxRestart + 1];
    constexpr int kSumW = 4;
    auto block_sum = [&](int slot0, int ns) {
        if constexpr (kWarpParts<T>) {
            for (int s0 = 0; s0 < ns; s0 += kSumW) {
                double a[kSumW];
#pragma unroll
                for (int u = 0; u < kSumW; ++u) a[u] = 0.0;
#pragma unroll 4
                for (int q = threadIdx.x; q < nparts; q += kThreads) {
                    const double* pq = psum + (size_t)q * ps + slot0 + s0;
#pragma unroll
                    for (int u = 0; u < kSumW; ++u)
                        if (s0 + u < ns) a[u] += __ldcg(pq + u);
                }
#pragma unroll
                for (int u = 0; u < kSumW; ++u) {
                    const double v = warp_sum(a[u]);
                    if (lane == 0 && s0 + u < ns) bsum_w[s0 + u][warp] = v;
                }
            }
        } else {
            for (int s0 = 0; s0 < ns; s0 += 32) {
                const int sl = s0 + lane;
                if (sl < ns) {
                    const double* pq = psum + slot0 + sl;
                    double a = 0.0;
#pragma unroll 8
                    for (int q = warp; q < nparts; q += kWarps) a += __ldcg(pq + (size_t)q * ps);
                    bsum_w[sl][warp] = a;
                }
            }
        }
        csync<ST>();
        for (int i = threadIdx.x; i < ns; i += kThreads) {
            double t = 0.0;
#pragma unroll
            for (int w = 0; w < kWarps; ++w) t += bsum_w[i][w];
            bsum_out[i] = t;
        }
        csync<ST>();
    };

    // statistics of a solve that iterated, recorded by the leader that ends it
    auto account_solve = [&]() {
        const int it = sc->iters_solve;
        if (it > 0) {
            I.st->arnoldi += it;
            I.st->arnoldi_sq += (long long)it * it;
            I.st->solves += 1;
            if (it > I.st->max_arnoldi) I.st->max_arnoldi = it;
        }
    };

    auto leader_rhs = [&]() {
        block_sum(0, 2);
        if (warp == 0) {
            double b2 = bsum_out[0];
            double r2 = bsum_out[1];
            if (lane == 0) {
                double bn = sqrt(b2), rn = sqrt(r2);
                double atol_eff = fmax(I.atol, I.tol * bn);
                int act;
                if (!isfinite(bn) || !isfinite(rn)) act = ACT_FAIL;
                else if (bn == 0.0) act = ACT_ZERO_B;
                else if (rn <= atol_eff) act = ACT_DONE;
                else {
                    act = ACT_CYCLE;
                    sc->g[0] = rn;
                    sc->s[0] = 1.0 / rn;
                    sc->iters_solve = 0;
                    sc->iters_cap = 0;
                }
                sc->bnorm = bn;
                sc->rnorm = rn;
                sc->atol_eff = atol_eff;
                sc->action = act;
                if (act == ACT_FAIL) I.st->status = PHS_ERR_NONFINITE;
            }
        }
    };

    auto leader_dots = [&](int j) {
        // h_ij = s_i * sum <V_i, w>;  published coef_i = h_ij * s_i
        block_sum(0, j + 1);
        for (int i = threadIdx.x; i <= j; i += kThreads) {
            double si = sc->s[i];
            double h = si * bsum_out[i];
            sc->R[j * (kMaxRestart + 1) + i] = h;
            sc->coef[i] = h * si;
        }
    };

    // Givens update of Hessenberg column j and, when the cycle ends, the back
    // substitution R y = g.  The rotations, the column, g, s and (at a cycle
    // end) the k x k triangle of R are first loaded into shared memory by the
    // whole CTA, so the sequential parts run on shared memory instead of a
    // chain of dependent L2 round trips; the arithmetic and its order are
    // those of a plain sequential Givens QR.
    __shared__ double gv_cs[kMaxRestart], gv_sn[kMaxRestart], gv_col[kMaxRestart + 2];
    __shared__ double gv_g[kMaxRestart + 1], gv_s[kMaxRestart + 1], gv_y[kMaxRestart + 1];
    __shared__ double gv_R[kMaxRestart * (kMaxRestart + 1) / 2];   // column l, rows 0..l at l(l+1)/2 + i
    __shared__ int gv_act;
    auto leader_norm = [&](int j) {
        block_sum(0, 1);
        double* Rc = sc->R + j * (kMaxRestart + 1);
        for (int i = threadIdx.x; i < j; i += kThreads) {
            gv_cs[i] = __ldcg(sc->cs + i);
            gv_sn[i] = __ldcg(sc->sn + i);
        }
        for (int i = threadIdx.x; i <= j; i += kThreads) {
            gv_col[i] = __ldcg(Rc + i);
            gv_g[i] = __ldcg(sc->g + i);
            gv_s[i] = __ldcg(sc->s + i);
        }
        csync<ST>();
        if (threadIdx.x == 0) {
            const double hn = sqrt(bsum_out[0]);
            gv_col[j + 1] = hn;
            // apply the previous rotations to column j
            for (int i = 0; i < j; ++i) {
                const double c = gv_cs[i], s = gv_sn[i];
                const double a = gv_col[i], bb = gv_col[i + 1];
                gv_col[i] = c * a + s * bb;
                gv_col[i + 1] = -s * a + c * bb;
            }
            const double a = gv_col[j], bb = gv_col[j + 1];
            const double r = hypot(a, bb);
            const double c = (r == 0.0) ? 1.0 : a / r;
            const double s = (r == 0.0) ? 0.0 : bb / r;
            sc->cs[j] = c;
            sc->sn[j] = s;
            gv_col[j] = r;
            gv_col[j + 1] = 0.0;
            const double gj = gv_g[j];
            gv_g[j] = c * gj;
            gv_g[j + 1] = -s * gj;
            sc->g[j] = gv_g[j];
            sc->g[j + 1] = gv_g[j + 1];
            const double est = fabs(gv_g[j + 1]);
            sc->est = est;
            sc->iters_solve += 1;
            int act;
            const bool finite = isfinite(hn) && isfinite(r);
            const bool breakdown = (hn == 0.0);
            const bool conv = (!I.full_cycles) && (est <= sc->atol_eff);
            if (!finite) {
                act = ACT_FAIL;
                I.st->status = PHS_ERR_NONFINITE;
            } else if (conv || (breakdown && !I.full_cycles)) {
                act = ACT_UPDATE_FINAL;
            } else if (j + 1 >= I.m || breakdown) {
                act = ACT_UPDATE_CHECK;
            } else {
                act = ACT_NEXT_J;
                sc->s[j + 1] = 1.0 / hn;
            }
            if (act == ACT_UPDATE_FINAL || act == ACT_UPDATE_CHECK) sc->k = j + 1;
            if (act == ACT_UPDATE_FINAL) account_solve();
            sc->action = act;
            gv_act = act;
        }
        csync<ST>();
        for (int i = threadIdx.x; i <= j + 1; i += kThreads) Rc[i] = gv_col[i];
        const int act = gv_act;
        if (act != ACT_UPDATE_FINAL && act != ACT_UPDATE_CHECK) return;
        // back substitution R y = g (k x k upper triangular), k = j + 1
        const int k = j + 1;
        for (int l = warp; l < k; l += kWarps)
            for (int i = lane; i <= l; i += 32)
                gv_R[l * (l + 1) / 2 + i] = (l == j) ? gv_col[i] : __ldcg(sc->R + l * (kMaxRestart + 1) + i);
        csync<ST>();
        if (warp == 0) {
            for (int i = k - 1; i >= 0; --i) {
                double acc = 0.0;
                for (int l = i + 1 + lane; l < k; l += 32) acc += gv_R[l * (l + 1) / 2 + i] * gv_y[l];
                acc = warp_sum(acc);
                if (lane == 0) gv_y[i] = (gv_g[i] - acc) / gv_R[i * (i + 1) / 2 + i];
                __syncwarp();
            }
            // scale: x += sum_j y_j v_j = sum_j (y_j s_j) V_j
            for (int i = lane; i < k; i += 32) sc->coef[i] = gv_y[i] * gv_s[i];
        }
    };

    auto leader_check = [&]() {
        block_sum(0, 1);
        if (warp == 0) {
            double r2 = bsum_out[0];
            if (lane == 0) {
                double rn = sqrt(r2);
                sc->rnorm = rn;
                sc->iters_cap += I.m;
                int act;
                if (!isfinite(rn)) {
                    act = ACT_FAIL;
                    I.st->status = PHS_ERR_NONFINITE;
                } else if (rn <= sc->atol_eff) {
                    act = ACT_DONE;
                    account_solve();
                } else if (sc->iters_cap >= I.maxiter) {
                    act = ACT_DONE;
                    account_solve();
                    I.st->nonconv += 1;
                    if (I.st->status == PHS_OK) I.st->status = PHS_WARN_NO_CONVERGE;
                } else {
                    act = ACT_CYCLE;
                    sc->g[0] = rn;
                    sc->s[0] = 1.0 / rn;
                }
                sc->action = act;
            }
        }
    };


    // the action and cycle length of the barrier that just ended (team_sync)
    auto read_action = [&]() { return ctl.action; };

    auto load_shc = [&](int cnt) {
        csync<ST>();
        for (int i = threadIdx.x; i < cnt; i += kThreads) shc[i] = __ldcg(sc->coef + i);
        csync<ST>();
    };

    // ---- sample / activation bookkeeping of the state in u (after step s-1)
    auto sample_voxel = [&](long long n, T un, T hn, long long done_step) {
        if (pending >= 0) {
            I.hist_u[(size_t)pending * N + n] = un;
            if (I.save_h) I.hist_h[(size_t)pending * N + n] = hn;
        }
        if (done_step >= 0 && un >= T(0.5) && I.lat[n] < 0) I.lat[n] = (int32_t)done_step;
    };

    T* Vb = I.V;
    const size_t ldV = (size_t)I.ldv;

    // End-of-step work of voxel n whose new state un is known (the state after
    // step done_step): its sample into history slot `slot` (-1: none), its
    // activation entry (lat_n loaded when un >= 0.5), then the RK4 reaction of
    // the next step (stimulus bits stim_next) -> h of the step after it into
    // hdst, u* into the basis column 1.  This is the reaction pass of the next
    // step, done while the voxel's new state is still in registers.
    auto react_voxel = [&](long long n, T un, T hn, int32_t lat_n, long long done_step, int slot, uint8_t fl,
                           uint8_t stim_next, T* hdst) {
        if (slot >= 0) {
            I.hist_u[(size_t)slot * N + n] = un;
            if (I.save_h) I.hist_h[(size_t)slot * N + n] = hn;
        }
        if (done_step >= 0 && un >= T(0.5) && lat_n < 0) I.lat[n] = (int32_t)done_step;
        T p[5];
        params_of(n, p);
        const T J = (fl & stim_next & 3u) ? I.jmag : T(0);
        T us, hs;
        rk4(I.model, un, hn, J, p, I.dt, us, hs);
        hdst[n] = hs;
        Vb[ldV + n] = us;
    };

    // acc[v] += sum_{i < cnt} coef[i] * Vb[i][n_v], loads issued kChunk vectors at a time
    auto axpy_basis = [&](int tile, int cnt, const double* coef, double (&acc)[VPT]) {
        for (int i0 = 0; i0 < cnt; i0 += kChunk) {
            T vv[kChunk][VPT];
#pragma unroll
            for (int ii = 0; ii < kChunk; ++ii)
#pragma unroll
                for (int v = 0; v < VPT; ++v) {
                    long long n = voxel(tile, v);
                    vv[ii][v] = (i0 + ii < cnt && n < N) ? Vb[(size_t)(i0 + ii) * ldV + n] : T(0);
                }
#pragma unroll
            for (int ii = 0; ii < kChunk; ++ii) {
                if (i0 + ii < cnt) {
                    const double cf = coef[i0 + ii];
#pragma unroll
                    for (int v = 0; v < VPT; ++v) acc[v] += cf * (double)vv[ii][v];
                }
            }
        }
    };

    // the reaction pass of the current step was done at the end of the previous
    // one (by the same threads, for the same voxels)
    bool prepared = false;
    for (; step < step_end && !retired && !aborted; ++step) {
        const uint8_t stim_bits = __ldg(I.stim + step);
        const bool tb = step < I.tb_steps;
        T* hin = hbuf ? I.h1 : I.h0;
        T* hout = hbuf ? I.h0 : I.h1;

        // ================= RHS phase.  Pass 1: RK4 reaction of every voxel of the
        // team; u* goes to basis column 1 (unused until the first Arnoldi step).
        // Except in the first step of a launch and after a full-cycle solve, it
        // ran at the end of the previous step (react_voxel in the update and copy
        // passes), so it costs no pass of its own.
        // Pass 2, after a team barrier: b = u* + dt/2 L u*, the initial guess and
        // r0 = b - A x0 -> V0, gathering u* of the neighbours from memory.  (A
        // fused form that kept a tile's u* in shared memory and recomputed the RK4
        // of neighbours outside the tile did three RK4 per voxel in row order and
        // was 17 % slower over the batch.)
        T* Us = Vb + ldV;
        for (int tile = prepared ? I.n_tiles : rank; tile < I.n_tiles; tile += P) {
            if (threadIdx.x < 4) {
                const int t = threadIdx.x;
                if (t == 0) pf_slice(I.u, sizeof(T), tile + P);
                else if (t == 1) pf_slice(hin, sizeof(T), tile + P);
                else if (t == 2) pf_slice(I.vflags, 1, tile + P);
                else pf_slice(I.vparams, 5 * sizeof(T), tile + P);
            }
            // every load of the tile before its first store: plain loads cannot
            // move across stores the compiler must assume may alias them
            T un[VPT], hn[VPT];
            uint8_t fl[VPT];
            int32_t lt[VPT];
#pragma unroll
            for (int v = 0; v < VPT; ++v) {
                const long long n = voxel(tile, v);
                un[v] = T(0);
                hn[v] = T(0);
                fl[v] = 0;
                lt[v] = 0;
                if (n < N) {
                    un[v] = I.u[n];
                    hn[v] = hin[n];
                    fl[v] = __ldg(I.vflags + n);
                }
            }
#pragma unroll
            for (int v = 0; v < VPT; ++v) {
                const long long n = voxel(tile, v);
                if (n < N && step > 0 && un[v] >= T(0.5)) lt[v] = I.lat[n];
            }
#pragma unroll
            for (int v = 0; v < VPT; ++v) {
                const long long n = voxel(tile, v);
                if (n < N) react_voxel(n, un[v], hn[v], lt[v], step - 1, pending, fl[v], stim_bits, hout);
            }
        }
        pending = -1;
        mark(PF_RHS1);
        if (!team_sync<ST>(I.sync, P, abort_word, ctl, sc, I.prof, [&]() {})) { aborted = true; break; }
        mark(PF_RHS_WAIT);
        int nst = 0;
        if constexpr (ST) {
            stg.begin();
            const int o_us = stg.add(Us, sizeof(T));
            const int o_nb = I.nbr ? stg.add(I.nbr, 8) : -1;
            const int o_cw = I.cw ? stg.add(I.cw, sizeof(T)) : stg.add(I.coef, 6 * sizeof(T));
            const int o_m6 = I.cw ? stg.add(I.m6, 1) : -1;
            const int o_dx = I.dx ? stg.add(I.dx, sizeof(T)) : -1;
            const int o_fl = tb ? stg.add(I.vflags, 1) : -1;
            nst = stg.publish(rank, P, I.n_tiles);
            for (int tile = rank; nst > 0 && tile < I.n_tiles; tile += P) {
                const unsigned char* sb = stg.acquire(abort_word);
                double ab = 0.0, ar = 0.0;
#pragma unroll
                for (int v = 0; v < VPT; ++v) {
                    const int li = v * kThreads + threadIdx.x;
                    const long long n = (long long)tile * TILE + li;
                    if (n < N) {
                        const T us = reinterpret_cast<const T*>(sb + o_us)[li];
                        const bool rz = tb && (sb[o_fl + li] & PHS_VFLAG_TBLOCK);
                        int32_t q[6];
                        T c[6];
                        stage_nb(sb, o_nb, li, n, q);
                        stage_coef(sb, o_cw, o_m6, li, c);
                        T lap = T(0), dp = T(0), lapd = T(0);
                        if (!rz) {
                            lap = lap_row(Us, us, q, c);
                            if (EDGE && I.ecf) lap += edge_row(Us, I.enb, I.ecf, n);
                        }
                        if (o_dx >= 0) {
                            dp = reinterpret_cast<const T*>(sb + o_dx)[li];
                            if (!rz) {
                                lapd = lap_row(I.dx, dp, q, c);
                                if (EDGE && I.ecf) lapd += edge_row(I.dx, I.enb, I.ecf, n);
                            }
                        }
                        const T x0 = us + dp;
                        const T bn = us + I.half_dt * lap;
                        const T ax = x0 - I.half_dt * (lap + lapd);
                        const T rn = bn - ax;
                        I.x[n] = x0;
                        I.b[n] = bn;
                        Vb[n] = rn;
                        ab += (double)bn * (double)bn;
                        ar += (double)rn * (double)rn;
                    }
                }
                stg.release();
                ab = warp_sum(ab);
                ar = warp_sum(ar);
                put(tile, 0, ab);
                put(tile, 1, ar);
                tile_done(tile, 2);
            }
        }
        for (int tile = rank; nst == 0 && tile < I.n_tiles; tile += P) {
            if (threadIdx.x < kRowArrays) pf_rows(threadIdx.x, tile + P);
            else if (threadIdx.x == kRowArrays) pf_slice(Us, sizeof(T), tile + P);
            else if (threadIdx.x == kRowArrays + 1) pf_slice(I.dx, sizeof(T), tile + P);
            double ab = 0.0, ar = 0.0;
#pragma unroll
            for (int v = 0; v < VPT; ++v) {
                const long long n = voxel(tile, v);
                if (n < N) {
                    const T us = __ldcg(Us + n);
                    const bool rz = tb && (__ldg(I.vflags + n) & PHS_VFLAG_TBLOCK);
                    int32_t q[6];
                    T c[6];
                    row_nb(n, q);
                    row_coef(I.coef, I.cw, I.m6, n, c);
                    T lap = T(0), dp = T(0), lapd = T(0);
                    if (!rz) {
                        lap = lap_row(Us, us, q, c);
                        if (EDGE && I.ecf) lap += edge_row(Us, I.enb, I.ecf, n);
                    }
                    // initial guess: u* (the reference's x0), or u* plus the previous
                    // step's diffusion increment when dx is kept
                    if (I.dx) {
                        dp = I.dx[n];
                        if (!rz) {
                            lapd = lap_row(I.dx, dp, q, c);
                            if (EDGE && I.ecf) lapd += edge_row(I.dx, I.enb, I.ecf, n);
                        }
                    }
                    const T x0 = us + dp;
                    const T bn = us + I.half_dt * lap;
                    const T ax = x0 - I.half_dt * (lap + lapd);
                    const T rn = bn - ax;
                    I.x[n] = x0;
                    I.b[n] = bn;
                    Vb[n] = rn;
                    ab += (double)bn * (double)bn;
                    ar += (double)rn * (double)rn;
                }
            }
            ab = warp_sum(ab);
            ar = warp_sum(ar);
            put(tile, 0, ab);
            put(tile, 1, ar);
            tile_done(tile, 2);
        }
        groups_done(2);
        mark(PF_RHS);
        if (!team_sync<ST>(I.sync, P, abort_word, ctl, sc, I.prof, leader_rhs)) { aborted = true; break; }
        int act = read_action();
        mark(PF_RHS_WAIT);
        // end of this step: its history slot, and whether the pass that writes
        // the new state also runs the next step's reaction (not after the last
        // step of the launch)
        const bool due_now = (I.stride > 0) ? (step % I.stride == 0) : true;
        const int slot_now = (due_now && id_save < I.n_samples) ? id_save : -1;
        const bool fuse_next = step + 1 < step_end;
        const uint8_t stim_next = fuse_next ? __ldg(I.stim + step + 1) : (uint8_t)0;
        bool fused = false;

        if (act == ACT_CYCLE) {
            bool leave_solve = false;
            while (!leave_solve) {
                int j = 0;
                for (;;) {
                    // ============ phase A: w = A (s_j V_j) -> V_{j+1}; dots <V_i, w>
                    if (threadIdx.x == 0) ctl.sj = __ldcg(&sc->s[j]);
                    csync<ST>();
                    const T sj = (T)ctl.sj;
                    const T* Vj = Vb + (size_t)j * ldV;
                    T* Vn = Vb + (size_t)(j + 1) * ldV;
                    int nsa = 0;
                    if constexpr (ST) {
                        stg.begin();
                        const int o_vj = stg.add(Vj, sizeof(T));
                        const int o_nb = I.nbr ? stg.add(I.nbr, 8) : -1;
                        const int o_cw = I.cw ? stg.add(I.cw, sizeof(T)) : stg.add(I.coef, 6 * sizeof(T));
                        const int o_m6 = I.cw ? stg.add(I.m6, 1) : -1;
                        const int o_fl = tb ? stg.add(I.vflags, 1) : -1;
                        const int nvs = min(j, stg.vec_cap());      // V_0 .. V_{nvs-1} staged too
                        const int o_v = stg.lay_off;
                        for (int i = 0; i < nvs; ++i) stg.add(Vb + (size_t)i * ldV, sizeof(T));
                        nsa = stg.publish(rank, P, I.n_tiles);
                        for (int tile = rank; nsa > 0 && tile < I.n_tiles; tile += P) {
                            const unsigned char* sb = stg.acquire(abort_word);
                            const T* vjs = reinterpret_cast<const T*>(sb + o_vj);
                            T wr[VPT];
#pragma unroll
                            for (int v = 0; v < VPT; ++v) {
                                const int li = v * kThreads + threadIdx.x;
                                const long long n = (long long)tile * TILE + li;
                                wr[v] = T(0);
                                if (n < N) {
                                    const T vj = vjs[li];
                                    const bool rz = tb && (sb[o_fl + li] & PHS_VFLAG_TBLOCK);
                                    int32_t q[6];
                                    T c[6];
                                    stage_nb(sb, o_nb, li, n, q);
                                    stage_coef(sb, o_cw, o_m6, li, c);
                                    T lap = rz ? T(0) : lap_row(Vj, vj, q, c);
                                    if (EDGE && I.ecf && !rz) lap += edge_row(Vj, I.enb, I.ecf, n);
                                    const T w = sj * (vj - I.half_dt * lap);
                                    Vn[n] = w;
                                    wr[v] = w;
                                }
                            }
                            for (int i0 = 0; i0 <= j; i0 += kChunk) {
                                T vv[kChunk][VPT];
#pragma unroll
                                for (int ii = 0; ii < kChunk; ++ii)
#pragma unroll
                                    for (int v = 0; v < VPT; ++v) {
                                        const int li = v * kThreads + threadIdx.x;
                                        const long long n = (long long)tile * TILE + li;
                                        const int i = i0 + ii;
                                        T val = T(0);
                                        if (i <= j && n < N)
                                            val = (i == j) ? vjs[li]
                                                  : (i < nvs) ? reinterpret_cast<const T*>(sb + o_v + i * TILE * (int)sizeof(T))[li]
                                                              : Vb[(size_t)i * ldV + n];
                                        vv[ii][v] = val;
                                    }
#pragma unroll
                                for (int ii = 0; ii < kChunk; ++ii) {
                                    double d = 0.0;
#pragma unroll
                                    for (int v = 0; v < VPT; ++v) d += (double)vv[ii][v] * (double)wr[v];
                                    if (i0 + ii <= j) {          // uniform over the warp
                                        d = warp_sum(d);
                                        put(tile, i0 + ii, d);
                                    }
                                }
                            }
                            stg.release();
                            tile_done(tile, j + 1);
                        }
                    }
                    for (int tile = rank; nsa == 0 && tile < I.n_tiles; tile += P) {
                        if (threadIdx.x < kRowArrays) pf_rows(threadIdx.x, tile + P);
                        else if (threadIdx.x <= kRowArrays + j)
                            pf_slice(Vb + (size_t)(threadIdx.x - kRowArrays) * ldV, sizeof(T), tile + P);
                        T wr[VPT];
#pragma unroll
                        for (int v = 0; v < VPT; ++v) {
                            const long long n = voxel(tile, v);
                            wr[v] = T(0);
                            if (n < N) {
                                const T vj = Vj[n];
                                const bool rz = tb && (__ldg(I.vflags + n) & PHS_VFLAG_TBLOCK);
                                int32_t q[6];
                                T c[6];
                                row_nb(n, q);
                                row_coef(I.coef, I.cw, I.m6, n, c);
                                T lap = rz ? T(0) : lap_row(Vj, vj, q, c);
                                if (EDGE && I.ecf && !rz) lap += edge_row(Vj, I.enb, I.ecf, n);
                                const T w = sj * (vj - I.half_dt * lap);
                                Vn[n] = w;
                                wr[v] = w;
                            }
                        }
                        for (int i0 = 0; i0 <= j; i0 += kChunk) {
                            T vv[kChunk][VPT];
#pragma unroll
                            for (int ii = 0; ii < kChunk; ++ii)
#pragma unroll
                                for (int v = 0; v < VPT; ++v) {
                                    const long long n = voxel(tile, v);
                                    vv[ii][v] = (i0 + ii <= j && n < N) ? Vb[(size_t)(i0 + ii) * ldV + n] : T(0);
                                }
#pragma unroll
                            for (int ii = 0; ii < kChunk; ++ii) {
                                double d = 0.0;
#pragma unroll
                                for (int v = 0; v < VPT; ++v) d += (double)vv[ii][v] * (double)wr[v];
                                if (i0 + ii <= j) {          // uniform over the warp
                                    d = warp_sum(d);
                                    put(tile, i0 + ii, d);
                                }
                            }
                        }
                        tile_done(tile, j + 1);
                    }
                    groups_done(j + 1);
                    mark(PF_A);
                    if (!team_sync<ST>(I.sync, P, abort_word, ctl, sc, I.prof, [&]() { leader_dots(j); })) { aborted = true; break; }
                    load_shc(j + 1);
                    mark(PF_A_WAIT);
                    // ============ phase C: u = w - sum_i c_i V_i  (in place), ||u||^2
                    int nsc = 0;
                    if constexpr (ST) {
                        stg.begin();
                        const int o_w = stg.add(Vn, sizeof(T));
                        const int nvs = min(j + 1, stg.vec_cap());
                        const int o_v = stg.lay_off;
                        for (int i = 0; i < nvs; ++i) stg.add(Vb + (size_t)i * ldV, sizeof(T));
                        nsc = stg.publish(rank, P, I.n_tiles);
                        for (int tile = rank; nsc > 0 && tile < I.n_tiles; tile += P) {
                            const unsigned char* sb = stg.acquire(abort_word);
                            double acc[VPT];
#pragma unroll
                            for (int v = 0; v < VPT; ++v) {
                                const int li = v * kThreads + threadIdx.x;
                                const long long n = (long long)tile * TILE + li;
                                acc[v] = (n < N) ? (double)reinterpret_cast<const T*>(sb + o_w)[li] : 0.0;
                            }
                            for (int i0 = 0; i0 <= j; i0 += kChunk) {
                                T vv[kChunk][VPT];
#pragma unroll
                                for (int ii = 0; ii < kChunk; ++ii)
#pragma unroll
                                    for (int v = 0; v < VPT; ++v) {
                                        const int li = v * kThreads + threadIdx.x;
                                        const long long n = (long long)tile * TILE + li;
                                        const int i = i0 + ii;
                                        T val = T(0);
                                        if (i <= j && n < N)
                                            val = (i < nvs) ? reinterpret_cast<const T*>(sb + o_v + i * TILE * (int)sizeof(T))[li]
                                                            : Vb[(size_t)i * ldV + n];
                                        vv[ii][v] = val;
                                    }
#pragma unroll
                                for (int ii = 0; ii < kChunk; ++ii) {
                                    if (i0 + ii <= j) {
                                        const double cf = shc[i0 + ii];
#pragma unroll
                                        for (int v = 0; v < VPT; ++v) acc[v] -= cf * (double)vv[ii][v];
                                    }
                                }
                            }
                            stg.release();
                            double a2 = 0.0;
#pragma unroll
                            for (int v = 0; v < VPT; ++v) {
                                const long long n = voxel(tile, v);
                                if (n < N) {
                                    const T ut = (T)acc[v];
                                    Vn[n] = ut;
                                    a2 += (double)ut * (double)ut;
                                }
                            }
                            a2 = warp_sum(a2);
                            put(tile, 0, a2);
                            tile_done(tile, 1);
                        }
                    }
                    for (int tile = rank; nsc == 0 && tile < I.n_tiles; tile += P) {
                        if (threadIdx.x <= j + 1) pf_slice(Vb + (size_t)threadIdx.x * ldV, sizeof(T), tile + P);
                        double acc[VPT];
#pragma unroll
                        for (int v = 0; v < VPT; ++v) {
                            const long long n = voxel(tile, v);
                            acc[v] = (n < N) ? (double)Vn[n] : 0.0;
                        }
                        // acc -= sum_i shc[i] V_i
                        for (int i0 = 0; i0 <= j; i0 += kChunk) {
                            T vv[kChunk][VPT];
#pragma unroll
                            for (int ii = 0; ii < kChunk; ++ii)
#pragma unroll
                                for (int v = 0; v < VPT; ++v) {
                                    const long long n = voxel(tile, v);
                                    vv[ii][v] = (i0 + ii <= j && n < N) ? Vb[(size_t)(i0 + ii) * ldV + n] : T(0);
                                }
#pragma unroll
                            for (int ii = 0; ii < kChunk; ++ii) {
                                if (i0 + ii <= j) {
                                    const double cf = shc[i0 + ii];
#pragma unroll
                                    for (int v = 0; v < VPT; ++v) acc[v] -= cf * (double)vv[ii][v];
                                }
                            }
                        }
                        double a2 = 0.0;
#pragma unroll
                        for (int v = 0; v < VPT; ++v) {
                            const long long n = voxel(tile, v);
                            if (n < N) {
                                const T ut = (T)acc[v];
                                Vn[n] = ut;
                                a2 += (double)ut * (double)ut;
                            }
                        }
                        a2 = warp_sum(a2);
                        put(tile, 0, a2);
                        tile_done(tile, 1);
                    }
                    groups_done(1);
                    mark(PF_C);
                    if (!team_sync<ST>(I.sync, P, abort_word, ctl, sc, I.prof, [&]() { leader_norm(j); })) { aborted = true; break; }
                    act = read_action();
                    mark(PF_C_WAIT);
                    if (prof_on && threadIdx.x == 0) pf[PF_SOLVE_ITERS] += 1;
                    if (act != ACT_NEXT_J) break;
                    ++j;
                }
                if (aborted) break;
                if (act == ACT_FAIL) { retired = true; break; }
                // ============ phase X: x += sum_j c_j V_j
                const int k = ctl.k;
                load_shc(k);
                const bool final = (act == ACT_UPDATE_FINAL);
                const bool react = final && fuse_next;
                int nsx = 0;
                if constexpr (ST) {
                    stg.begin();
                    const int o_x = stg.add(I.x, sizeof(T));
                    const int o_dx = (final && I.dx) ? stg.add(I.dx, sizeof(T)) : -1;
                    const int o_h = react ? stg.add(hout, sizeof(T)) : -1;
                    const int o_fl = react ? stg.add(I.vflags, 1) : -1;
                    const int nvs = min(k, stg.vec_cap());
                    const int o_v = stg.lay_off;
                    for (int i = 0; i < nvs; ++i) stg.add(Vb + (size_t)i * ldV, sizeof(T));
                    nsx = stg.publish(rank, P, I.n_tiles);
                    for (int tile = rank; nsx > 0 && tile < I.n_tiles; tile += P) {
                        const unsigned char* sb = stg.acquire(abort_word);
                        const T* xs = reinterpret_cast<const T*>(sb + o_x);
                        double acc[VPT];
#pragma unroll
                        for (int v = 0; v < VPT; ++v) {
                            const int li = v * kThreads + threadIdx.x;
                            acc[v] = ((long long)tile * TILE + li < N) ? (double)xs[li] : 0.0;
                        }
                        for (int i0 = 0; i0 < k; i0 += kChunk) {
                            T vv[kChunk][VPT];
#pragma unroll
                            for (int ii = 0; ii < kChunk; ++ii)
#pragma unroll
                                for (int v = 0; v < VPT; ++v) {
                                    const int li = v * kThreads + threadIdx.x;
                                    const long long n = (long long)tile * TILE + li;
                                    const int i = i0 + ii;
                                    T val = T(0);
                                    if (i < k && n < N)
                                        val = (i < nvs) ? reinterpret_cast<const T*>(sb + o_v + i * TILE * (int)sizeof(T))[li]
                                                        : Vb[(size_t)i * ldV + n];
                                    vv[ii][v] = val;
                                }
#pragma unroll
                            for (int ii = 0; ii < kChunk; ++ii) {
                                if (i0 + ii < k) {
                                    const double cf = shc[i0 + ii];
#pragma unroll
                                    for (int v = 0; v < VPT; ++v) acc[v] += cf * (double)vv[ii][v];
                                }
                            }
                        }
#pragma unroll
                        for (int v = 0; v < VPT; ++v) {
                            const int li = v * kThreads + threadIdx.x;
                            const long long n = (long long)tile * TILE + li;
                            if (n < N) {
                                if (final) {
                                    I.u[n] = (T)acc[v];
                                    if (o_dx >= 0) {
                                        const double dxo = (double)reinterpret_cast<const T*>(sb + o_dx)[li];
                                        I.dx[n] = (T)(dxo + (acc[v] - (double)xs[li]));
                                    }
                                } else {
                                    I.x[n] = (T)acc[v];
                                }
                            }
                        }
                        if (react) {
                            int32_t lt[VPT];
#pragma unroll
                            for (int v = 0; v < VPT; ++v) {
                                const long long n = voxel(tile, v);
                                lt[v] = (n < N && (T)acc[v] >= T(0.5)) ? I.lat[n] : 0;
                            }
#pragma unroll
                            for (int v = 0; v < VPT; ++v) {
                                const int li = v * kThreads + threadIdx.x;
                                const long long n = (long long)tile * TILE + li;
                                if (n < N)
                                    react_voxel(n, (T)acc[v], reinterpret_cast<const T*>(sb + o_h)[li], lt[v], step, slot_now,
                                                sb[o_fl + li], stim_next, hin);
                            }
                        }
                        stg.release();
                    }
                }
                for (int tile = rank; nsx == 0 && tile < I.n_tiles; tile += P) {
                    if (threadIdx.x < k) pf_slice(Vb + (size_t)threadIdx.x * ldV, sizeof(T), tile + P);
                    else if (threadIdx.x == k) pf_slice(I.x, sizeof(T), tile + P);
                    else if (threadIdx.x == k + 1 && final) pf_slice(I.dx, sizeof(T), tile + P);
                    else if (threadIdx.x == k + 2 && react) pf_slice(hout, sizeof(T), tile + P);
                    else if (threadIdx.x == k + 3 && react) pf_slice(I.vflags, 1, tile + P);
                    double acc[VPT], x_in[VPT];
                    T hn[VPT];
                    uint8_t fl[VPT];
#pragma unroll
                    for (int v = 0; v < VPT; ++v) {
                        const long long n = voxel(tile, v);
                        acc[v] = (n < N) ? (double)I.x[n] : 0.0;
                        x_in[v] = acc[v];
                        hn[v] = (react && n < N) ? hout[n] : T(0);
                        fl[v] = (react && n < N) ? __ldg(I.vflags + n) : (uint8_t)0;
                    }
                    axpy_basis(tile, k, shc, acc);
#pragma unroll
                    for (int v = 0; v < VPT; ++v) {
                        const long long n = voxel(tile, v);
                        if (n < N) {
                            if (final) {
                                I.u[n] = (T)acc[v];
                                // increment u_next - u* for the next step's initial guess
                                if (I.dx) I.dx[n] = (T)((double)I.dx[n] + (acc[v] - x_in[v]));
                            } else {
                                I.x[n] = (T)acc[v];
                            }
                        }
                    }
                    if (react) {
                        int32_t lt[VPT];
#pragma unroll
                        for (int v = 0; v < VPT; ++v) {
                            const long long n = voxel(tile, v);
                            lt[v] = (n < N && (T)acc[v] >= T(0.5)) ? I.lat[n] : 0;
                        }
#pragma unroll
                        for (int v = 0; v < VPT; ++v) {
                            const long long n = voxel(tile, v);
                            if (n < N) react_voxel(n, (T)acc[v], hn[v], lt[v], step, slot_now, fl[v], stim_next, hin);
                        }
                    }
                }
                mark(PF_X);
                if (final) {
                    fused = react;
                    break;
                }
                // ============ true residual of the new iterate (start of the next cycle)
                if (!team_sync<ST>(I.sync, P, abort_word, ctl, sc, I.prof, [&]() {})) { aborted = true; break; }
                for (int tile = rank; tile < I.n_tiles; tile += P) {
                    if (threadIdx.x < kRowArrays) pf_rows(threadIdx.x, tile + P);
                    else if (threadIdx.x == kRowArrays) pf_slice(I.x, sizeof(T), tile + P);
                    else if (threadIdx.x == kRowArrays + 1) pf_slice(I.b, sizeof(T), tile + P);
                    double a2 = 0.0;
#pragma unroll
                    for (int v = 0; v < VPT; ++v) {
                        const long long n = voxel(tile, v);
                        if (n < N) {
                            const T xv = I.x[n];
                            const bool rz = tb && (__ldg(I.vflags + n) & PHS_VFLAG_TBLOCK);
                            int32_t q[6];
                            T c[6];
                            row_nb(n, q);
                            row_coef(I.coef, I.cw, I.m6, n, c);
                            T lap = rz ? T(0) : lap_row(I.x, xv, q, c);
                            if (EDGE && I.ecf && !rz) lap += edge_row(I.x, I.enb, I.ecf, n);
                            const T ax = xv - I.half_dt * lap;
                            const T r = I.b[n] - ax;
                            Vb[n] = r;
                            I.u[n] = xv;
                            a2 += (double)r * (double)r;
                        }
                    }
                    a2 = warp_sum(a2);
                    put(tile, 0, a2);
                    tile_done(tile, 1);
                }
                groups_done(1);
                mark(PF_CHECK);
                if (!team_sync<ST>(I.sync, P, abort_word, ctl, sc, I.prof, leader_check)) { aborted = true; break; }
                act = read_action();
                mark(PF_CHECK_WAIT);
                if (act == ACT_DONE) break;
                if (act == ACT_FAIL) { retired = true; break; }
                // ACT_CYCLE: V0 holds the new residual
            }
            if (aborted || retired) break;
        } else if (act == ACT_ZERO_B || act == ACT_DONE) {
            const T* src = (act == ACT_ZERO_B) ? I.b : I.x;
            for (int tile = rank; tile < I.n_tiles; tile += P) {
                if (threadIdx.x == 0) pf_slice(src, sizeof(T), tile + P);
                else if (threadIdx.x == 1 && fuse_next) pf_slice(hout, sizeof(T), tile + P);
                else if (threadIdx.x == 2 && fuse_next) pf_slice(I.vflags, 1, tile + P);
                T cv[VPT], hn[VPT];
                uint8_t fl[VPT];
#pragma unroll
                for (int v = 0; v < VPT; ++v) {
                    const long long n = voxel(tile, v);
                    cv[v] = (n < N) ? src[n] : T(0);
                    hn[v] = (fuse_next && n < N) ? hout[n] : T(0);
                    fl[v] = (fuse_next && n < N) ? __ldg(I.vflags + n) : (uint8_t)0;
                }
#pragma unroll
                for (int v = 0; v < VPT; ++v) {
                    const long long n = voxel(tile, v);
                    if (n < N) I.u[n] = cv[v];
                }
                if (fuse_next) {
                    int32_t lt[VPT];
#pragma unroll
                    for (int v = 0; v < VPT; ++v) {
                        const long long n = voxel(tile, v);
                        lt[v] = (n < N && cv[v] >= T(0.5)) ? I.lat[n] : 0;
                    }
#pragma unroll
                    for (int v = 0; v < VPT; ++v) {
                        const long long n = voxel(tile, v);
                        if (n < N) react_voxel(n, cv[v], hn[v], lt[v], step, slot_now, fl[v], stim_next, hin);
                    }
                }
            }
            fused = fuse_next;
        } else {  // ACT_FAIL
            retired = true;
            break;
        }
        mark(PF_COPY);
        // No barrier at the end of the step: each voxel's u and h are written and
        // read again (next RHS pass 1) by the same thread, and every cross-CTA read
        // of the next step follows its mid-RHS barrier.
        if (prof_on && threadIdx.x == 0) pf[PF_STEPS] += 1;
        hbuf ^= 1;
        if (slot_now >= 0) {
            ++id_save;
            pending = fused ? -1 : slot_now;    // a fused pass wrote the sample already
        }
        prepared = fused;
    }

    // flush the sample and activation test of the last completed step
    if (!aborted && !retired) {
        const T* hcur = hbuf ? I.h1 : I.h0;
        if (pending >= 0 || step > sh_step0) {
            for (int tile = rank; tile < I.n_tiles; tile += P) {
#pragma unroll
                for (int v = 0; v < VPT; ++v) {
                    const long long n = voxel(tile, v);
                    if (n < N) sample_voxel(n, I.u[n], hcur[n], step - 1);
                }
            }
        }
        pending = -1;
    }
    if (prof_on && threadIdx.x == 0) {
        for (int i = 0; i < PF_TEAM; ++i) atomicAdd(I.prof + i, pf[i]);
        atomicExch(I.prof + PF_TEAM, (unsigned long long)P);
    }
    if (!aborted) {
        if (!team_sync<ST>(I.sync, P, abort_word, ctl, sc, I.prof, [&]() {
                if (threadIdx.x == 0) {
                    I.st->step = step;
                    I.st->id_save = id_save;
                    I.st->pending = pending;
                    I.st->hbuf = hbuf;
                }
            })) {
            aborted = true;
        }
    }
    if constexpr (ST) stg.quit();   // the producer warp drains its copies and exits
}

// ------------------------------------------------------------------ fill kernel
template <typename T>
__global__ void fill_kernel(T* p, long long n, T v) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long s = (long long)gridDim.x * blockDim.x;
    for (; i < n; i += s) p[i] = v;
}

template <typename T>
__global__ void convert_kernel(const double* src, T* dst, long long n) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long s = (long long)gridDim.x * blockDim.x;
    for (; i < n; i += s) dst[i] = (T)src[i];
}

}  // namespace phs

// ====================================================================== host side
using namespace phs;

namespace {

constexpr int kVptF32 = 4;
constexpr int kVptF32Min = 2;    // the smallest voxels-per-thread of any FP32 variant
constexpr int kVptF64 = 1;

// Compiled step-kernel variants: the same algorithm with different tile
// lengths (voxels per thread; a tile is 256 x VPT consecutive voxels),
// register budgets (__launch_bounds__ minimum CTAs per SM), neighbour tables
// (int32 or compact) and, for the FP32 staged ones, the shared-memory ring of
// the producer warp (bytes; sized so that MINB CTAs fit an SM next to the
// kernel's static shared memory).  The autotuner picks one.  Each exists
// without and with the anisotropic edge terms.
using StepFnF = void (*)(const InstDev<float>*, const int4*, long long, unsigned int*);
using StepFnD = void (*)(const InstDev<double>*, const int4*, long long, unsigned int*);
constexpr int kRing3 = 56 * 1024, kRing2 = 88 * 1024;
const StepFnF kStepF32[] = {step_kernel<float, kVptF32, 2, false, 0, false>, step_kernel<float, kVptF32, 3, false, 0, false>,
                            step_kernel<float, kVptF32, 4, false, 0, false>, step_kernel<float, 2, 4, false, 0, false>,
                            step_kernel<float, 2, 5, false, 0, false>,       step_kernel<float, 2, 3, false, kRing3, false>,
                            step_kernel<float, 4, 2, false, kRing2, false>,  step_kernel<float, 2, 5, false, 0, true>,
                            step_kernel<float, kVptF32, 4, false, 0, true>};
const StepFnF kStepF32Edge[] = {step_kernel<float, kVptF32, 2, true, 0, false>, step_kernel<float, kVptF32, 3, true, 0, false>,
                                step_kernel<float, kVptF32, 4, true, 0, false>, step_kernel<float, 2, 4, true, 0, false>,
                                step_kernel<float, 2, 5, true, 0, false>,       step_kernel<float, 2, 3, true, kRing3, false>,
                                step_kernel<float, 4, 2, true, kRing2, false>,  step_kernel<float, 2, 5, true, 0, true>,
                                step_kernel<float, kVptF32, 4, true, 0, true>};
const int kMinbF32[] = {2, 3, 4, 4, 5, 3, 2, 5, 4};
const int kVptOfF32[] = {kVptF32, kVptF32, kVptF32, 2, 2, 2, 4, 2, kVptF32};
const int kRingF32[] = {0, 0, 0, 0, 0, kRing3, kRing2, 0, 0};
// variants that read the compact neighbour table of every instance, and their
// int32-table twin (launched instead when an unfinished instance has none)
const int kTwinF32[] = {-1, -1, -1, -1, -1, -1, -1, 4, 2};
const StepFnD kStepF64[] = {step_kernel<double, kVptF64, 2, false, 0, false>, step_kernel<double, kVptF64, 3, false, 0, false>};
const StepFnD kStepF64Edge[] = {step_kernel<double, kVptF64, 2, true, 0, false>,
                                step_kernel<double, kVptF64, 3, true, 0, false>};
const int kMinbF64[] = {2, 3};
constexpr int kNumF32 = 9, kNumF64 = 2;
// Threads per CTA and dynamic shared memory of a variant's launch.
int ring_of(int prec_bytes, int variant) { return prec_bytes == 8 ? 0 : kRingF32[variant]; }
int threads_of(int prec_bytes, int variant) { return kThreads + (ring_of(prec_bytes, variant) > 0 ? 32 : 0); }
int dyn_smem_of(int prec_bytes, int variant) {
    const int r = ring_of(prec_bytes, variant);
    return r > 0 ? kRingHeader + r : 0;
}

// Tiles of an instance of n voxels under a variant.
int tiles_of(long long n, int vpt) { return (int)((n + (long long)kThreads * vpt - 1) / ((long long)kThreads * vpt)); }
int vpt_of(int prec_bytes, int variant) { return prec_bytes == 8 ? kVptF64 : kVptOfF32[variant]; }
// FP32: 64 registers, 4 CTAs/SM (the autotuner's pick on B200); FP64: 80
// registers, 3 CTAs/SM (plain GMRES(50) on a 157k-voxel shell: 2.06 ms per
// step against 2.46 ms with 128 registers and 2 CTAs/SM)
constexpr int kDefaultF32 = 2, kDefaultF64 = 1;

template <typename T>
const void* step_fn(int variant, bool edge = false) {
    if (sizeof(T) == 8) return edge ? (const void*)kStepF64Edge[variant] : (const void*)kStepF64[variant];
    return edge ? (const void*)kStepF32Edge[variant] : (const void*)kStepF32[variant];
}

struct InstHost {
    bool used = false;
    bool finished = false;
    phs_instance_desc d{};
    long long n = 0;
    long long ldv = 0;           // padded voxel count: length of every per-voxel array
    int n_tiles = 0;
    int m = 0;
    void* nb = nullptr;
    int16_t* nbr = nullptr;      // compact neighbour table, or nullptr
    int32_t* nbase = nullptr;
    void* coef = nullptr;
    void* cw = nullptr;
    void* m6 = nullptr;
    void* enb = nullptr;
    void* ecf = nullptr;
    void* vflags = nullptr;
    void* vparams = nullptr;
    void* stim = nullptr;
    void* u = nullptr;
    void* h0 = nullptr;
    void* h1 = nullptr;
    void* x = nullptr;
    void* b = nullptr;
    void* V = nullptr;
    void* dx = nullptr;
    void* hist_u = nullptr;
    void* hist_h = nullptr;
    int32_t* lat = nullptr;
    double* part = nullptr;
    double* gpart = nullptr;
    unsigned int* gcnt = nullptr;
    int n_groups = 0;
    Scalars* sc = nullptr;
    TeamSync* sync = nullptr;
    InstState* st = nullptr;
    unsigned long long* prof = nullptr;
    InstState st_host{};
    double kavg = 4.0;           // recent Arnoldi steps per step (cost model)
    long long ref_arnoldi = 0;   // counters at the last rebalance
    long long ref_step = 0;
    double weight = 0.0;         // measured CTA-time per step (0: use the model)
    int team = 0;                // CTAs given to this instance by the current plan
    unsigned long long prof_ref[16] = {};
};

void free_inst(InstHost& h) {
    void* ptrs[] = {h.nb, h.nbr, h.nbase, h.coef, h.cw, h.m6, h.enb, h.ecf, h.dx, h.vflags, h.vparams, h.stim, h.u, h.h0, h.h1, h.x, h.b, h.V,
                    h.hist_u, h.hist_h, h.lat, h.part, h.gpart, h.gcnt, h.sc, h.sync, h.st, h.prof};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    h = InstHost();
}

}  // namespace

struct phs_engine {
    int prec = PHS_PREC_F32;
    int device = 0;
    int sms = 0;
    std::vector<InstHost> inst;
    unsigned int* abort_word = nullptr;
    void* d_desc = nullptr;
    size_t d_desc_bytes = 0;
    int4* d_map = nullptr;
    size_t d_map_n = 0;
    long long launches = 0;
    bool broken = false;
    // cached launch plan (rebuilt when the instance set changes)
    bool dirty = true;
    std::vector<int> act;
    std::vector<std::pair<size_t, int>> waves;
    int plan_cps = -1;
    bool plan_edge = false;  // the plan launches the edge-term kernel
    bool auto_balance = true;  // rebalance on the 2nd and 3rd advance after the instance set changes
    int auto_left = 0;
    long long auto_mark = 0;   // launch count when the set changed / at the last automatic rebalance
    bool auto_prof = false;    // the phase timers were switched on by the automatic balancing
    // CUDA graphs of the launch sequence, keyed by steps per launch
    std::map<long long, cudaGraphExec_t> graphs;
    bool graphs_ok = true;
    int variant = -1;        // step-kernel variant (-1: default of the precision)
    bool profile = false;    // per-instance phase timers
    bool test_overcount = false;  // test hook: first team waits for one CTA too many
    int default_cps = 0;     // CTAs per SM when advance() is given 0 (0: occupancy limit)
    int wave_instances = 0;  // instances per launch wave (0: as many as the grid holds)
    bool group_sums = true;  // FP64: partial sums combined in groups of tiles before the leader
    bool compact_nb = true;  // instances read the compact neighbour table when they have one
};

namespace {

template <typename T>
int occupancy_for(int* ctas, int variant, bool edge = false) {
    const void* fn = step_fn<T>(variant, edge);
    const int smem = dyn_smem_of((int)sizeof(T), variant);
    if (smem > 0) {
        cudaError_t a = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (a != cudaSuccess) { set_last_error("ring shared memory", a); return PHS_ERR_CUDA; }
    }
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, fn, threads_of((int)sizeof(T), variant), smem);
    if (e != cudaSuccess) { set_last_error("occupancy", e); return PHS_ERR_CUDA; }
    return PHS_OK;
}

template <typename T>
void fill_dev(T* p, long long n, T v, cudaStream_t s) {
    if (n <= 0) return;
    long long blocks = std::min<long long>((n + 255) / 256, 65535);
    fill_kernel<T><<<(unsigned)blocks, 256, 0, s>>>(p, n, v);
}

// Device-side form of validate_desc's table checks (device_tables instances).
template <typename T>
__global__ void check_tables(long long n, const int32_t* nb, const T* coef, const T* cw, const uint8_t* m6,
                             const int32_t* enb, const T* ecf, unsigned int* err) {
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {
        bool bad = false;
        for (int k = 0; k < 6; ++k) {
            const int32_t q = nb[6 * r + k];
            bad |= (q < 0 || q >= n);
            if (coef) bad |= !isfinite((double)coef[6 * r + k]);
        }
        if (cw) bad |= !isfinite((double)cw[r]) || (m6[r] & 0xC0u);
        if (enb) {
            for (int k = 0; k < 12; ++k) bad |= (enb[12 * r + k] < 0 || enb[12 * r + k] >= n);
            for (int k = 0; k < 6; ++k) bad |= !isfinite((double)ecf[6 * r + k]);
        }
        if (bad) atomicOr(err, 1u);
    }
}

// ---- compact neighbour table (decode_nb)
// Whether slot k of row v has a neighbour the operator reads: its coefficient
// is nonzero, the test lap_row makes.
template <typename T>
__device__ __forceinline__ bool nb_present(const T* coef, const T* cw, const uint8_t* m6, long long v, int k) {
    if (cw) return ((m6[v] >> k) & 1u) && cw[v] != T(0);
    return coef[6 * v + k] != T(0);
}

// flags[k] bit 0: some present neighbour of slot k is not n + 1; bit 1: not n - 1.
template <typename T>
__global__ void nb_slot_kinds(long long n, const int32_t* nb, const T* coef, const T* cw, const uint8_t* m6,
                              unsigned int* flags) {
    unsigned int f[6] = {0u, 0u, 0u, 0u, 0u, 0u};
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        for (int k = 0; k < 6; ++k) {
            if (!nb_present(coef, cw, m6, v, k)) continue;
            const long long dq = (long long)nb[6 * v + k] - v;
            f[k] |= (dq != 1 ? 1u : 0u) | (dq != -1 ? 2u : 0u);
        }
    }
    for (int k = 0; k < 6; ++k) {
        unsigned int a = f[k];
        for (int o = 16; o > 0; o >>= 1) a |= __shfl_xor_sync(0xffffffffu, a, o);
        if ((threadIdx.x & 31) == 0 && a) atomicOr(flags + k, a);
    }
}

// One CTA of 256 threads per 512-voxel block: for slots 2..5 the base offset
// (middle of the block's range over present neighbours) and the int16
// residuals; *fail set when a block's range does not fit.  Voxels past n
// (padding) get zeros.
template <typename T>
__global__ void nb_compact(long long n, const int32_t* nb, const T* coef, const T* cw, const uint8_t* m6,
                           int16_t* nbr, int32_t* nbase, unsigned int* fail) {
    __shared__ long long lo[8][4], hi[8][4];
    __shared__ int32_t base[4];
    const long long v0 = (long long)blockIdx.x * 512;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    long long mn[4], mx[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) { mn[r] = LLONG_MAX; mx[r] = LLONG_MIN; }
    for (int h = 0; h < 2; ++h) {
        const long long v = v0 + h * 256 + threadIdx.x;
        if (v >= n) continue;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            if (!nb_present(coef, cw, m6, v, r + 2)) continue;
            const long long dq = (long long)nb[6 * v + r + 2] - v;
            mn[r] = min(mn[r], dq);
            mx[r] = max(mx[r], dq);
        }
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        for (int o = 16; o > 0; o >>= 1) {
            mn[r] = min(mn[r], (long long)__shfl_xor_sync(0xffffffffu, mn[r], o));
            mx[r] = max(mx[r], (long long)__shfl_xor_sync(0xffffffffu, mx[r], o));
        }
        if (lane == 0) { lo[w][r] = mn[r]; hi[w][r] = mx[r]; }
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        const int r = threadIdx.x;
        long long a = LLONG_MAX, b = LLONG_MIN;
        for (int q = 0; q < 8; ++q) { a = min(a, lo[q][r]); b = max(b, hi[q][r]); }
        long long bs = 0;
        if (a <= b) {
            bs = a + (b - a) / 2;
            if (b - bs > 32767 || a - bs < -32768 || bs > INT_MAX / 2 || bs < INT_MIN / 2) atomicOr(fail, 1u);
        }
        base[r] = (int32_t)bs;
        nbase[blockIdx.x * 4 + r] = (int32_t)bs;
    }
    __syncthreads();
    for (int h = 0; h < 2; ++h) {
        const long long v = v0 + h * 256 + threadIdx.x;
        long long d[4] = {0, 0, 0, 0};
        if (v < n) {
#pragma unroll
            for (int r = 0; r < 4; ++r)
                if (nb_present(coef, cw, m6, v, r + 2)) d[r] = (long long)nb[6 * v + r + 2] - v - base[r];
        }
        short res[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) res[r] = (short)max(-32768ll, min(32767ll, d[r]));
        reinterpret_cast<short4*>(nbr)[v] = make_short4(res[0], res[1], res[2], res[3]);
    }
}

// Copy n doubles (host, or device when on_device) into a new array of T of
// alloc_n >= n elements (the tail is zero).
template <typename T>
int upload_converted(void** dst, const double* src, long long n, bool on_device, long long alloc_n) {
    PHS_CUDA_TRY(cudaMalloc(dst, (size_t)alloc_n * sizeof(T)));
    if (alloc_n > n) PHS_CUDA_TRY(cudaMemset((char*)*dst + (size_t)n * sizeof(T), 0, (size_t)(alloc_n - n) * sizeof(T)));
    if (sizeof(T) == 8) {
        PHS_CUDA_TRY(cudaMemcpy(*dst, src, (size_t)n * 8, cudaMemcpyDefault));
        return PHS_OK;
    }
    double* tmp = nullptr;
    cudaError_t e = cudaSuccess;
    if (!on_device) {
        PHS_CUDA_TRY(cudaMalloc(&tmp, (size_t)n * 8));
        e = cudaMemcpy(tmp, src, (size_t)n * 8, cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) {
        long long blocks = std::min<long long>((n + 255) / 256, 65535);
        convert_kernel<T><<<(unsigned)std::max<long long>(blocks, 1), 256>>>(on_device ? src : tmp, (T*)*dst, n);
        e = cudaDeviceSynchronize();
    }
    if (tmp) cudaFree(tmp);
    if (e != cudaSuccess) { set_last_error("upload_converted", e); return PHS_ERR_CUDA; }
    return PHS_OK;
}

int validate_desc(const phs_instance_desc* d) {
    if (!d || d->n_voxel <= 0 || d->n_voxel > (1ll << 31) - 1) return PHS_ERR_BAD_ARG;
    if (d->model != PHS_MODEL_MS && d->model != PHS_MODEL_AP) return PHS_ERR_BAD_ARG;
    if (d->restart < 1 || d->restart > kMaxRestart) return PHS_ERR_BAD_ARG;
    if (!d->nb6 || !d->vflags) return PHS_ERR_BAD_ARG;
    if (!d->coef6 && !(d->cw && d->mask6)) return PHS_ERR_BAD_ARG;
    if (d->n_steps < 0 || (d->n_steps > 0 && !d->stim)) return PHS_ERR_BAD_ARG;
    if (d->n_samples < 0 || d->sample_stride < 0 || d->maxiter < 1) return PHS_ERR_BAD_ARG;
    if (!(d->dt > 0.0)) return PHS_ERR_BAD_ARG;
    if ((d->nb_edge == nullptr) != (d->coef_edge == nullptr)) return PHS_ERR_BAD_ARG;
    if (d->device_tables) return PHS_OK;   // checked on the device after the copy (check_tables)
    const long long n = d->n_voxel;
    for (long long i = 0; i < 6 * n; ++i) {
        int32_t q = d->nb6[i];
        if (q < 0 || q >= n) return PHS_ERR_BAD_TABLE;
        if (d->coef6 && !std::isfinite(d->coef6[i])) return PHS_ERR_BAD_TABLE;
    }
    if (d->cw)
        for (long long i = 0; i < n; ++i)
            if (!std::isfinite(d->cw[i]) || (d->mask6[i] & 0xC0u)) return PHS_ERR_BAD_TABLE;
    if (d->nb_edge) {
        for (long long i = 0; i < 12 * n; ++i)
            if (d->nb_edge[i] < 0 || d->nb_edge[i] >= n) return PHS_ERR_BAD_TABLE;
        for (long long i = 0; i < 6 * n; ++i)
            if (!std::isfinite(d->coef_edge[i])) return PHS_ERR_BAD_TABLE;
    }
    return PHS_OK;
}

// Build the compact neighbour table (decode_nb) of an instance whose tables
// are on the device (h.nb with the coefficients).  Leaves h.nbr null when a
// present neighbour of slot 0 is not n + 1, one of slot 1 not n - 1, or a
// block's offsets of another slot do not fit int16.
template <typename T>
int build_compact_nb(InstHost& h) {
    const long long n = h.n;
    unsigned int* d_w = nullptr;
    PHS_CUDA_TRY(cudaMalloc((void**)&d_w, 8 * sizeof(unsigned int)));
    unsigned int w[8] = {};
    cudaError_t ce = cudaMemset(d_w, 0, 8 * sizeof(unsigned int));
    const long long blocks = std::max<long long>(1, std::min<long long>((n + 255) / 256, 4096));
    if (ce == cudaSuccess) {
        nb_slot_kinds<T><<<(unsigned)blocks, 256>>>(n, (const int32_t*)h.nb, (const T*)h.coef, (const T*)h.cw,
                                                    (const uint8_t*)h.m6, d_w);
        ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) ce = cudaMemcpy(w, d_w, 8 * sizeof(unsigned int), cudaMemcpyDeviceToHost);
    if (ce == cudaSuccess && !(w[0] & 1u) && !(w[1] & 2u)) {
        const long long nblk = h.ldv / 512;
        ce = cudaMalloc((void**)&h.nbr, (size_t)h.ldv * 4 * sizeof(int16_t));
        if (ce == cudaSuccess) ce = cudaMalloc((void**)&h.nbase, (size_t)nblk * 4 * sizeof(int32_t));
        if (ce == cudaSuccess) ce = cudaMemset(d_w + 6, 0, sizeof(unsigned int));
        if (ce == cudaSuccess) {
            nb_compact<T><<<(unsigned)nblk, 256>>>(n, (const int32_t*)h.nb, (const T*)h.coef, (const T*)h.cw,
                                                   (const uint8_t*)h.m6, h.nbr, h.nbase, d_w + 6);
            ce = cudaGetLastError();
        }
        if (ce == cudaSuccess) ce = cudaMemcpy(w + 6, d_w + 6, sizeof(unsigned int), cudaMemcpyDeviceToHost);
        if (ce != cudaSuccess || w[6] != 0u) {
            if (h.nbr) cudaFree(h.nbr);
            if (h.nbase) cudaFree(h.nbase);
            h.nbr = nullptr;
            h.nbase = nullptr;
        }
    }
    cudaFree(d_w);
    if (ce != cudaSuccess) { set_last_error("build_compact_nb", ce); return PHS_ERR_CUDA; }
    return PHS_OK;
}

template <typename T>
int add_instance(phs_engine* e, const phs_instance_desc* d, int* slot) {
    int rc = validate_desc(d);
    if (rc != PHS_OK) return rc;
    InstHost h;
    h.used = true;
    h.d = *d;
    h.n = d->n_voxel;
    const int vpt = sizeof(T) == 8 ? kVptF64 : kVptF32Min;   // allocations cover every variant's tiles
    const long long tile = (long long)kThreads * vpt;
    h.n_tiles = (int)((h.n + tile - 1) / tile);
    h.m = (int)std::min<long long>(d->restart, h.n);
    const size_t n = (size_t)h.n;
    // per-voxel arrays hold a whole number of the largest tile (zero tail), so
    // a tile's slice of any of them can be copied whole
    const size_t np = (n + kPadVoxels - 1) / kPadVoxels * kPadVoxels;
    h.ldv = (long long)np;
    auto fail = [&](int code) { free_inst(h); return code; };
#define PHS_ALLOC(ptr, bytes)                                            \
    do {                                                                 \
        cudaError_t _e = cudaMalloc((void**)&(ptr), (bytes));            \
        if (_e != cudaSuccess) { set_last_error("cudaMalloc", _e); return fail(PHS_ERR_OOM); } \
    } while (0)
    // tables: host arrays, or device arrays when device_tables (cudaMemcpyDefault)
    const bool dev = d->device_tables != 0;
    auto copy_in = [&](void* dst, const void* src, size_t bytes, size_t alloc_bytes) {
        if (alloc_bytes > bytes && cudaMemset((char*)dst + bytes, 0, alloc_bytes - bytes) != cudaSuccess) return false;
        return cudaMemcpy(dst, src, bytes, cudaMemcpyDefault) == cudaSuccess;
    };
    PHS_ALLOC(h.nb, np * 6 * sizeof(int32_t));
    if (!copy_in(h.nb, d->nb6, n * 6 * sizeof(int32_t), np * 6 * sizeof(int32_t))) return fail(PHS_ERR_CUDA);
    if (d->cw) {
        if ((rc = upload_converted<T>(&h.cw, d->cw, (long long)n, dev, (long long)np)) != PHS_OK) return fail(rc);
        PHS_ALLOC(h.m6, np);
        if (!copy_in(h.m6, d->mask6, n, np)) return fail(PHS_ERR_CUDA);
    } else {
        if ((rc = upload_converted<T>(&h.coef, d->coef6, (long long)n * 6, dev, (long long)np * 6)) != PHS_OK)
            return fail(rc);
    }
    if (d->nb_edge) {
        PHS_ALLOC(h.enb, np * 12 * sizeof(int32_t));
        if (!copy_in(h.enb, d->nb_edge, n * 12 * sizeof(int32_t), np * 12 * sizeof(int32_t))) return fail(PHS_ERR_CUDA);
        if ((rc = upload_converted<T>(&h.ecf, d->coef_edge, (long long)n * 6, dev, (long long)np * 6)) != PHS_OK)
            return fail(rc);
    }
    PHS_ALLOC(h.vflags, np);
    if (!copy_in(h.vflags, d->vflags, n, np)) return fail(PHS_ERR_CUDA);
    if (d->vparams) {
        if ((rc = upload_converted<T>(&h.vparams, d->vparams, (long long)n * 5, dev, (long long)np * 5)) != PHS_OK)
            return fail(rc);
    }
    if (dev) {
        // the checks validate_desc makes on host tables, on the copies
        unsigned int* d_err = nullptr;
        if (cudaMalloc((void**)&d_err, sizeof(unsigned int)) != cudaSuccess) return fail(PHS_ERR_OOM);
        unsigned int h_err = 0;
        cudaError_t ce = cudaMemset(d_err, 0, sizeof(unsigned int));
        if (ce == cudaSuccess) {
            const long long blocks = std::max<long long>(1, std::min<long long>(((long long)n + 255) / 256, 65535));
            check_tables<T><<<(unsigned)blocks, 256>>>((long long)n, (const int32_t*)h.nb, (const T*)h.coef,
                                                       (const T*)h.cw, (const uint8_t*)h.m6, (const int32_t*)h.enb,
                                                       (const T*)h.ecf, d_err);
            ce = cudaGetLastError();
        }
        if (ce == cudaSuccess) ce = cudaMemcpy(&h_err, d_err, sizeof(h_err), cudaMemcpyDeviceToHost);
        cudaFree(d_err);
        if (ce != cudaSuccess) { set_last_error("check_tables", ce); return fail(PHS_ERR_CUDA); }
        if (h_err) return fail(PHS_ERR_BAD_TABLE);
    }
    if ((rc = build_compact_nb<T>(h)) != PHS_OK) return fail(rc);
    const size_t ns = (size_t)std::max<int64_t>(d->n_steps, 1);
    PHS_ALLOC(h.stim, ns);
    if (d->n_steps > 0) {
        if (cudaMemcpy(h.stim, d->stim, (size_t)d->n_steps, cudaMemcpyHostToDevice) != cudaSuccess) return fail(PHS_ERR_CUDA);
    } else {
        cudaMemset(h.stim, 0, ns);
    }
    PHS_ALLOC(h.u, np * sizeof(T));
    PHS_ALLOC(h.h0, np * sizeof(T));
    PHS_ALLOC(h.h1, np * sizeof(T));
    PHS_ALLOC(h.x, np * sizeof(T));
    PHS_ALLOC(h.b, np * sizeof(T));
    PHS_ALLOC(h.V, np * (size_t)(h.m + 1) * sizeof(T));
    if (d->guess) PHS_ALLOC(h.dx, np * sizeof(T));
    const size_t S = (size_t)std::max(d->n_samples, 1);
    PHS_ALLOC(h.hist_u, S * n * sizeof(T));
    if (d->save_h) PHS_ALLOC(h.hist_h, S * n * sizeof(T));
    PHS_ALLOC(h.lat, np * sizeof(int32_t));
    const size_t nparts = (size_t)h.n_tiles * (kWarpParts<T> ? kWarps : 1);
    PHS_ALLOC(h.part, nparts * (h.m + 2) * sizeof(double));
    h.n_groups = (h.n_tiles + kGroupTiles - 1) / kGroupTiles;
    if (!kWarpParts<T>) {
        PHS_ALLOC(h.gpart, (size_t)h.n_groups * (h.m + 2) * sizeof(double));
        PHS_ALLOC(h.gcnt, (size_t)h.n_groups * sizeof(unsigned int));
    }
    PHS_ALLOC(h.sc, sizeof(Scalars));
    PHS_ALLOC(h.sync, sizeof(TeamSync));
    PHS_ALLOC(h.st, sizeof(InstState));
#undef PHS_ALLOC
    fill_dev<T>((T*)h.u, (long long)np, (T)d->u0, 0);
    fill_dev<T>((T*)h.h0, (long long)np, (T)d->h0, 0);
    fill_dev<T>((T*)h.h1, (long long)np, (T)d->h0, 0);
    fill_dev<T>((T*)h.x, (long long)np, (T)0, 0);
    fill_dev<T>((T*)h.b, (long long)np, (T)0, 0);
    cudaMemset(h.V, 0, np * (size_t)(h.m + 1) * sizeof(T));
    if (h.dx) cudaMemset(h.dx, 0, np * sizeof(T));
    cudaMemset(h.hist_u, 0, S * n * sizeof(T));
    if (h.hist_h) cudaMemset(h.hist_h, 0, S * n * sizeof(T));
    cudaMemset(h.lat, 0xff, np * sizeof(int32_t));
    cudaMemset(h.part, 0, nparts * (h.m + 2) * sizeof(double));
    if (h.gpart) cudaMemset(h.gpart, 0, (size_t)h.n_groups * (h.m + 2) * sizeof(double));
    if (h.gcnt) cudaMemset(h.gcnt, 0, (size_t)h.n_groups * sizeof(unsigned int));
    cudaMemset(h.sc, 0, sizeof(Scalars));
    cudaMemset(h.sync, 0, sizeof(TeamSync));
    InstState st{};
    st.step = 0;
    st.id_save = 0;
    st.pending = -1;
    st.status = PHS_OK;
    st.hbuf = 0;
    cudaMemcpy(h.st, &st, sizeof(st), cudaMemcpyHostToDevice);
    cudaError_t ce = cudaDeviceSynchronize();
    if (ce != cudaSuccess) { set_last_error("add_instance", ce); return fail(PHS_ERR_CUDA); }
    h.st_host = st;
    h.finished = (d->n_steps == 0);
    // find a free slot
    int s = -1;
    for (size_t i = 0; i < e->inst.size(); ++i)
        if (!e->inst[i].used) { s = (int)i; break; }
    if (s < 0) { s = (int)e->inst.size(); e->inst.push_back(InstHost()); }
    if (e->profile) {
        if (cudaMalloc((void**)&h.prof, kProfSlots * sizeof(unsigned long long)) == cudaSuccess)
            cudaMemset(h.prof, 0, kProfSlots * sizeof(unsigned long long));
    }
    e->inst[s] = h;
    e->dirty = true;
    e->auto_left = 2;
    e->auto_mark = e->launches;
    *slot = s;
    return PHS_OK;
}

template <typename T>
InstDev<T> make_dev(const InstHost& h, bool group_sums, int vpt, bool compact_nb) {
    InstDev<T> I{};
    I.nb = (const int32_t*)h.nb;
    if (compact_nb && h.nbr) {
        I.nbr = h.nbr;
        I.nbase = h.nbase;
    }
    I.coef = (const T*)h.coef;
    I.cw = (const T*)h.cw;
    I.m6 = (const uint8_t*)h.m6;
    I.enb = (const int32_t*)h.enb;
    I.ecf = (const T*)h.ecf;
    I.vflags = (const uint8_t*)h.vflags;
    I.vparams = (const T*)h.vparams;
    I.stim = (const uint8_t*)h.stim;
    I.u = (T*)h.u;
    I.h0 = (T*)h.h0;
    I.h1 = (T*)h.h1;
    I.x = (T*)h.x;
    I.b = (T*)h.b;
    I.V = (T*)h.V;
    I.ldv = h.ldv;
    I.dx = (T*)h.dx;
    I.hist_u = (T*)h.hist_u;
    I.hist_h = (T*)h.hist_h;
    I.lat = h.lat;
    I.part = h.part;
    I.gpart = group_sums ? h.gpart : nullptr;
    I.gcnt = h.gcnt;
    I.n_groups = (tiles_of(h.n, vpt) + kGroupTiles - 1) / kGroupTiles;
    I.sc = h.sc;
    I.sync = h.sync;
    I.st = h.st;
    I.prof = h.prof;
    T raw[5];
    for (int q = 0; q < 5; ++q) raw[q] = (T)h.d.params[q];
    model_form<T>(h.d.model, raw, I.params);
    I.dt = (T)h.d.dt;
    I.half_dt = (T)h.d.dt / T(2);
    I.jmag = (T)h.d.j_stim;
    I.tol = h.d.tol;
    I.atol = h.d.atol;
    I.n = h.n;
    I.n_steps = h.d.n_steps;
    I.tb_steps = h.d.tblock_steps;
    I.n_tiles = tiles_of(h.n, vpt);
    I.ps = h.m + 2;
    I.model = h.d.model;
    I.m = h.m;
    I.maxiter = h.d.maxiter;
    I.full_cycles = h.d.full_cycles;
    I.stride = h.d.sample_stride;
    I.n_samples = h.d.n_samples;
    I.save_h = h.d.save_h;
    return I;
}

// Split G CTAs over the instances.  A team of P CTAs over `tiles` tiles takes
// time proportional to (cost per tile) x ceil(tiles / P): its CTAs walk their
// tiles one after another and the one with the most tiles sets the pace.  The
// cost of an instance is `weight` (voxels times the cost of a step in units of
// one Arnoldi iteration, or the measured CTA-time per step), per tile weight /
// tiles.  Starting from one CTA each, the instance with the longest time
// receives the fewest CTAs that lower its tiles-per-CTA count, until the CTAs
// run out or the longest one cannot be helped; CTAs left over (when every team
// already has one CTA per tile, or the longest would need more than remain) go
// to no one.  Never more CTAs than tiles.
std::vector<int> team_sizes(const std::vector<int>& tiles, const std::vector<double>& weight, int G) {
    const int A = (int)tiles.size();
    std::vector<int> P(A, 1);
    int used = A;
    auto per_tile = [&](int i) { return weight[i] / std::max(tiles[i], 1); };
    auto span = [&](int i, int p) { return (tiles[i] + p - 1) / p; };
    while (used < G) {
        int worst = -1;
        double wt = -1.0;
        for (int i = 0; i < A; ++i) {
            const double t = per_tile(i) * span(i, P[i]);
            if (t > wt) { wt = t; worst = i; }
        }
        if (worst < 0) break;
        const int cur = span(worst, P[worst]);
        if (cur <= 1) break;                                   // one tile per CTA already
        const int need = (tiles[worst] + (cur - 1) - 1) / (cur - 1);   // fewest CTAs with span cur - 1
        if (used + (need - P[worst]) > G) break;
        used += need - P[worst];
        P[worst] = need;
    }
    return P;
}

// The variant a launch uses: the configured one, or its int32-table twin when
// it reads compact tables and an unfinished instance has none (or the engine's
// compact tables are off).
template <typename T>
int variant_of(const phs_engine* e) {
    int v = e->variant >= 0 ? e->variant : (sizeof(T) == 8 ? kDefaultF64 : kDefaultF32);
    if (sizeof(T) == 4 && kTwinF32[v] >= 0) {
        bool all = e->compact_nb;
        for (const auto& h : e->inst)
            if (h.used && !h.finished && !h.nbr) all = false;
        if (!all) v = kTwinF32[v];
    }
    return v;
}

void drop_graphs(phs_engine* e) {
    for (auto& kv : e->graphs) cudaGraphExecDestroy(kv.second);
    e->graphs.clear();
}

template <typename T>
cudaError_t launch_waves(phs_engine* e, long long n_steps, cudaStream_t stream) {
    for (auto& wv : e->waves) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)wv.second);
        const int variant = variant_of<T>(e);
        cfg.blockDim = dim3((unsigned)threads_of((int)sizeof(T), variant));
        cfg.dynamicSmemBytes = (size_t)dyn_smem_of((int)sizeof(T), variant);
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        const InstDev<T>* dd = (const InstDev<T>*)e->d_desc;
        const int4* mp = e->d_map + wv.first;
        long long ns = n_steps;
        unsigned int* ab = e->abort_word;
        void* args[] = {(void*)&dd, (void*)&mp, (void*)&ns, (void*)&ab};
        cudaError_t ce = cudaLaunchKernelExC(&cfg, step_fn<T>(variant, e->plan_edge), args);
        if (ce != cudaSuccess) return ce;
    }
    return cudaSuccess;
}

// (Re)build the launch plan: device descriptors, team map and waves.
template <typename T>
int build_plan(phs_engine* e, int cps, bool edge) {
    // earlier launches may still read the old descriptors
    PHS_CUDA_TRY(cudaDeviceSynchronize());
    const int G = e->sms * cps;
    std::vector<int> act;
    for (size_t i = 0; i < e->inst.size(); ++i)
        if (e->inst[i].used && !e->inst[i].finished) act.push_back((int)i);
    e->act = act;
    e->waves.clear();
    drop_graphs(e);
    e->plan_cps = cps;
    e->plan_edge = edge;
    e->dirty = false;
    if (act.empty()) return PHS_OK;
    std::vector<InstDev<T>> descs;
    descs.reserve(act.size());
    const int vpt = vpt_of((int)sizeof(T), variant_of<T>(e));
    for (int i : act) descs.push_back(make_dev<T>(e->inst[i], e->group_sums, vpt, e->compact_nb));
    size_t bytes = descs.size() * sizeof(InstDev<T>);
    if (bytes > e->d_desc_bytes) {
        if (e->d_desc) cudaFree(e->d_desc);
        PHS_CUDA_TRY(cudaMalloc(&e->d_desc, bytes));
        e->d_desc_bytes = bytes;
    }
    PHS_CUDA_TRY(cudaMemcpy(e->d_desc, descs.data(), bytes, cudaMemcpyHostToDevice));

    // waves of at most G instances (fewer with wave_instances: each wave is a
    // launch of its own over the whole grid, so the instances of a wave share
    // the L2 with fewer others)
    std::vector<int4> map_all;
    std::vector<std::pair<size_t, int>>& waves = e->waves;  // (offset into map, grid)
    const size_t per_wave = (size_t)((e->wave_instances > 0) ? std::min(G, e->wave_instances) : G);
    for (size_t w0 = 0; w0 < act.size(); w0 += per_wave) {
        size_t w1 = std::min(act.size(), w0 + per_wave);
        std::vector<int> tiles;
        std::vector<double> weight;
        bool measured = true;
        for (size_t i = w0; i < w1; ++i) measured = measured && e->inst[act[i]].weight > 0.0;
        for (size_t i = w0; i < w1; ++i) {
            const InstHost& h = e->inst[act[i]];
            tiles.push_back(tiles_of(h.n, vpt));
            weight.push_back(measured ? h.weight : (double)h.n * (1.6 + h.kavg));
        }
        std::vector<int> P = team_sizes(tiles, weight, G);
        for (size_t i = w0; i < w1; ++i) e->inst[act[i]].team = P[i - w0];
        size_t off = map_all.size();
        int grid = 0;
        for (size_t i = w0; i < w1; ++i) {
            int p = P[i - w0];
            // test hook: the first team expects one CTA that is never launched, so
            // its first barrier can only end through the bounded wait
            const int claimed = p + ((e->test_overcount && i == w0) ? 1 : 0);
            for (int r = 0; r < p; ++r) map_all.push_back(make_int4((int)i, r, claimed, 0));
            grid += p;
        }
        waves.push_back({off, grid});
    }
    if (map_all.size() > e->d_map_n) {
        if (e->d_map) cudaFree(e->d_map);
        PHS_CUDA_TRY(cudaMalloc(&e->d_map, map_all.size() * sizeof(int4)));
        e->d_map_n = map_all.size();
    }
    PHS_CUDA_TRY(cudaMemcpy(e->d_map, map_all.data(), map_all.size() * sizeof(int4), cudaMemcpyHostToDevice));
    return PHS_OK;
}

template <typename T>
int advance_impl(phs_engine* e, long long n_steps, int ctas_per_sm, cudaStream_t stream, bool sync) {
    if (e->broken) return PHS_ERR_STATE;
    if (n_steps <= 0) return PHS_OK;
    // automatic balancing: the launch after an instance set change runs with the
    // phase timers on (unless the caller has them on already), the next two
    // re-split the CTAs by the measured cost, then the timers go off again
    if (e->auto_balance && e->auto_left > 0 && !e->profile) {
        const int rp = phs_engine_config(e, PHS_CFG_PROFILE, 1);
        if (rp != PHS_OK) return rp;
        e->auto_prof = true;
    }
    if (e->auto_balance && e->auto_left > 0 && e->launches > e->auto_mark) {
        const int rb = phs_engine_rebalance(e);
        if (rb != PHS_OK) return rb;
        e->auto_left -= 1;
        e->auto_mark = e->launches;
        if (e->auto_left == 0 && e->auto_prof) {
            const int rp = phs_engine_config(e, PHS_CFG_PROFILE, 0);
            if (rp != PHS_OK) return rp;
            e->auto_prof = false;
        }
    }
    // the edge-term kernel only when an unfinished instance is anisotropic
    bool edge = false;
    for (const auto& h : e->inst)
        if (h.used && !h.finished && h.enb) edge = true;
    int occ = 0;
    int rc = occupancy_for<T>(&occ, variant_of<T>(e), edge);
    if (rc != PHS_OK) return rc;
    if (occ < 1) return PHS_ERR_CUDA;
    if (ctas_per_sm <= 0) ctas_per_sm = e->default_cps;
    int cps = (ctas_per_sm > 0) ? std::min(ctas_per_sm, occ) : occ;
    if (e->dirty || cps != e->plan_cps || edge != e->plan_edge) {
        rc = build_plan<T>(e, cps, edge);
        if (rc != PHS_OK) return rc;
    }
    const std::vector<int>& act = e->act;
    if (act.empty()) return PHS_OK;
    cudaError_t ce = cudaSuccess;
    bool launched = false;
    if (stream != nullptr && e->graphs_ok) {
        auto it = e->graphs.find(n_steps);
        if (it == e->graphs.end()) {
            cudaGraph_t g = nullptr;
            cudaGraphExec_t ge = nullptr;
            ce = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
            if (ce == cudaSuccess) {
                cudaError_t le = launch_waves<T>(e, n_steps, stream);
                ce = cudaStreamEndCapture(stream, &g);
                if (le != cudaSuccess) ce = le;
            }
            if (ce == cudaSuccess) ce = cudaGraphInstantiate(&ge, g, 0);
            if (g) cudaGraphDestroy(g);
            if (ce == cudaSuccess) {
                it = e->graphs.emplace(n_steps, ge).first;
            } else {
                cudaGetLastError();  // clear; fall back to direct launches
                e->graphs_ok = false;
            }
        }
        if (e->graphs_ok) {
            ce = cudaGraphLaunch(it->second, stream);
            if (ce != cudaSuccess) { set_last_error("cudaGraphLaunch", ce); return PHS_ERR_CUDA; }
            launched = true;
        }
    }
    if (!launched) {
        ce = launch_waves<T>(e, n_steps, stream);
        if (ce != cudaSuccess) { set_last_error("launch step_kernel", ce); return PHS_ERR_CUDA; }
    }
    e->launches += (long long)e->waves.size();
    if (!sync) return PHS_OK;
    PHS_CUDA_TRY(cudaStreamSynchronize(stream));
    unsigned int ab = 0;
    PHS_CUDA_TRY(cudaMemcpy(&ab, e->abort_word, sizeof(ab), cudaMemcpyDeviceToHost));
    if (ab) { e->broken = true; return PHS_ERR_TIMEOUT; }
    int worst = PHS_OK;
    for (int i : act) {
        InstHost& h = e->inst[i];
        PHS_CUDA_TRY(cudaMemcpy(&h.st_host, h.st, sizeof(InstState), cudaMemcpyDeviceToHost));
        if (h.st_host.step >= h.d.n_steps || h.st_host.status == PHS_ERR_NONFINITE) {
            if (!h.finished) e->dirty = true;
            h.finished = true;
        }
        if (h.st_host.status == PHS_ERR_NONFINITE) worst = PHS_ERR_NONFINITE;
        else if (h.st_host.status == PHS_WARN_NO_CONVERGE && worst == PHS_OK) worst = PHS_WARN_NO_CONVERGE;
    }
    return worst;
}

}  // namespace

// ====================================================================== C ABI
extern "C" {

int phs_device_query(int precision, int* sm_count, int* ctas_per_sm) {
    int dev = 0;
    PHS_CUDA_TRY(cudaGetDevice(&dev));
    int sms = 0;
    PHS_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    int occ = 0;
    int rc = (precision == PHS_PREC_F64) ? occupancy_for<double>(&occ, kDefaultF64)
                                         : occupancy_for<float>(&occ, kDefaultF32);
    if (rc != PHS_OK) return rc;
    if (sm_count) *sm_count = sms;
    if (ctas_per_sm) *ctas_per_sm = occ;
    return PHS_OK;
}

int phs_engine_create(int precision, phs_engine** out) {
    if (!out || (precision != PHS_PREC_F32 && precision != PHS_PREC_F64)) return PHS_ERR_BAD_ARG;
    phs_engine* e = new phs_engine();
    e->prec = precision;
    cudaError_t ce = cudaGetDevice(&e->device);
    if (ce == cudaSuccess) ce = cudaDeviceGetAttribute(&e->sms, cudaDevAttrMultiProcessorCount, e->device);
    if (ce == cudaSuccess) ce = cudaMalloc(&e->abort_word, sizeof(unsigned int));
    if (ce == cudaSuccess) ce = cudaMemset(e->abort_word, 0, sizeof(unsigned int));
    if (ce != cudaSuccess) {
        set_last_error("phs_engine_create", ce);
        if (e->abort_word) cudaFree(e->abort_word);
        delete e;
        return PHS_ERR_CUDA;
    }
    *out = e;
    return PHS_OK;
}

int phs_engine_destroy(phs_engine* e) {
    if (!e) return PHS_ERR_BAD_ARG;
    cudaDeviceSynchronize();
    drop_graphs(e);
    for (auto& h : e->inst)
        if (h.used) free_inst(h);
    if (e->abort_word) cudaFree(e->abort_word);
    if (e->d_desc) cudaFree(e->d_desc);
    if (e->d_map) cudaFree(e->d_map);
    delete e;
    return PHS_OK;
}

int phs_instance_add(phs_engine* e, const phs_instance_desc* d, int* slot) {
    if (!e || !d || !slot) return PHS_ERR_BAD_ARG;
    return e->prec == PHS_PREC_F64 ? add_instance<double>(e, d, slot) : add_instance<float>(e, d, slot);
}

int phs_instance_remove(phs_engine* e, int slot) {
    if (!e || slot < 0 || slot >= (int)e->inst.size() || !e->inst[slot].used) return PHS_ERR_BAD_ARG;
    cudaDeviceSynchronize();
    free_inst(e->inst[slot]);
    e->dirty = true;
    e->auto_left = 2;
    e->auto_mark = e->launches;
    return PHS_OK;
}

int phs_instance_info_get(phs_engine* e, int slot, phs_instance_info* info) {
    if (!e || !info || slot < 0 || slot >= (int)e->inst.size() || !e->inst[slot].used) return PHS_ERR_BAD_ARG;
    InstHost& h = e->inst[slot];
    PHS_CUDA_TRY(cudaMemcpy(&h.st_host, h.st, sizeof(InstState), cudaMemcpyDeviceToHost));
    info->n_voxel = h.n;
    info->step = h.st_host.step;
    info->n_steps = h.d.n_steps;
    info->samples = h.st_host.id_save;
    info->status = h.st_host.status;
    info->arnoldi_steps = h.st_host.arnoldi;
    info->solves = h.st_host.solves;
    info->max_arnoldi = h.st_host.max_arnoldi;
    info->nonconverged = h.st_host.nonconv;
    info->arnoldi_sq = h.st_host.arnoldi_sq;
    return PHS_OK;
}

int phs_engine_advance(phs_engine* e, int64_t n_steps, int ctas_per_sm, void* stream, int sync) {
    if (!e || n_steps < 0) return PHS_ERR_BAD_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    return e->prec == PHS_PREC_F64 ? advance_impl<double>(e, n_steps, ctas_per_sm, s, sync != 0)
                                   : advance_impl<float>(e, n_steps, ctas_per_sm, s, sync != 0);
}

int phs_instance_read_history(phs_engine* e, int slot, int32_t s0, int32_t count, void* u_dst, void* h_dst) {
    if (!e || slot < 0 || slot >= (int)e->inst.size() || !e->inst[slot].used) return PHS_ERR_BAD_ARG;
    InstHost& h = e->inst[slot];
    if (s0 < 0 || count < 0 || s0 + count > h.d.n_samples) return PHS_ERR_BAD_ARG;
    const size_t es = (e->prec == PHS_PREC_F64) ? 8 : 4;
    const size_t off = (size_t)s0 * h.n * es, bytes = (size_t)count * h.n * es;
    PHS_CUDA_TRY(cudaDeviceSynchronize());
    if (u_dst && bytes) PHS_CUDA_TRY(cudaMemcpy(u_dst, (char*)h.hist_u + off, bytes, cudaMemcpyDeviceToHost));
    if (h_dst && bytes) {
        if (!h.hist_h) return PHS_ERR_STATE;
        PHS_CUDA_TRY(cudaMemcpy(h_dst, (char*)h.hist_h + off, bytes, cudaMemcpyDeviceToHost));
    }
    return PHS_OK;
}

int phs_instance_read_state(phs_engine* e, int slot, void* u_dst, void* h_dst, int32_t* lat_dst) {
    if (!e || slot < 0 || slot >= (int)e->inst.size() || !e->inst[slot].used) return PHS_ERR_BAD_ARG;
    InstHost& h = e->inst[slot];
    PHS_CUDA_TRY(cudaDeviceSynchronize());
    PHS_CUDA_TRY(cudaMemcpy(&h.st_host, h.st, sizeof(InstState), cudaMemcpyDeviceToHost));
    const size_t es = (e->prec == PHS_PREC_F64) ? 8 : 4;
    if (u_dst) PHS_CUDA_TRY(cudaMemcpy(u_dst, h.u, (size_t)h.n * es, cudaMemcpyDeviceToHost));
    if (h_dst) {
        const void* hc = h.st_host.hbuf ? h.h1 : h.h0;
        PHS_CUDA_TRY(cudaMemcpy(h_dst, hc, (size_t)h.n * es, cudaMemcpyDeviceToHost));
    }
    if (lat_dst) PHS_CUDA_TRY(cudaMemcpy(lat_dst, h.lat, (size_t)h.n * 4, cudaMemcpyDeviceToHost));
    return PHS_OK;
}

int phs_instance_device_ptrs(phs_engine* e, int slot, void** u, void** hist_u, int32_t** lat) {
    if (!e || slot < 0 || slot >= (int)e->inst.size() || !e->inst[slot].used) return PHS_ERR_BAD_ARG;
    InstHost& h = e->inst[slot];
    if (u) *u = h.u;
    if (hist_u) *hist_u = h.hist_u;
    if (lat) *lat = h.lat;
    return PHS_OK;
}

int64_t phs_engine_launch_count(phs_engine* e) { return e ? e->launches : -1; }

int phs_engine_rebalance(phs_engine* e) {
    if (!e) return PHS_ERR_BAD_ARG;
    PHS_CUDA_TRY(cudaDeviceSynchronize());
    for (auto& h : e->inst) {
        if (!h.used) continue;
        PHS_CUDA_TRY(cudaMemcpy(&h.st_host, h.st, sizeof(InstState), cudaMemcpyDeviceToHost));
        const long long ds = h.st_host.step - h.ref_step;
        if (ds > 0) h.kavg = (double)(h.st_host.arnoldi - h.ref_arnoldi) / (double)ds;
        h.ref_step = h.st_host.step;
        h.ref_arnoldi = h.st_host.arnoldi;
        // measured cost: the team's time per step times its CTAs
        h.weight = 0.0;
        if (h.prof) {
            unsigned long long pf[kProfSlots];
            PHS_CUDA_TRY(cudaMemcpy(pf, h.prof, sizeof(pf), cudaMemcpyDeviceToHost));
            const unsigned long long steps = pf[PF_STEPS] - h.prof_ref[PF_STEPS];
            unsigned long long ns = 0;
            for (int i = 0; i <= PF_RHS1; ++i) ns += pf[i] - h.prof_ref[i];
            if (steps > 0 && h.team > 0) h.weight = (double)ns / (double)steps * (double)h.team;
            for (int i = 0; i < kProfSlots; ++i) h.prof_ref[i] = pf[i];
        }
    }
    e->dirty = true;
    return PHS_OK;
}

int phs_instance_profile(phs_engine* e, int slot, uint64_t* out16) {
    if (!e || !out16 || slot < 0 || slot >= (int)e->inst.size() || !e->inst[slot].used) return PHS_ERR_BAD_ARG;
    InstHost& h = e->inst[slot];
    if (!h.prof) return PHS_ERR_STATE;
    PHS_CUDA_TRY(cudaDeviceSynchronize());
    PHS_CUDA_TRY(cudaMemcpy(out16, h.prof, kProfSlots * sizeof(uint64_t), cudaMemcpyDeviceToHost));
    return PHS_OK;
}

int phs_instance_table_bytes(phs_engine* e, int slot, int32_t* bytes_per_voxel) {
    if (!e || !bytes_per_voxel || slot < 0 || slot >= (int)e->inst.size() || !e->inst[slot].used)
        return PHS_ERR_BAD_ARG;
    *bytes_per_voxel = (e->compact_nb && e->inst[slot].nbr) ? 8 : 24;
    return PHS_OK;
}

int phs_step_variants(int precision, int32_t* count, int32_t* min_ctas_per_sm, int32_t* max_regs) {
    if (precision != PHS_PREC_F32 && precision != PHS_PREC_F64) return PHS_ERR_BAD_ARG;
    const int nv = precision == PHS_PREC_F64 ? kNumF64 : kNumF32;
    if (count) *count = nv;
    for (int v = 0; v < nv; ++v) {
        if (min_ctas_per_sm) min_ctas_per_sm[v] = precision == PHS_PREC_F64 ? kMinbF64[v] : kMinbF32[v];
        if (max_regs) {
            cudaFuncAttributes a{};
            const void* fn = precision == PHS_PREC_F64 ? step_fn<double>(v) : step_fn<float>(v);
            max_regs[v] = (cudaFuncGetAttributes(&a, fn) == cudaSuccess) ? a.numRegs : -1;
        }
    }
    return PHS_OK;
}

namespace {
// Phase timers on or off for every instance (counters reset).
int set_profile(phs_engine* e, bool on) {
    cudaDeviceSynchronize();
    e->profile = on;
    for (auto& h : e->inst) {
        if (!h.used) continue;
        if (e->profile && !h.prof) {
            if (cudaMalloc((void**)&h.prof, kProfSlots * sizeof(unsigned long long)) != cudaSuccess)
                return PHS_ERR_OOM;
        }
        if (h.prof) cudaMemset(h.prof, 0, kProfSlots * sizeof(unsigned long long));
        if (!e->profile && h.prof) { cudaFree(h.prof); h.prof = nullptr; }
        for (int i = 0; i < kProfSlots; ++i) h.prof_ref[i] = 0;
    }
    e->dirty = true;
    return PHS_OK;
}
}  // namespace

int phs_step_variant_vpt(int precision, int32_t count, int32_t* vpt) {
    if (precision != PHS_PREC_F32 && precision != PHS_PREC_F64) return PHS_ERR_BAD_ARG;
    const int nv = precision == PHS_PREC_F64 ? kNumF64 : kNumF32;
    if (count < nv || !vpt) return PHS_ERR_BAD_ARG;
    for (int v = 0; v < nv; ++v) vpt[v] = precision == PHS_PREC_F64 ? kVptF64 : kVptOfF32[v];
    return PHS_OK;
}

int phs_step_variant_layout(int precision, int32_t count, int32_t* ring_bytes, int32_t* compact_table) {
    if (precision != PHS_PREC_F32 && precision != PHS_PREC_F64) return PHS_ERR_BAD_ARG;
    const int nv = precision == PHS_PREC_F64 ? kNumF64 : kNumF32;
    if (count < nv) return PHS_ERR_BAD_ARG;
    for (int v = 0; v < nv; ++v) {
        const bool f32 = precision == PHS_PREC_F32;
        if (ring_bytes) ring_bytes[v] = f32 ? kRingF32[v] : 0;
        // staged variants read the compact table of every instance that has one
        if (compact_table) compact_table[v] = (f32 && (kTwinF32[v] >= 0 || kRingF32[v] > 0)) ? 1 : 0;
    }
    return PHS_OK;
}

int phs_engine_config(phs_engine* e, int key, int64_t value) {
    if (!e) return PHS_ERR_BAD_ARG;
    switch (key) {
        case PHS_CFG_VARIANT: {
            const int nv = e->prec == PHS_PREC_F64 ? kNumF64 : kNumF32;
            if (value < -1 || value >= nv) return PHS_ERR_BAD_ARG;
            if (e->variant != (int)value) {
                e->variant = (int)value;
                e->dirty = true;
            }
            return PHS_OK;
        }
        case PHS_CFG_CTAS_PER_SM:
            if (value < 0 || value > 32) return PHS_ERR_BAD_ARG;
            e->default_cps = (int)value;
            return PHS_OK;
        case PHS_CFG_AUTO_BALANCE:
            e->auto_balance = value != 0;
            return PHS_OK;
        case PHS_CFG_TEST_TEAM_OVERCOUNT:
            e->test_overcount = value != 0;
            e->dirty = true;
            return PHS_OK;
        case PHS_CFG_PROFILE:
            // the caller's setting wins over the automatic balancing's
            e->auto_prof = false;
            return set_profile(e, value != 0);
        case PHS_CFG_GROUP_SUMS:
            if (e->group_sums != (value != 0)) {
                e->group_sums = value != 0;
                e->dirty = true;
            }
            return PHS_OK;
        case PHS_CFG_COMPACT_NB:
            if (e->compact_nb != (value != 0)) {
                e->compact_nb = value != 0;
                e->dirty = true;
            }
            return PHS_OK;
        case PHS_CFG_WAVE_INSTANCES:
            if (value < 0 || value > (1 << 20)) return PHS_ERR_BAD_ARG;
            if (e->wave_instances != (int)value) {
                e->wave_instances = (int)value;
                e->dirty = true;
            }
            return PHS_OK;
        default:
            return PHS_ERR_BAD_ARG;
    }
}

int phs_simulate(const phs_instance_desc* desc, int precision, void* u_hist, void* h_hist, int32_t* lat,
                 int32_t* n_saved, phs_instance_info* info) {
    if (!desc) return PHS_ERR_BAD_ARG;
    phs_engine* e = nullptr;
    int rc = phs_engine_create(precision, &e);
    if (rc != PHS_OK) return rc;
    int slot = -1;
    rc = phs_instance_add(e, desc, &slot);
    if (rc != PHS_OK) { phs_engine_destroy(e); return rc; }
    // bounded launches keep each kernel short
    const long long chunk = 2000;
    int worst = PHS_OK;
    for (long long done = 0; done < desc->n_steps; done += chunk) {
        rc = phs_engine_advance(e, chunk, 0, nullptr, 1);
        if (rc == PHS_WARN_NO_CONVERGE) worst = rc;
        else if (rc != PHS_OK) { phs_engine_destroy(e); return rc; }
    }
    phs_instance_info inf{};
    rc = phs_instance_info_get(e, slot, &inf);
    if (rc == PHS_OK && n_saved) *n_saved = inf.samples;
    if (rc == PHS_OK && inf.samples > 0 && (u_hist || h_hist))
        rc = phs_instance_read_history(e, slot, 0, inf.samples, u_hist, desc->save_h ? h_hist : nullptr);
    if (rc == PHS_OK && lat) rc = phs_instance_read_state(e, slot, nullptr, nullptr, lat);
    if (info) *info = inf;
    phs_engine_destroy(e);
    if (rc != PHS_OK) return rc;
    if (inf.status == PHS_ERR_NONFINITE) return PHS_ERR_NONFINITE;
    return worst != PHS_OK ? worst : inf.status;
}

}  // extern "C"
