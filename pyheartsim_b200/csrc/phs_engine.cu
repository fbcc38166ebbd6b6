// Time-stepping engine of the PyHeartSim B200 path.
//
// One persistent kernel advances every active simulation instance.  Each
// instance is owned by a "team" of CTAs that synchronise with their own bounded
// barrier, so instances of different sizes progress independently inside one
// launch.  Per step and instance:
//
//   RHS phase   fused RK4 reaction (simulation/simulation_gpu.py:27-43, 71-130)
//               evaluated in registers for the voxel and its six neighbours, fed
//               straight into the Crank-Nicolson right-hand side
//               b = u* + dt/2 L u*  (simulation/simulation_gpu.py:245) and the
//               initial residual r0 = b - A u*  (A = I - dt/2 L, :321-322)
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
};

template <typename T>
struct InstDev {
    const int32_t* nb;      // [n*6]
    const T* coef;          // [n*6]
    const uint8_t* vflags;  // [n]
    const T* vparams;       // [n*5] or nullptr
    const uint8_t* stim;    // [n_steps]
    T* u;
    T* h0;
    T* h1;
    T* x;
    T* b;
    T* V;                   // [(m+1)*n]
    T* hist_u;              // [S*n]
    T* hist_h;              // [S*n] or nullptr
    int32_t* lat;           // [n]
    double* part;           // [n_tiles*kSlots]
    Scalars* sc;
    TeamSync* sync;
    InstState* st;
    T params[5];
    T dt, half_dt, jmag;
    double tol, atol;
    long long n;
    long long n_steps;
    long long tb_steps;
    int n_tiles;
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

// Classical RK4 with J held over the step, simulation/simulation_gpu.py:71-130.
template <typename T>
__device__ __forceinline__ void rk4(int model, T u, T h, T J, const T* p, T dt, T& us, T& hs) {
    T k1u, k1h, k2u, k2h, k3u, k3h, k4u, k4h;
    reaction(model, u, h, J, p, k1u, k1h);
    T ut = u + T(0.5) * dt * k1u;
    T ht = h + T(0.5) * dt * k1h;
    reaction(model, ut, ht, J, p, k2u, k2h);
    ut = u + T(0.5) * dt * k2u;
    ht = h + T(0.5) * dt * k2h;
    reaction(model, ut, ht, J, p, k3u, k3h);
    ut = u + dt * k3u;
    ht = h + dt * k3h;
    reaction(model, ut, ht, J, p, k4u, k4h);
    us = u + (dt / T(6)) * (k1u + T(2) * k2u + T(2) * k3u + k4u);
    hs = h + (dt / T(6)) * (k1h + T(2) * k2h + T(2) * k3h + k4h);
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
template <typename Leader>
__device__ __forceinline__ bool team_sync(TeamSync* ts, int P, unsigned int* abort_word, SharedCtl& ctl,
                                          Leader&& leader) {
    __syncthreads();
    if (threadIdx.x == 0) {
        cuda::atomic_ref<unsigned int, cuda::thread_scope_device> gen(ts->gen);
        cuda::atomic_ref<unsigned int, cuda::thread_scope_device> cnt(ts->count);
        unsigned int g = gen.load(cuda::memory_order_relaxed);
        __threadfence();
        unsigned int a = cnt.fetch_add(1u, cuda::memory_order_acq_rel);
        ctl.last = (a == (unsigned int)(P - 1));
        ctl.gen = g;
        ctl.abort = 0;
        if (ctl.last) __threadfence();
    }
    __syncthreads();
    if (ctl.last) {
        leader();
        __syncthreads();
        if (threadIdx.x == 0) {
            cuda::atomic_ref<unsigned int, cuda::thread_scope_device> gen(ts->gen);
            cuda::atomic_ref<unsigned int, cuda::thread_scope_device> cnt(ts->count);
            cnt.store(0u, cuda::memory_order_relaxed);
            __threadfence();
            gen.store(ctl.gen + 1u, cuda::memory_order_release);
        }
    } else if (threadIdx.x == 0) {
        cuda::atomic_ref<unsigned int, cuda::thread_scope_device> gen(ts->gen);
        cuda::atomic_ref<unsigned int, cuda::thread_scope_device> ab(*abort_word);
        unsigned long long t0 = global_ns();
        unsigned int polls = 0;
        while (gen.load(cuda::memory_order_acquire) == ctl.gen) {
            if (ab.load(cuda::memory_order_relaxed) != 0u) { ctl.abort = 1; break; }
            if (++polls > kWaitPolls || global_ns() - t0 > kWaitNs) {
                ab.fetch_or(1u, cuda::memory_order_relaxed);
                ctl.abort = 1;
                break;
            }
            __nanosleep(64);
        }
        __threadfence();
    }
    __syncthreads();
    return ctl.abort == 0;
}

// Leader helper: sum slot `slot` over all tiles in tile order (deterministic).
// Called by one warp; returns the sum in every lane.
__device__ __forceinline__ double tile_sum(const double* part, int n_tiles, int slot) {
    const int lane = threadIdx.x & 31;
    double acc = 0.0;
    for (int t = lane; t < n_tiles; t += 32) acc += __ldcg(part + (size_t)t * kSlots + slot);
    return warp_sum(acc);
}

// ------------------------------------------------------------------ the kernel
template <typename T, int VPT>
__global__ void __launch_bounds__(kThreads)
step_kernel(const InstDev<T>* __restrict__ insts, const int4* __restrict__ cta_map,
            long long n_steps_launch, unsigned int* abort_word) {
    constexpr int TILE = kThreads * VPT;
    const int4 cm = cta_map[blockIdx.x];
    const int rank = cm.y;
    const int P = cm.z;

    __shared__ InstDev<T> I;
    __shared__ SharedCtl ctl;
    __shared__ double red[kWarps][kSlots];
    __shared__ double shc[kMaxRestart + 1];
    __shared__ long long sh_step0;
    __shared__ int sh_id_save, sh_pending, sh_hbuf, sh_status;

    if (threadIdx.x == 0) {
        I = insts[cm.x];
        sh_step0 = __ldcg(&I.st->step);
        sh_id_save = __ldcg(&I.st->id_save);
        sh_pending = __ldcg(&I.st->pending);
        sh_hbuf = __ldcg(&I.st->hbuf);
        sh_status = __ldcg(&I.st->status);
    }
    __syncthreads();

    const long long N = I.n;
    const int m = I.m;
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

    // ---- tile partial writer: threads 0..nslot-1 sum the kWarps warp partials
    auto write_partials = [&](int tile, int nslot) {
        __syncthreads();
        for (int t = threadIdx.x; t < nslot; t += kThreads) {
            double s = 0.0;
#pragma unroll
            for (int w = 0; w < kWarps; ++w) s += red[w][t];
            I.part[(size_t)tile * kSlots + t] = s;
        }
        __syncthreads();
    };

    // ---- stencil of a vector at voxel n (matrix-free row of L)
    auto lap_at = [&](const T* vec, long long n, T vn, bool rowzero) -> T {
        T acc = T(0);
        if (!rowzero) {
            const int32_t* nbp = I.nb + 6 * n;
            const T* cp = I.coef + 6 * n;
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                T c = cp[k];
                if (c != T(0)) acc += c * (vec[nbp[k]] - vn);
            }
        }
        return acc;
    };

    auto params_of = [&](long long n, T* p) {
        if (I.vparams) {
#pragma unroll
            for (int q = 0; q < 5; ++q) p[q] = I.vparams[5 * n + q];
        } else {
#pragma unroll
            for (int q = 0; q < 5; ++q) p[q] = I.params[q];
        }
    };

    // ---- leader bodies ------------------------------------------------------
    auto leader_rhs = [&]() {
        if (warp == 0) {
            double b2 = tile_sum(I.part, I.n_tiles, 0);
            double r2 = tile_sum(I.part, I.n_tiles, 1);
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
        // h_ij = s_i * sum_tiles <V_i, w>;  published coef_i = h_ij * s_i
        for (int i = warp; i <= j; i += kWarps) {
            double d = tile_sum(I.part, I.n_tiles, i);
            if (lane == 0) {
                double si = sc->s[i];
                double h = si * d;
                sc->R[j * (kMaxRestart + 1) + i] = h;
                sc->coef[i] = h * si;
            }
        }
    };

    auto leader_norm = [&](int j) {
        if (warp == 0) {
            double u2 = tile_sum(I.part, I.n_tiles, 0);
            if (lane == 0) {
                double* Rc = sc->R + j * (kMaxRestart + 1);
                double hn = sqrt(u2);
                Rc[j + 1] = hn;
                // apply the previous rotations to column j
                for (int i = 0; i < j; ++i) {
                    double c = sc->cs[i], s = sc->sn[i];
                    double a = Rc[i], bb = Rc[i + 1];
                    Rc[i] = c * a + s * bb;
                    Rc[i + 1] = -s * a + c * bb;
                }
                double a = Rc[j], bb = Rc[j + 1];
                double r = hypot(a, bb);
                double c = (r == 0.0) ? 1.0 : a / r;
                double s = (r == 0.0) ? 0.0 : bb / r;
                sc->cs[j] = c;
                sc->sn[j] = s;
                Rc[j] = r;
                Rc[j + 1] = 0.0;
                double gj = sc->g[j];
                sc->g[j] = c * gj;
                sc->g[j + 1] = -s * gj;
                double est = fabs(sc->g[j + 1]);
                sc->est = est;
                sc->iters_solve += 1;
                int act;
                bool finite = isfinite(hn) && isfinite(r);
                bool breakdown = (hn == 0.0);
                bool conv = (!I.full_cycles) && (est <= sc->atol_eff);
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
                sc->action = act;
            }
        }
        __syncthreads();
        // back substitution R y = g (k x k upper triangular), one warp
        if (warp == 0) {
            int act = sc->action;
            if (act == ACT_UPDATE_FINAL || act == ACT_UPDATE_CHECK) {
                int k = sc->k;
                for (int i = k - 1; i >= 0; --i) {
                    double acc = 0.0;
                    for (int l = i + 1 + lane; l < k; l += 32)
                        acc += sc->R[l * (kMaxRestart + 1) + i] * sc->coef[l];
                    acc = warp_sum(acc);
                    if (lane == 0) sc->coef[i] = (sc->g[i] - acc) / sc->R[i * (kMaxRestart + 1) + i];
                    __syncwarp();
                }
                __syncwarp();
                // scale: x += sum_j y_j v_j = sum_j (y_j s_j) V_j
                for (int i = lane; i < k; i += 32) sc->coef[i] *= sc->s[i];
            }
        }
    };

    auto leader_check = [&]() {
        if (warp == 0) {
            double r2 = tile_sum(I.part, I.n_tiles, 0);
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
                } else if (sc->iters_cap >= I.maxiter) {
                    act = ACT_DONE;
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

    auto leader_solve_stats = [&]() {
        if (threadIdx.x == 0) {
            int it = sc->iters_solve;
            if (it > 0) {
                I.st->arnoldi += it;
                I.st->solves += 1;
                if (it > I.st->max_arnoldi) I.st->max_arnoldi = it;
            }
        }
    };

    auto read_action = [&]() {
        if (threadIdx.x == 0) {
            ctl.action = __ldcg(&sc->action);
            ctl.k = __ldcg(&sc->k);
        }
        __syncthreads();
        return ctl.action;
    };

    auto load_coef = [&](int cnt) {
        for (int i = threadIdx.x; i < cnt; i += kThreads) shc[i] = __ldcg(sc->coef + i);
        __syncthreads();
    };

    // ---- sample / activation bookkeeping of the state in u (after step s-1)
    auto sample_voxel = [&](long long n, T un, T hn, long long done_step) {
        if (pending >= 0) {
            I.hist_u[(size_t)pending * N + n] = un;
            if (I.save_h) I.hist_h[(size_t)pending * N + n] = hn;
        }
        if (done_step >= 0 && I.lat[n] < 0 && un >= T(0.5)) I.lat[n] = (int32_t)done_step;
    };

    T* Vb = I.V;
    const size_t ldV = (size_t)N;

    for (; step < step_end && !retired && !aborted; ++step) {
        const uint8_t stim_bits = I.stim[step];
        const bool tb = step < I.tb_steps;
        const T* hin = hbuf ? I.h1 : I.h0;
        T* hout = hbuf ? I.h0 : I.h1;

        // ================= RHS phase: fused RK4 + b + r0
        for (int tile = rank; tile < I.n_tiles; tile += P) {
            double ab = 0.0, ar = 0.0;
#pragma unroll
            for (int v = 0; v < VPT; ++v) {
                long long n = (long long)tile * TILE + v * kThreads + threadIdx.x;
                if (n < N) {
                    T un = I.u[n], hn = hin[n];
                    sample_voxel(n, un, hn, step - 1);
                    uint8_t f = I.vflags[n];
                    T p[5];
                    params_of(n, p);
                    T J = (f & stim_bits & 3u) ? I.jmag : T(0);
                    T us, hs;
                    rk4(I.model, un, hn, J, p, I.dt, us, hs);
                    I.x[n] = us;
                    hout[n] = hs;
                    T lap = T(0);
                    if (!(tb && (f & PHS_VFLAG_TBLOCK))) {
                        const int32_t* nbp = I.nb + 6 * n;
                        const T* cp = I.coef + 6 * n;
#pragma unroll 1
                        for (int k = 0; k < 6; ++k) {
                            T c = cp[k];
                            if (c != T(0)) {
                                int32_t q = nbp[k];
                                T pq[5];
                                params_of(q, pq);
                                T Jq = (I.vflags[q] & stim_bits & 3u) ? I.jmag : T(0);
                                T usq, hsq;
                                rk4(I.model, I.u[q], hin[q], Jq, pq, I.dt, usq, hsq);
                                lap += c * (usq - us);
                            }
                        }
                    }
                    T bn = us + I.half_dt * lap;
                    T ax = us - I.half_dt * lap;
                    T rn = bn - ax;
                    I.b[n] = bn;
                    Vb[n] = rn;
                    ab += (double)bn * (double)bn;
                    ar += (double)rn * (double)rn;
                }
            }
            ab = warp_sum(ab);
            ar = warp_sum(ar);
            if (lane == 0) { red[warp][0] = ab; red[warp][1] = ar; }
            write_partials(tile, 2);
        }
        pending = -1;
        if (!team_sync(I.sync, P, abort_word, ctl, leader_rhs)) { aborted = true; break; }
        int act = read_action();

        if (act == ACT_CYCLE) {
            bool leave_solve = false;
            while (!leave_solve) {
                int j = 0;
                for (;;) {
                    // ============ phase A: w = A (s_j V_j) -> V_{j+1}; dots <V_i, w>
                    if (threadIdx.x == 0) ctl.sj = __ldcg(&sc->s[j]);
                    __syncthreads();
                    const T sj = (T)ctl.sj;
                    const T* Vj = Vb + (size_t)j * ldV;
                    T* Vn = Vb + (size_t)(j + 1) * ldV;
                    for (int tile = rank; tile < I.n_tiles; tile += P) {
                        T wr[VPT];
#pragma unroll
                        for (int v = 0; v < VPT; ++v) {
                            long long n = (long long)tile * TILE + v * kThreads + threadIdx.x;
                            wr[v] = T(0);
                            if (n < N) {
                                T vj = Vj[n];
                                bool rz = tb && (I.vflags[n] & PHS_VFLAG_TBLOCK);
                                T lap = lap_at(Vj, n, vj, rz);
                                T w = sj * (vj - I.half_dt * lap);
                                Vn[n] = w;
                                wr[v] = w;
                            }
                        }
                        for (int i = 0; i <= j; ++i) {
                            const T* Vi = Vb + (size_t)i * ldV;
                            double d = 0.0;
#pragma unroll
                            for (int v = 0; v < VPT; ++v) {
                                long long n = (long long)tile * TILE + v * kThreads + threadIdx.x;
                                if (n < N) d += (double)Vi[n] * (double)wr[v];
                            }
                            d = warp_sum(d);
                            if (lane == 0) red[warp][i] = d;
                        }
                        write_partials(tile, j + 1);
                    }
                    if (!team_sync(I.sync, P, abort_word, ctl, [&]() { leader_dots(j); })) { aborted = true; break; }
                    load_coef(j + 1);
                    // ============ phase C: u = w - sum_i c_i V_i  (in place), ||u||^2
                    for (int tile = rank; tile < I.n_tiles; tile += P) {
                        double a2 = 0.0;
#pragma unroll
                        for (int v = 0; v < VPT; ++v) {
                            long long n = (long long)tile * TILE + v * kThreads + threadIdx.x;
                            if (n < N) {
                                double uu = (double)Vn[n];
                                for (int i = 0; i <= j; ++i) uu -= shc[i] * (double)Vb[(size_t)i * ldV + n];
                                T ut = (T)uu;
                                Vn[n] = ut;
                                a2 += (double)ut * (double)ut;
                            }
                        }
                        a2 = warp_sum(a2);
                        if (lane == 0) red[warp][0] = a2;
                        write_partials(tile, 1);
                    }
                    if (!team_sync(I.sync, P, abort_word, ctl, [&]() { leader_norm(j); })) { aborted = true; break; }
                    act = read_action();
                    if (act != ACT_NEXT_J) break;
                    ++j;
                }
                if (aborted) break;
                if (act == ACT_FAIL) { retired = true; break; }
                // ============ phase X: x += sum_j c_j V_j
                const int k = ctl.k;
                load_coef(k);
                const bool final = (act == ACT_UPDATE_FINAL);
                for (int tile = rank; tile < I.n_tiles; tile += P) {
#pragma unroll
                    for (int v = 0; v < VPT; ++v) {
                        long long n = (long long)tile * TILE + v * kThreads + threadIdx.x;
                        if (n < N) {
                            double xv = (double)I.x[n];
                            for (int jj = 0; jj < k; ++jj) xv += shc[jj] * (double)Vb[(size_t)jj * ldV + n];
                            if (final) I.u[n] = (T)xv;
                            else I.x[n] = (T)xv;
                        }
                    }
                }
                if (final) break;
                // ============ true residual of the new iterate (start of the next cycle)
                if (!team_sync(I.sync, P, abort_word, ctl, [&]() {})) { aborted = true; break; }
                for (int tile = rank; tile < I.n_tiles; tile += P) {
                    double a2 = 0.0;
#pragma unroll
                    for (int v = 0; v < VPT; ++v) {
                        long long n = (long long)tile * TILE + v * kThreads + threadIdx.x;
                        if (n < N) {
                            T xv = I.x[n];
                            bool rz = tb && (I.vflags[n] & PHS_VFLAG_TBLOCK);
                            T lap = lap_at(I.x, n, xv, rz);
                            T ax = xv - I.half_dt * lap;
                            T r = I.b[n] - ax;
                            Vb[n] = r;
                            I.u[n] = xv;
                            a2 += (double)r * (double)r;
                        }
                    }
                    a2 = warp_sum(a2);
                    if (lane == 0) red[warp][0] = a2;
                    write_partials(tile, 1);
                }
                if (!team_sync(I.sync, P, abort_word, ctl, leader_check)) { aborted = true; break; }
                act = read_action();
                if (act == ACT_DONE) break;
                if (act == ACT_FAIL) { retired = true; break; }
                // ACT_CYCLE: V0 holds the new residual
            }
            if (aborted || retired) break;
        } else if (act == ACT_ZERO_B || act == ACT_DONE) {
            const T* src = (act == ACT_ZERO_B) ? I.b : I.x;
            for (int tile = rank; tile < I.n_tiles; tile += P) {
#pragma unroll
                for (int v = 0; v < VPT; ++v) {
                    long long n = (long long)tile * TILE + v * kThreads + threadIdx.x;
                    if (n < N) I.u[n] = src[n];
                }
            }
        } else {  // ACT_FAIL
            retired = true;
            break;
        }
        // end of step: u visible to every CTA of the team; solve statistics
        if (!team_sync(I.sync, P, abort_word, ctl, leader_solve_stats)) { aborted = true; break; }
        hbuf ^= 1;
        const bool due = (I.stride > 0) ? (step % I.stride == 0) : true;
        if (due && id_save < I.n_samples) pending = id_save++;
    }

    // flush the sample and activation test of the last completed step
    if (!aborted && !retired) {
        const T* hcur = hbuf ? I.h1 : I.h0;
        if (pending >= 0 || step > sh_step0) {
            for (int tile = rank; tile < I.n_tiles; tile += P) {
#pragma unroll
                for (int v = 0; v < VPT; ++v) {
                    long long n = (long long)tile * TILE + v * kThreads + threadIdx.x;
                    if (n < N) sample_voxel(n, I.u[n], hcur[n], step - 1);
                }
            }
        }
        pending = -1;
    }
    if (!aborted) {
        if (!team_sync(I.sync, P, abort_word, ctl, [&]() {
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
constexpr int kVptF64 = 1;

struct InstHost {
    bool used = false;
    bool finished = false;
    phs_instance_desc d{};
    long long n = 0;
    int n_tiles = 0;
    int m = 0;
    void* nb = nullptr;
    void* coef = nullptr;
    void* vflags = nullptr;
    void* vparams = nullptr;
    void* stim = nullptr;
    void* u = nullptr;
    void* h0 = nullptr;
    void* h1 = nullptr;
    void* x = nullptr;
    void* b = nullptr;
    void* V = nullptr;
    void* hist_u = nullptr;
    void* hist_h = nullptr;
    int32_t* lat = nullptr;
    double* part = nullptr;
    Scalars* sc = nullptr;
    TeamSync* sync = nullptr;
    InstState* st = nullptr;
    InstState st_host{};
};

void free_inst(InstHost& h) {
    void* ptrs[] = {h.nb, h.coef, h.vflags, h.vparams, h.stim, h.u, h.h0, h.h1, h.x, h.b, h.V,
                    h.hist_u, h.hist_h, h.lat, h.part, h.sc, h.sync, h.st};
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
};

namespace {

template <typename T>
int occupancy_for(int* ctas) {
    int vpt = sizeof(T) == 8 ? kVptF64 : kVptF32;
    cudaError_t e;
    if (vpt == 1)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, step_kernel<T, 1>, kThreads, 0);
    else
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, step_kernel<T, kVptF32>, kThreads, 0);
    if (e != cudaSuccess) { set_last_error("occupancy", e); return PHS_ERR_CUDA; }
    return PHS_OK;
}

template <typename T>
void fill_dev(T* p, long long n, T v, cudaStream_t s) {
    if (n <= 0) return;
    long long blocks = std::min<long long>((n + 255) / 256, 65535);
    fill_kernel<T><<<(unsigned)blocks, 256, 0, s>>>(p, n, v);
}

template <typename T>
int upload_converted(void** dst, const double* src, long long n) {
    PHS_CUDA_TRY(cudaMalloc(dst, (size_t)n * sizeof(T)));
    if (sizeof(T) == 8) {
        PHS_CUDA_TRY(cudaMemcpy(*dst, src, (size_t)n * 8, cudaMemcpyHostToDevice));
        return PHS_OK;
    }
    double* tmp = nullptr;
    PHS_CUDA_TRY(cudaMalloc(&tmp, (size_t)n * 8));
    cudaError_t e = cudaMemcpy(tmp, src, (size_t)n * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        long long blocks = std::min<long long>((n + 255) / 256, 65535);
        convert_kernel<T><<<(unsigned)std::max<long long>(blocks, 1), 256>>>(tmp, (T*)*dst, n);
        e = cudaDeviceSynchronize();
    }
    cudaFree(tmp);
    if (e != cudaSuccess) { set_last_error("upload_converted", e); return PHS_ERR_CUDA; }
    return PHS_OK;
}

int validate_desc(const phs_instance_desc* d) {
    if (!d || d->n_voxel <= 0 || d->n_voxel > (1ll << 31) - 1) return PHS_ERR_BAD_ARG;
    if (d->model != PHS_MODEL_MS && d->model != PHS_MODEL_AP) return PHS_ERR_BAD_ARG;
    if (d->restart < 1 || d->restart > kMaxRestart) return PHS_ERR_BAD_ARG;
    if (!d->nb6 || !d->coef6 || !d->vflags) return PHS_ERR_BAD_ARG;
    if (d->n_steps < 0 || (d->n_steps > 0 && !d->stim)) return PHS_ERR_BAD_ARG;
    if (d->n_samples < 0 || d->sample_stride < 0 || d->maxiter < 1) return PHS_ERR_BAD_ARG;
    if (!(d->dt > 0.0)) return PHS_ERR_BAD_ARG;
    const long long n = d->n_voxel;
    for (long long i = 0; i < 6 * n; ++i) {
        int32_t q = d->nb6[i];
        if (q < 0 || q >= n) return PHS_ERR_BAD_TABLE;
        if (!std::isfinite(d->coef6[i])) return PHS_ERR_BAD_TABLE;
    }
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
    const int vpt = sizeof(T) == 8 ? kVptF64 : kVptF32;
    const long long tile = (long long)kThreads * vpt;
    h.n_tiles = (int)((h.n + tile - 1) / tile);
    h.m = (int)std::min<long long>(d->restart, h.n);
    const size_t n = (size_t)h.n;
    auto fail = [&](int code) { free_inst(h); return code; };
#define PHS_ALLOC(ptr, bytes)                                            \
    do {                                                                 \
        cudaError_t _e = cudaMalloc((void**)&(ptr), (bytes));            \
        if (_e != cudaSuccess) { set_last_error("cudaMalloc", _e); return fail(PHS_ERR_OOM); } \
    } while (0)
    PHS_ALLOC(h.nb, n * 6 * sizeof(int32_t));
    if (cudaMemcpy(h.nb, d->nb6, n * 6 * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess) return fail(PHS_ERR_CUDA);
    if ((rc = upload_converted<T>(&h.coef, d->coef6, (long long)n * 6)) != PHS_OK) return fail(rc);
    PHS_ALLOC(h.vflags, n);
    if (cudaMemcpy(h.vflags, d->vflags, n, cudaMemcpyHostToDevice) != cudaSuccess) return fail(PHS_ERR_CUDA);
    if (d->vparams) {
        if ((rc = upload_converted<T>(&h.vparams, d->vparams, (long long)n * 5)) != PHS_OK) return fail(rc);
    }
    const size_t ns = (size_t)std::max<int64_t>(d->n_steps, 1);
    PHS_ALLOC(h.stim, ns);
    if (d->n_steps > 0) {
        if (cudaMemcpy(h.stim, d->stim, (size_t)d->n_steps, cudaMemcpyHostToDevice) != cudaSuccess) return fail(PHS_ERR_CUDA);
    } else {
        cudaMemset(h.stim, 0, ns);
    }
    PHS_ALLOC(h.u, n * sizeof(T));
    PHS_ALLOC(h.h0, n * sizeof(T));
    PHS_ALLOC(h.h1, n * sizeof(T));
    PHS_ALLOC(h.x, n * sizeof(T));
    PHS_ALLOC(h.b, n * sizeof(T));
    PHS_ALLOC(h.V, n * (size_t)(h.m + 1) * sizeof(T));
    const size_t S = (size_t)std::max(d->n_samples, 1);
    PHS_ALLOC(h.hist_u, S * n * sizeof(T));
    if (d->save_h) PHS_ALLOC(h.hist_h, S * n * sizeof(T));
    PHS_ALLOC(h.lat, n * sizeof(int32_t));
    PHS_ALLOC(h.part, (size_t)h.n_tiles * kSlots * sizeof(double));
    PHS_ALLOC(h.sc, sizeof(Scalars));
    PHS_ALLOC(h.sync, sizeof(TeamSync));
    PHS_ALLOC(h.st, sizeof(InstState));
#undef PHS_ALLOC
    fill_dev<T>((T*)h.u, (long long)n, (T)d->u0, 0);
    fill_dev<T>((T*)h.h0, (long long)n, (T)d->h0, 0);
    fill_dev<T>((T*)h.h1, (long long)n, (T)d->h0, 0);
    fill_dev<T>((T*)h.x, (long long)n, (T)0, 0);
    fill_dev<T>((T*)h.b, (long long)n, (T)0, 0);
    cudaMemset(h.V, 0, n * (size_t)(h.m + 1) * sizeof(T));
    cudaMemset(h.hist_u, 0, S * n * sizeof(T));
    if (h.hist_h) cudaMemset(h.hist_h, 0, S * n * sizeof(T));
    cudaMemset(h.lat, 0xff, n * sizeof(int32_t));
    cudaMemset(h.part, 0, (size_t)h.n_tiles * kSlots * sizeof(double));
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
    e->inst[s] = h;
    *slot = s;
    return PHS_OK;
}

template <typename T>
InstDev<T> make_dev(const InstHost& h) {
    InstDev<T> I{};
    I.nb = (const int32_t*)h.nb;
    I.coef = (const T*)h.coef;
    I.vflags = (const uint8_t*)h.vflags;
    I.vparams = (const T*)h.vparams;
    I.stim = (const uint8_t*)h.stim;
    I.u = (T*)h.u;
    I.h0 = (T*)h.h0;
    I.h1 = (T*)h.h1;
    I.x = (T*)h.x;
    I.b = (T*)h.b;
    I.V = (T*)h.V;
    I.hist_u = (T*)h.hist_u;
    I.hist_h = (T*)h.hist_h;
    I.lat = h.lat;
    I.part = h.part;
    I.sc = h.sc;
    I.sync = h.sync;
    I.st = h.st;
    for (int q = 0; q < 5; ++q) I.params[q] = (T)h.d.params[q];
    I.dt = (T)h.d.dt;
    I.half_dt = (T)h.d.dt / T(2);
    I.jmag = (T)h.d.j_stim;
    I.tol = h.d.tol;
    I.atol = h.d.atol;
    I.n = h.n;
    I.n_steps = h.d.n_steps;
    I.tb_steps = h.d.tblock_steps;
    I.n_tiles = h.n_tiles;
    I.model = h.d.model;
    I.m = h.m;
    I.maxiter = h.d.maxiter;
    I.full_cycles = h.d.full_cycles;
    I.stride = h.d.sample_stride;
    I.n_samples = h.d.n_samples;
    I.save_h = h.d.save_h;
    return I;
}

// Split G CTAs over the instances in proportion to their tiles (at least one
// CTA each, never more CTAs than tiles).
std::vector<int> team_sizes(const std::vector<int>& tiles, int G) {
    const int A = (int)tiles.size();
    std::vector<int> P(A, 1);
    long long total = 0;
    for (int t : tiles) total += t;
    int used = A;
    for (int i = 0; i < A; ++i) {
        long long want = (long long)((double)G * tiles[i] / (double)std::max<long long>(total, 1));
        int p = (int)std::max<long long>(1, std::min<long long>(want, tiles[i]));
        used += p - 1;
        P[i] = p;
    }
    while (used < G) {
        int best = -1;
        double best_ratio = 0.0;
        for (int i = 0; i < A; ++i) {
            if (P[i] >= tiles[i]) continue;
            double r = (double)tiles[i] / P[i];
            if (r > best_ratio) { best_ratio = r; best = i; }
        }
        if (best < 0) break;
        P[best] += 1;
        ++used;
    }
    while (used > G) {
        int best = -1;
        double best_ratio = 1e300;
        for (int i = 0; i < A; ++i) {
            if (P[i] <= 1) continue;
            double r = (double)tiles[i] / P[i];
            if (r < best_ratio) { best_ratio = r; best = i; }
        }
        if (best < 0) break;
        P[best] -= 1;
        --used;
    }
    return P;
}

template <typename T>
int advance_impl(phs_engine* e, long long n_steps, int ctas_per_sm, cudaStream_t stream, bool sync) {
    if (e->broken) return PHS_ERR_STATE;
    if (n_steps <= 0) return PHS_OK;
    int occ = 0;
    int rc = occupancy_for<T>(&occ);
    if (rc != PHS_OK) return rc;
    if (occ < 1) return PHS_ERR_CUDA;
    int cps = (ctas_per_sm > 0) ? std::min(ctas_per_sm, occ) : occ;
    const int G = e->sms * cps;
    std::vector<int> act;
    for (size_t i = 0; i < e->inst.size(); ++i)
        if (e->inst[i].used && !e->inst[i].finished) act.push_back((int)i);
    if (act.empty()) return PHS_OK;

    // descriptors of all active instances
    std::vector<InstDev<T>> descs;
    descs.reserve(act.size());
    for (int i : act) descs.push_back(make_dev<T>(e->inst[i]));
    size_t bytes = descs.size() * sizeof(InstDev<T>);
    if (bytes > e->d_desc_bytes) {
        if (e->d_desc) cudaFree(e->d_desc);
        PHS_CUDA_TRY(cudaMalloc(&e->d_desc, bytes));
        e->d_desc_bytes = bytes;
    }
    PHS_CUDA_TRY(cudaMemcpyAsync(e->d_desc, descs.data(), bytes, cudaMemcpyHostToDevice, stream));

    // waves of at most G instances
    std::vector<int4> map_all;
    std::vector<std::pair<size_t, int>> waves;  // (offset into map, grid)
    for (size_t w0 = 0; w0 < act.size(); w0 += (size_t)G) {
        size_t w1 = std::min(act.size(), w0 + (size_t)G);
        std::vector<int> tiles;
        for (size_t i = w0; i < w1; ++i) tiles.push_back(e->inst[act[i]].n_tiles);
        std::vector<int> P = team_sizes(tiles, G);
        size_t off = map_all.size();
        int grid = 0;
        for (size_t i = w0; i < w1; ++i) {
            int p = P[i - w0];
            for (int r = 0; r < p; ++r) map_all.push_back(make_int4((int)i, r, p, 0));
            grid += p;
        }
        waves.push_back({off, grid});
    }
    if (map_all.size() > e->d_map_n) {
        if (e->d_map) cudaFree(e->d_map);
        PHS_CUDA_TRY(cudaMalloc(&e->d_map, map_all.size() * sizeof(int4)));
        e->d_map_n = map_all.size();
    }
    PHS_CUDA_TRY(cudaMemcpyAsync(e->d_map, map_all.data(), map_all.size() * sizeof(int4),
                                 cudaMemcpyHostToDevice, stream));
    for (auto& wv : waves) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)wv.second);
        cfg.blockDim = dim3(kThreads);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        const InstDev<T>* dd = (const InstDev<T>*)e->d_desc;
        const int4* mp = e->d_map + wv.first;
        cudaError_t ce;
        if (sizeof(T) == 8)
            ce = cudaLaunchKernelEx(&cfg, step_kernel<T, kVptF64>, dd, mp, (long long)n_steps, e->abort_word);
        else
            ce = cudaLaunchKernelEx(&cfg, step_kernel<T, kVptF32>, dd, mp, (long long)n_steps, e->abort_word);
        if (ce != cudaSuccess) { set_last_error("launch step_kernel", ce); return PHS_ERR_CUDA; }
        e->launches += 1;
    }
    if (!sync) return PHS_OK;
    PHS_CUDA_TRY(cudaStreamSynchronize(stream));
    unsigned int ab = 0;
    PHS_CUDA_TRY(cudaMemcpy(&ab, e->abort_word, sizeof(ab), cudaMemcpyDeviceToHost));
    if (ab) { e->broken = true; return PHS_ERR_TIMEOUT; }
    int worst = PHS_OK;
    for (int i : act) {
        InstHost& h = e->inst[i];
        PHS_CUDA_TRY(cudaMemcpy(&h.st_host, h.st, sizeof(InstState), cudaMemcpyDeviceToHost));
        if (h.st_host.step >= h.d.n_steps || h.st_host.status == PHS_ERR_NONFINITE) h.finished = true;
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
    int rc = (precision == PHS_PREC_F64) ? occupancy_for<double>(&occ) : occupancy_for<float>(&occ);
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
