/*
 * phs.h -- C ABI of the B200 time-stepping and electrogram path of PyHeartSim.
 *
 * Plain C: pointers, sizes and status codes only.  Every entry point returns an
 * int status (PHS_OK on success).  Device pointers are marked "device"; all
 * other pointers are host memory.  Streams are passed as `void*` holding a
 * cudaStream_t (NULL = the legacy default stream).
 *
 * Reference interfaces replaced (paths inside jiyuehe/PyHeartSim):
 *   simulation/simulation_gpu.py:261-409   compute(n_voxel, P_2d, geometry_data,
 *                                           simulation_parameters, arrhythmia_parameters)
 *   simulation/simulation_gpu.py:71-136    rk4_reaction_kernel / reaction_step_gpu_rk4
 *   simulation/simulation_gpu.py:138-225   build_diffusion_matrix_gpu (replaced by a
 *                                           matrix-free stencil on a compacted table)
 *   simulation/simulation_gpu.py:227-259   crank_nicolson_diffusion_step_gpu (CuPy GMRES(50))
 *   simulation/pacing.py:136-170           apply_pacing (compiled to a per-step schedule)
 *   simulation/unipolar_electrogram_gpu.py:21-152  compute_egm_kernel_batched / compute
 *   simulation/unipolar_electrogram_equation_parts.py:41-124  distances, gradients, normalisation
 */
#ifndef PHS_H
#define PHS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define PHS_OK                 0
#define PHS_ERR_BAD_ARG        1  /* invalid argument or size                       */
#define PHS_ERR_BAD_TABLE      2  /* neighbour index out of range                    */
#define PHS_WARN_NO_CONVERGE   3  /* a CN solve hit maxiter (reference prints a warning,
                                     simulation/simulation_gpu.py:254-255)           */
#define PHS_ERR_NONFINITE      4  /* NaN/Inf in a solver norm                         */
#define PHS_ERR_OOM            5  /* device allocation failed                         */
#define PHS_ERR_TIMEOUT        6  /* a bounded device-side wait gave up               */
#define PHS_ERR_CUDA           7  /* other CUDA runtime error                         */
#define PHS_ERR_UNSUPPORTED    8  /* input the build does not handle                  */
#define PHS_ERR_STATE          9  /* call not valid in the current state              */

#define PHS_MODEL_MS 0           /* Mitchell-Schaeffer (heart_model_flag 0)            */
#define PHS_MODEL_AP 1           /* Aliev-Panfilov     (heart_model_flag 1)            */

#define PHS_PREC_F32 32          /* FP32 state/basis, FP64 dots and norms              */
#define PHS_PREC_F64 64          /* FP64 everywhere (plain drop-in form)               */

#define PHS_VFLAG_S1      1u     /* voxel is in the S1 pacing set                      */
#define PHS_VFLAG_S2      2u     /* voxel is in the S2 pacing set                      */
#define PHS_VFLAG_TBLOCK  4u     /* voxel row is zeroed while the temporary block holds */

#define PHS_EGM_F64    0         /* FP64 contraction (plain drop-in form)              */
#define PHS_EGM_BF16X3 1         /* BF16 hi/lo split, 3 tcgen05 products, FP32 accumulate */

const char* phs_status_string(int status);
int phs_version(void);
/* SM count and resident CTAs per SM of the step kernel for a precision. */
int phs_device_query(int precision, int* sm_count, int* ctas_per_sm);
/* Last CUDA error text recorded by the library (static storage). */
const char* phs_last_error(void);

/* ------------------------------------------------------- one instance
 * A simulation instance, compacted and ready to upload.  Built on the host from
 * the reference's inputs (P_2d, neighbor_id_2d, the parameter dicts).          */
typedef struct phs_instance_desc {
    int64_t n_voxel;
    int32_t model;            /* PHS_MODEL_MS / PHS_MODEL_AP                              */
    int32_t restart;          /* GMRES restart length m (reference: 50), 1..50            */
    const int32_t* nb6;       /* [n][6] neighbours +x,-x,+y,-y,+z,-z; absent (-1) -> 0 as in the reference */
    const double* coef6;      /* [n][6] c_n/(4 Delta^2) * P_2d[n,k]  (permanent block: 0), or
                                 NULL when every row is isotropic (cw, mask6 below)         */
    const uint8_t* vflags;    /* [n] PHS_VFLAG_* bits                                       */
    const double* vparams;    /* [n][5] P_2d[:,15:20], or NULL to use params[]              */
    double params[5];         /* MS: tau_open, tau_close, tau_in, tau_out, v_gate;
                                 AP: k, a, eps0, mu1, mu2 (P_2d columns 15..19)             */
    double dt;                /* model time step                                            */
    double j_stim;            /* stimulus magnitude (reference: 1)                          */
    int64_t n_steps;          /* steps to run: int(round(t_final/dt))                       */
    const uint8_t* stim;      /* [n_steps] bit0: S1 window active, bit1: S2 window active   */
    int64_t tblock_steps;     /* steps 0..tblock_steps-1 use the temporary-block operator   */
    int32_t sample_stride;    /* sample after step s when s % stride == 0 (0: every step)   */
    int32_t n_samples;        /* history length S                                           */
    int32_t save_h;           /* also keep the gate history                                 */
    int32_t full_cycles;      /* 1: CuPy GMRES semantics (full restart cycles, true-residual
                                 test at each cycle start); 0: Givens early exit            */
    double u0, h0;            /* initial state (MS: 0,1; AP: 0,0)                           */
    double tol, atol;         /* stop when ||r|| <= max(atol, tol*||b||)                    */
    int32_t maxiter;          /* Arnoldi steps per solve before giving up (reference 10000) */
    int32_t guess;            /* 0: start each solve from u* (the reference's x0); 1: from u*
                                 plus the previous step's diffusion increment (same stopping
                                 test, fewer iterations)                                    */
    const double* cw;         /* [n] isotropic rows: the one non-zero coefficient of row n  */
    const uint8_t* mask6;     /* [n] isotropic rows: bit k set when coefficient k is cw[n]  */
    /* Anisotropic tensors (D0 != I).  The face cross terms P_2d[:,6..8] of
     * simulation/simulation_gpu.py:172-197 are folded into coef6 (+ on the + side,
     * - on the - side); the edge cross terms P_2d[:,9..14] of :199-217 are six
     * antisymmetric pairs per row: (L u)_n += coef_edge[n][p] * (u[a] - u[b]) with
     * a = nb_edge[n][2p], b = nb_edge[n][2p+1].  Both NULL for D0 = I.          */
    const int32_t* nb_edge;   /* [n][12] edge neighbours (a0,b0,...,a5,b5), absent -> 0     */
    const double* coef_edge;  /* [n][6]  c_n/(4 Delta^2) * P_2d[n,9+p]                      */
    int32_t device_tables;    /* 1: nb6, coef6, cw, mask6, vflags, vparams, nb_edge and
                                 coef_edge are device pointers (built by phs_operator_tables;
                                 checked on the device); stim stays on the host            */
    int32_t _pad;
} phs_instance_desc;

/* Per-instance progress and solver statistics. */
typedef struct phs_instance_info {
    int64_t n_voxel;
    int64_t step;             /* steps completed                                   */
    int64_t n_steps;
    int32_t samples;          /* history samples written                           */
    int32_t status;           /* PHS_OK / PHS_WARN_NO_CONVERGE / PHS_ERR_NONFINITE  */
    int64_t arnoldi_steps;    /* total Arnoldi iterations                          */
    int64_t solves;           /* CN solves that iterated                           */
    int32_t max_arnoldi;      /* most Arnoldi iterations in one solve              */
    int32_t nonconverged;     /* solves that stopped on maxiter                    */
    int64_t arnoldi_sq;       /* sum over solves of (Arnoldi iterations)^2         */
} phs_instance_info;

/* ------------------------------------------------ batched engine
 * An engine owns device memory for any number of instances of one precision and
 * advances all active instances with one persistent launch per call.            */
typedef struct phs_engine phs_engine;

int phs_engine_create(int precision, phs_engine** out);
int phs_engine_destroy(phs_engine* eng);
/* Upload an instance; returns its slot. */
int phs_instance_add(phs_engine* eng, const phs_instance_desc* desc, int* slot);
int phs_instance_remove(phs_engine* eng, int slot);
int phs_instance_info_get(phs_engine* eng, int slot, phs_instance_info* info);
/* Advance every unfinished instance by up to n_steps steps (one persistent launch,
 * or one per wave when waves > 1).  ctas_per_sm 0 = occupancy limit.  Returns the
 * worst instance status; the launch is asynchronous unless sync != 0.           */
int phs_engine_advance(phs_engine* eng, int64_t n_steps, int ctas_per_sm, void* stream, int sync);
/* Copy history samples [s0, s0+count) of a slot to host buffers ([count][n],
 * element type = engine precision; h_dst may be NULL).  Synchronous.           */
int phs_instance_read_history(phs_engine* eng, int slot, int32_t s0, int32_t count,
                              void* u_dst, void* h_dst);
/* Copy the current state u, h ([n] each, engine precision) and the activation
 * step table lat ([n] int32, -1 = not activated) to host.  Any may be NULL.    */
int phs_instance_read_state(phs_engine* eng, int slot, void* u_dst, void* h_dst, int32_t* lat_dst);
/* Device pointers of an instance's state (for device-side consumers). */
int phs_instance_device_ptrs(phs_engine* eng, int slot, void** u, void** hist_u, int32_t** lat);
/* Number of kernel launches the engine issued since creation. */
int64_t phs_engine_launch_count(phs_engine* eng);
/* Engine settings.  PHS_CFG_VARIANT: step-kernel variant index (-1 = default);
 * PHS_CFG_CTAS_PER_SM: CTAs per SM used when advance() is given 0 (0 = occupancy
 * limit).  Used by the autotuner.                                               */
#define PHS_CFG_VARIANT      1
#define PHS_CFG_CTAS_PER_SM  2
#define PHS_CFG_PROFILE      3   /* 1: per-instance device phase timers on (small overhead) */
#define PHS_CFG_TEST_TEAM_OVERCOUNT 4  /* test hook: the first team of the next plan waits for a CTA
                                          that is never launched; its bounded barrier gives up after
                                          4 s and advance() returns PHS_ERR_TIMEOUT (the engine is
                                          then unusable, the CUDA context is not affected)        */
#define PHS_CFG_AUTO_BALANCE 5   /* 1 (default): after an instance is added or removed, the next
                                    launch runs with the phase timers on (if they are off) and
                                    the two after it first call phs_engine_rebalance, so team
                                    sizes follow the measured cost; then the timers go off
                                    again.  0: team sizes change only on explicit rebalance  */
#define PHS_CFG_WAVE_INSTANCES 6 /* at most this many instances per launch wave (0, the default: as
                                    many as the grid holds).  Each wave is one launch over the whole
                                    grid for the same steps, one wave after another, so a wave's
                                    instances have the L2 to themselves                             */
#define PHS_CFG_GROUP_SUMS 7  /* FP64 engines: 1 (default) combines the per-tile partial sums of
                                 every reduction in fixed groups of 8 consecutive tiles before the
                                 leader CTA sums the groups; 0: the leader sums every tile.  The
                                 order is fixed either way (results do not depend on team size) */
#define PHS_CFG_COMPACT_NB 9  /* 1 (default): an instance whose present neighbours of slots 0 and 1
                                 are n+1 and n-1 (the +-x ones in the lattice row order) and whose
                                 other slots' offsets fit int16 around a base per 512-voxel block
                                 has a compact table (8 bytes per voxel instead of 24), read by the
                                 variants of phs_step_variant_layout; same indices, same results.
                                 0: every instance reads the int32 table                       */
int phs_engine_config(phs_engine* eng, int key, int64_t value);
/* Compiled step-kernel variants of a precision: count, and per variant the
 * minimum CTAs per SM it was compiled for and its register count (arrays of at
 * least *count entries, may be NULL).                                           */
int phs_step_variants(int precision, int32_t* count, int32_t* min_ctas_per_sm, int32_t* max_regs);
/* Voxels per thread of each step-kernel variant of a precision (a tile is 256 x
 * that many consecutive voxels); vpt must hold `count` >= the variant count.   */
int phs_step_variant_vpt(int precision, int32_t count, int32_t* vpt);
/* Per variant: bytes of the shared-memory staging ring (0: the variant reads
 * global memory directly; > 0: a producer warp copies each tile's slices into
 * the ring with 1-D bulk copies) and whether it reads the compact neighbour
 * table (PHS_CFG_COMPACT_NB; an unstaged variant that needs it for every
 * instance runs its int32-table twin when one lacks it).  Arrays of at least
 * count entries, may be NULL.                                                  */
int phs_step_variant_layout(int precision, int32_t count, int32_t* ring_bytes, int32_t* compact_table);
/* Re-split the CTAs over the instances in proportion to their cost since the
 * last rebalance: the measured team time per step x team CTAs when the phase
 * timers (PHS_CFG_PROFILE) are on, else voxels x (1.6 + Arnoldi iterations per
 * step).  Synchronises the device; the next advance() rebuilds its plan.        */
int phs_engine_rebalance(phs_engine* eng);
/* Phase timers of an instance (PHS_CFG_PROFILE on): 16 counters, nanoseconds
 * spent by the team's first CTA in [0] RHS pass 2 (right-hand side, initial
 * residual), [1] the RHS barriers, [2] Arnoldi phase A, [3] its barrier, [4]
 * phase C, [5] its barrier, [6] update, [7] residual check, [8] its barrier,
 * [9] final copy, [10] RHS pass 1 (reaction); [11] steps and
 * [12] Arnoldi iterations counted; [13] CTAs in the team at the last launch;
 * [14] nanoseconds in the leader bodies of the team's barriers (whichever CTA
 * led) and [15] team barriers passed.                                          */
int phs_instance_profile(phs_engine* eng, int slot, uint64_t* out16);
/* Bytes per voxel of the neighbour table the instance's compact-table variants
 * read: 8 (compact form, PHS_CFG_COMPACT_NB) or 24 (int32 table).              */
int phs_instance_table_bytes(phs_engine* eng, int slot, int32_t* bytes_per_voxel);

/* ------------------------------------------- one-shot drop-in (host buffers)
 * Runs a whole instance: upload, all steps, download.  Replaces
 * simulation/simulation_gpu.py:261-409.  u_hist/h_hist: [n_samples][n] host,
 * element type = precision.  *n_saved receives the samples written.            */
int phs_simulate(const phs_instance_desc* desc, int precision, void* u_hist, void* h_hist,
                 int32_t* lat, int32_t* n_saved, phs_instance_info* info);

/* ------------------------------------------------------------ electrogram
 * Lead field: M[w][e] such that egm[t][e] = sum_w V[t][w] * M[w][e] reproduces
 * simulation/unipolar_electrogram_gpu.py:55-69 with the gradients of
 * simulation/unipolar_electrogram_equation_parts.py:60-103 folded in.
 * Output is stored transposed, Mt[e][w] (K-major), FP64, on the device.
 *   voxel_xyz  device [n_v][3] f64      electrode_xyz device [n_e][3] f64
 *   c_voxel    device [n_v] f64         D0 device [n_v][9] f64 row-major, or NULL (identity)
 *   in_ptr     device [n_v+1] int32     CSR of incoming gradient terms per voxel w
 *   in_src     device [nnz] int32       source voxel v of each term
 *   in_dir     device [nnz] int8        +(d+1) or -(d+1), d = 0,1,2 (x,y,z)          */
int phs_egm_leadfield_f64(int64_t n_v, int64_t n_e, const double* voxel_xyz,
                          const double* electrode_xyz, const double* c_voxel, const double* D0,
                          const int32_t* in_ptr, const int32_t* in_src, const int8_t* in_dir,
                          double inv_two_delta, double* Mt, void* stream);
/* egm[t][e] = sum_w V[t][w] Mt[e][w], FP64 (device pointers). */
int phs_egm_contract_f64(int64_t T, int64_t n_v, int64_t n_e, const double* V, int64_t ldv,
                         const double* Mt, double* egm, void* stream);
/* Split an FP64/FP32 matrix (rows x cols, leading dim ld) into BF16 hi and lo parts,
 * written with leading dimension ld_out (zero padding to ld_out).  src_is_f64 selects
 * the source type.                                                               */
int phs_split_bf16(int64_t rows, int64_t cols, const void* src, int64_t ld, int src_is_f64,
                   uint16_t* hi, uint16_t* lo, int64_t rows_out, int64_t ld_out, void* stream);
/* egm[t][e] = sum_w (Vhi Mhi + Vhi Mlo + Vlo Mhi) on the tcgen05 tensor cores,
 * FP32 accumulation in TMEM, split-K partials reduced in a fixed order.
 * Vhi/Vlo: [T_pad][K_pad] bf16; Mhi/Mlo: [n_e_pad][K_pad] bf16 (device).
 * T_pad % 128 == 0, n_e_pad % 128 == 0, K_pad % 64 == 0.  work: device scratch
 * of phs_egm_bf16x3_workspace() bytes, whose first 4 bytes are an error word.
 * Asynchronous on `stream` (no host synchronisation): a contraction whose
 * bounded pipeline waits gave up leaves the error word non-zero; read it with
 * phs_egm_bf16x3_status.                                                        */
int64_t phs_egm_bf16x3_workspace(int64_t T_pad, int64_t n_e_pad, int64_t K_pad);
int phs_egm_contract_bf16x3(int64_t T, int64_t n_e, int64_t T_pad, int64_t n_e_pad, int64_t K_pad,
                            const uint16_t* Vhi, const uint16_t* Vlo, const uint16_t* Mhi,
                            const uint16_t* Mlo, float* egm, void* work, void* stream);
/* phs_egm_contract_bf16x3 with a tile configuration, 0 .. count-1 (output tile
 * 128 x 128 or 128 x 256, K blocks of 64 or 32 per pipeline stage); the
 * workspace size above covers every configuration.  For the autotuner.         */
int phs_egm_contract_bf16x3_cfg(int64_t T, int64_t n_e, int64_t T_pad, int64_t n_e_pad, int64_t K_pad,
                                const uint16_t* Vhi, const uint16_t* Vlo, const uint16_t* Mhi,
                                const uint16_t* Mlo, float* egm, void* work, int config, void* stream);
int phs_egm_bf16x3_config_count(void);
/* Synchronise `stream` and read the error word of the last contraction that used
 * `work`: PHS_OK, or PHS_ERR_TIMEOUT when its pipeline waits gave up.          */
int phs_egm_bf16x3_status(const void* work, void* stream);
/* Allocation-free form of phs_egm_contract_f64 (no counterpart in the reference).
 * For callers that cannot allocate device memory when they contract: inside a
 * global-mode stream capture, under another allocator that owns the device
 * memory, or in loops that cannot absorb cudaFree's device-wide synchronisation.
 * Same inputs and result as phs_egm_contract_f64; its split-K partial sums live
 * in a fixed 16 MiB device array (phs_egm_noalloc_capacity() doubles) inside the
 * library, so T * n_e must not exceed that capacity (else PHS_ERR_BAD_ARG).  The
 * array's address is looked up on every call made outside a stream capture (so
 * it stays valid after a device reset) and cached for calls made during one:
 * make the first call on a device before any stream capture (else
 * PHS_ERR_STATE).  All calls share the array, so calls that overlap on the GPU
 * race. */
int phs_egm_contract_f64_noalloc(int64_t T, int64_t n_v, int64_t n_e, const double* V, int64_t ldv,
                                 const double* Mt, double* egm, void* stream);
int64_t phs_egm_noalloc_capacity(void);
/* Scale egm ([T][n_e], f64 or f32 per is_f64) in place by 1/mean_e(max_t - min_t),
 * simulation/unipolar_electrogram_equation_parts.py:118-124.                      */
int phs_egm_normalize(int64_t T, int64_t n_e, void* egm, int is_f64, void* stream);

/* One-shot drop-in for simulation/unipolar_electrogram_gpu.py:71-152 with host
 * buffers: V [T][n_v] f64, tables as above (host), egm_out [T][n_e] f64. */
int phs_electrogram(int64_t T, int64_t n_v, int64_t n_e, const double* V, const double* voxel_xyz,
                    const double* electrode_xyz, const double* c_voxel, const double* D0,
                    const int32_t* in_ptr, const int32_t* in_src, const int8_t* in_dir,
                    double delta, int mode, double* egm_out);

/* ------------------------------------------------ geometry on the device
 * The inputs of the time stepper built on the GPU from lattice coordinates.
 * Replaces the host loops of utility/voxelization.py:102-152
 * (find_neighbor_voxel_ids), simulation/equation_parts.py:36-114
 * (heart_model_equation_parts) and the table build of
 * simulation/simulation_gpu.py:138-225 / 294-330.  Array arguments are device
 * pointers; each call is ordered on `stream` and returns once it has drained. */

/* Neighbour table nb18 [n][18] of integer lattice coordinates ijk [n][3], in the
 * reference's column order with -1 for an absent neighbour.  order (may be NULL)
 * receives the voxels sorted by (z, y, x), x fastest: order[r] = voxel of rank r.
 * PHS_ERR_BAD_TABLE: two voxels share coordinates; PHS_ERR_UNSUPPORTED: the
 * bounding box exceeds 2^31 cells.  Works in a temporary dense grid over the box. */
int phs_lattice_neighbors(int64_t n, const int32_t* ijk, int32_t* nb18, int32_t* order, void* stream);

/* P_2d [n][21] (FP64), bit-identical to the reference, from nb18, D0 [n][3][3]
 * (NULL: identity, the reference's load_fiber) and par [n][6] = P_2d columns
 * 15..20 (five model parameters, then c). */
int phs_equation_parts(int64_t n, const int32_t* nb18, const double* D0, const double* par, double* P,
                       void* stream);

/* out3 (host): [0] some face cross term P_2d[:,6..8] is non-zero, [1] some edge
 * cross term P_2d[:,9..14] is non-zero, [2] P_2d[:,15..19] is the same on every row. */
int phs_operator_flags(int64_t n, const double* P, int32_t* out3, void* stream);

/* Operator tables of one instance in device row order, as the host compilation
 * builds them (face neighbours remapped -1 -> 0 and through the order, the
 * coefficients c/(4 Delta^2) P_2d[:,k] with the face cross terms folded in when
 * face_cross is set, the isotropic row form, S1/S2/temporary-block flags,
 * per-voxel parameters, edge pairs when edge is set).                        */
typedef struct phs_operator_tables_args {
    int64_t n_voxel;
    double Delta;
    const double* P;          /* [n][21], caller order                                      */
    const int32_t* nb18;      /* [n][18], caller order, -1 absent                           */
    const int32_t* node_flag; /* [n] or NULL: 4 permanent block (c -> 0), 3 temporary block */
    const int32_t* order;     /* [n]: device row r holds caller voxel order[r]; NULL = same */
    int32_t* inv;             /* [n] out: device row of each caller voxel                   */
    int32_t* nb6;             /* [n][6] out                                                 */
    double* coef6;            /* [n][6] out                                                 */
    double* cw;               /* [n] out: first non-zero coefficient of the row (or 0)      */
    uint8_t* mask6;           /* [n] out: bit k set when coefficient k is non-zero          */
    uint8_t* vflags;          /* [n] out: PHS_VFLAG_* bits                                  */
    double* vparams;          /* [n][5] out: P_2d[:,15..19], or NULL to skip                */
    int32_t* nb_edge;         /* [n][12] out when edge != 0                                 */
    double* coef_edge;        /* [n][6] out when edge != 0                                  */
    const int64_t* s1;        /* [n_s1] caller ids of the S1 pacing set, or NULL            */
    int64_t n_s1;
    const int64_t* s2;        /* [n_s2] caller ids of the S2 pacing set, or NULL            */
    int64_t n_s2;
    uint32_t* iso_word;       /* device workspace, one word                                 */
    int32_t face_cross;       /* in: from phs_operator_flags                                */
    int32_t edge;             /* in: from phs_operator_flags                                */
    int32_t iso;              /* out: every row is isotropic (cw, mask6 describe it)        */
    int32_t _pad;
    void* stream;
} phs_operator_tables_args;
int phs_operator_tables(phs_operator_tables_args* args);

/* ------------------------------------------------ electrogram analysis (device)
 * Electrode activation times, utility/lat_map.py:20-27: lat_out[e] (int32) =
 * first t maximising -(egm[t+1][e] - egm[t][e]) (NaN counts as the largest),
 * minus the minimum over electrodes.  egm [T][n_e], f64 (is_f64) or f32.      */
int phs_electrode_lat(int64_t T, int64_t n_e, const void* egm, int is_f64, int32_t* lat_out, void* stream);
/* utility/lat_map.py:29-46 (interpolate_lat) on the device: electrode LAT
 * spread over voxels.  Inputs (device, f64): voxel [n_v][ndim] and electrode
 * [n_e][ndim] coordinates with the constant dimensions already dropped (ndim 2
 * or 3), lat_electrode [n_e], and the Delaunay triangulation of the electrodes
 * as scipy.spatial.Delaunay gives it: simplices [n_simplex][ndim+1] (int32),
 * transform [n_simplex][ndim+1][ndim] (inverse vertex matrix, then the last
 * vertex), neighbors [n_simplex][ndim+1] (int32), min_bound/max_bound [ndim].
 * Output lat_voxel [n_v]: barycentric interpolation in the first simplex (index
 * order) containing the voxel within eps = 100 DBL_EPSILON, the nearest
 * electrode's LAT outside the hull.  Asynchronous on `stream`.                */
int phs_interpolate_lat(int64_t n_v, int ndim, const double* voxel, int64_t n_e, const double* electrode,
                        const double* lat_electrode, int64_t n_simplex, const int32_t* simplices,
                        const double* transform, const int32_t* neighbors, const double* min_bound,
                        const double* max_bound, double* lat_voxel, void* stream);
/* Every upward crossing of `threshold` by Vm, per voxel, in a device history
 * hist [S][ld] (f64 or f32 per is_f64; e.g. phs_instance_device_ptrs' hist_u):
 * sample s is a crossing when hist[s][v] >= threshold and hist[s-1][v] <
 * threshold (the state before sample 0 counts as below).  The first
 * max_per_voxel crossing samples of voxel v go to times[v*max_per_voxel + i]
 * (device), counts[v] (device) gets the number of crossings.  The first
 * crossing of a history sampled every step is the activation table of
 * utility/lat_map.py's Vm counterpart (the step kernel's lat); the later ones
 * are re-activations (re-entry).  Asynchronous on `stream`.                    */
int phs_activation_times(int64_t S, int64_t n, const void* hist, int64_t ld, int is_f64, double threshold,
                         int32_t max_per_voxel, int32_t* times, int32_t* counts, void* stream);
/* Conduction velocity, utility/conduction_velocity.py:23-70: for each of n_e
 * points xyz [n_e][3] with activation times lat [n_e] (f64), the minimum-norm
 * least-squares plane through the points within `radius` (itself included;
 * the reference uses 8 mm); v_vec [n_e][3] = grad / |grad|^2, v_mag [n_e] =
 * 1 / |grad|, NaN with fewer than 4 points or |grad|^2 <= 1e-8.             */
int phs_conduction_velocity(int64_t n_e, const double* xyz, const double* lat, double radius, double* v_vec,
                            double* v_mag, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* PHS_H */
