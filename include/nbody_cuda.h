/*
 * nbody_cuda.h - C-ABI of the B200 (sm_100a) direct-summation Hermite-4
 * N-body engine (libnbody_cuda.so).
 *
 * This header replaces the reference's force back-end interface:
 *   include/kernel.h:15-19        void force_calculation(13 x double*, Sys&)
 *   include/nbody_tt_integration.h  (TT-Metal host API plumbing)
 *   src/kernel.cpp:47-1224        five #if-selected force_calculation bodies
 * and exposes, as device kernels, the O(N) Hermite pieces of
 *   src/nbody.cpp:131-222         initialdt, prediction, snapandcrackle,
 *                                 correction, updatedt
 *   src/utils.cpp:125-153         compute_kinetic, compute_potential
 *
 * Conventions
 *   - Every entry returns nbody_status; no exception crosses the boundary.
 *     nbody_last_error() returns a thread-local message for the last failure.
 *   - Host arrays are borrowed for the duration of a call only.  The engine
 *     owns its device memory from nbody_create to nbody_destroy; no entry
 *     point allocates after nbody_create (the autotuner, graph capture and
 *     ensemble set-up allocate once, on first use).
 *   - An engine is not thread-safe; it serialises all work on its own CUDA
 *     stream.  Several engines may coexist.
 *   - Array layout is SoA float64: x, y, z, m, vx, vy, vz and ax, ay, az,
 *     jx, jy, jz ("jerk" = adot in the reference's names).
 *   - Physics: G = 1.  a_i = sum_j m_j r_ij / (r_ij^2 + eps2)^(3/2),
 *     r_ij = x_j - x_i; jerk_i = sum_j m_j [v_ij / (.)^(3/2)
 *     - 3 (r_ij . v_ij) r_ij / (.)^(5/2)]  (src/kernel.cpp:1187-1221).
 *     The self term (j = i) contributes exactly zero when eps2 > 0.
 */
#ifndef NBODY_CUDA_H
#define NBODY_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  NBODY_OK = 0,
  NBODY_ERR_INVALID_ARG = 1, /* bad size, null pointer, eps2 out of range ... */
  NBODY_ERR_OOM = 2,         /* device or pinned allocation failed at create */
  NBODY_ERR_CUDA = 3,        /* a CUDA runtime call failed                   */
  NBODY_ERR_TIMEOUT = 4,     /* a bounded in-kernel wait gave up             */
  NBODY_ERR_NONFINITE = 5,   /* NaN/Inf in a diagnostic                      */
  NBODY_ERR_NO_DEVICE = 6,   /* no sm_100 device visible                     */
  NBODY_ERR_STATE = 7        /* call order (e.g. step before set_state)      */
} nbody_status;

typedef enum {
  NBODY_FP64 = 0,  /* all-FP64 pair loop                                     */
  NBODY_MIXED = 1  /* FP32 pair loop on hi/lo positions, FP64 accumulation   */
} nbody_precision;

typedef struct {
  int n;              /* bodies, >= 1                                       */
  double eps2;        /* softening^2, 1e-30 <= eps2 <= 1e30 (runtime; the
                         reference hard-codes 1e-7: include/kernel.h:13)    */
  int precision;      /* nbody_precision (mixed: eps2 >= 1e-24)             */
  int device;         /* CUDA ordinal                                       */
  double dt;          /* > 0: fixed shared step; <= 0: adaptive (Aarseth,
                         src/nbody.cpp:131-150, 198-222)                    */
  double eta;         /* adaptive criterion, default 1e-2 (nbody.h:16)      */
  double eta0;        /* initial-dt criterion, default 1e-4 (nbody.h:15)    */
  int tune;           /* 1: time candidate tilings on first use (autotuner) */
  int threads, i_per_thread, j_tile, split_j; /* 0 = choose automatically   */
  int pair_variant;   /* mixed only: 0 = automatic (variant 4 from 16384
                         bodies, variant 3 below, where building the tiles
                         costs more than it saves), 1 = scalar FP32 kernel
                         on hi/lo positions, 2 = packed-pair (f32x2) hi/lo
                         kernel, FP64 accumulators in registers, 3 = packed
                         hi/lo kernel, FP64 accumulators in shared memory,
                         4 = near/far tile-relative packed-pair kernel: the
                         engine keeps its bodies in Hilbert order and cuts
                         them into j-tiles with float offsets from each
                         tile's centre; a tile far from a warp's rows
                         (separated by at least half its radius) costs one
                         add per separation component, a near tile forms
                         the separation in double-single (hi/lo offsets),
                         so close pairs keep the hi/lo kernels' accuracy
                         (the fastest for large systems), 5 = the same
                         kernel with every tile taken as far (plain
                         tile-relative offsets; a comparison)               */
  int sort_every;     /* tile-relative kernels: re-order the bodies along
                         the Hilbert curve every this many steps (tile
                         centres and offsets are rebuilt every step);
                         0 = 16                                             */
  int j_cluster;      /* pair_variant 4 with an explicit shape: CTAs per
                         thread-block cluster along j (2, 4 or 8), whose
                         split partials are summed in the cluster through
                         distributed shared memory (split_j is rounded up
                         to a multiple); 0 = no cluster.  Measured at
                         N = 65536 the smaller corrector read cancels the
                         slower pair pass, so the autotuner does not time
                         cluster kernels                                    */
} nbody_config;

typedef struct nbody_engine nbody_engine;

typedef struct {
  double pred_ms, eval_ms, corr_ms; /* last step, CUDA events: the reference's
                                       PRED / EVAL / CORR columns
                                       (src/main.cpp:107-116)               */
  double eval_init_ms;              /* first force evaluation               */
  int num_sms;
  int threads, i_per_thread, j_tile, split_j; /* tiling in use          */
  long long steps;                  /* Hermite steps taken                  */
  double t, dt;                     /* model time and current shared dt     */
  int record_format;                /* j-records of the pair kernel in use:
                                       0 FP64, 1 FP32 hi/lo, 2 packed hi/lo,
                                       3 packed near/far tile-relative
                                       (bodies kept in Hilbert order)       */
  int step_kernels;                 /* kernel launches in one captured step */
  long long reorders;               /* Hilbert re-orderings run by steps     */
  int order_kernels;                /* kernel launches in one re-ordering   */
  double dt_crit;                   /* criterion of the last completed pass:
                                       after a step, the Aarseth shared step
                                       min_i sqrt(eta (|a||a2| + |j|^2) /
                                       (|j||a3| + |a2|^2)) from the pre-step
                                       a, j (src/nbody.cpp:198-222), computed
                                       in fixed-dt mode too (where it is only
                                       reported); after an adaptive-mode
                                       nbody_acc_jerk, the initial criterion
                                       min_i eta0 |a|/|j| (src/nbody.cpp:
                                       131-150); 0 before either            */
  int tiling_source;                /* how the tiling in use was chosen:
                                       0 = not yet chosen, 1 = heuristic
                                       (wave model) or explicit config,
                                       2 = timed by the autotuner for this
                                       engine, 3 = the autotuner's earlier
                                       result for the same (device,
                                       precision, kernel family, size),
                                       reused from the process-wide cache  */
  double near_tile_fraction;        /* near/far tile-relative kernel: share
                                       of (warp, j-tile) pairs of the last
                                       pair pass over this engine's bodies
                                       that took the double-single (near)
                                       form; 0 for other kernels            */
  int j_cluster;                    /* CTAs per thread-block cluster along
                                       j of the kernel in use (1: none)     */
} nbody_timers;

/* Fill *cfg with defaults: eps2 = 1e-7, FP64, device 0, adaptive dt,
 * eta = 1e-2, eta0 = 1e-4, no tuning, automatic tiling. */
nbody_status nbody_config_init(nbody_config* cfg);

nbody_status nbody_create(nbody_engine** out, const nbody_config* cfg);
nbody_status nbody_destroy(nbody_engine* eng);

/* Upload x..vz (n each).  Resets model time and the derivative state. */
nbody_status nbody_set_state(nbody_engine* eng, const double* x, const double* y,
                             const double* z, const double* m, const double* vx,
                             const double* vy, const double* vz);
/* Download positions and velocities (any pointer may be NULL to skip). */
nbody_status nbody_get_state(nbody_engine* eng, double* x, double* y, double* z, double* vx,
                             double* vy, double* vz);
/* Download the current acc and jerk (any pointer may be NULL). */
nbody_status nbody_get_derivs(nbody_engine* eng, double* ax, double* ay, double* az,
                              double* jx, double* jy, double* jz);

/* Evaluate acc + jerk of the current state into the engine's derivative
 * arrays (the force_calculation equivalent; include/kernel.h:15-19).  In
 * adaptive mode also sets dt from the initial criterion (initialdt). */
nbody_status nbody_acc_jerk(nbody_engine* eng);

/* The three Hermite phases, individually (src/nbody.cpp:152-196):
 * predict x, v in place; evaluate acc/jerk of the predicted state into the
 * engine's new-derivative buffer; correct with snap/crackle and adopt the
 * new derivatives (and the Aarseth dt in adaptive mode). */
nbody_status nbody_predict(nbody_engine* eng);
nbody_status nbody_eval_predicted(nbody_engine* eng);
nbody_status nbody_correct(nbody_engine* eng);

/* nsteps complete Hermite steps (predict, evaluate, correct), replayed from
 * a captured CUDA graph.  Calls nbody_acc_jerk first if no derivatives
 * exist yet.  Asynchronous: returns once enqueued. */
nbody_status nbody_step(nbody_engine* eng, int nsteps);
nbody_status nbody_synchronize(nbody_engine* eng);

/* FP64 kinetic and potential energy of the current state, G = 1,
 * U = -sum_{i<j} m_i m_j / sqrt(r^2 + eps2).  ref_compat = 1 reproduces the
 * reference's printed potential, which uses m_j*m_j (src/utils.cpp:148). */
nbody_status nbody_energy(nbody_engine* eng, int ref_compat, double* T, double* U);

nbody_status nbody_get_timers(nbody_engine* eng, nbody_timers* out);
/* Set model time and (if dt > 0) the current shared step, e.g. on resume. */
nbody_status nbody_set_time(nbody_engine* eng, double t, double dt);
/* The engine's CUDA stream (cudaStream_t), for callers that order their own
 * work against it. */
nbody_status nbody_get_stream(nbody_engine* eng, void** stream);

const char* nbody_last_error(void);
const char* nbody_status_string(nbody_status s);

/* ---- the drop-in for the reference's force back end ------------------------
 * Same arguments and meaning as force_calculation (include/kernel.h:15-19):
 * reads x, y, z, m, vx, vy, vz (host), zeroes the six outputs and writes the
 * acc and jerk of i-rows [i_begin, i_end) against all n bodies; rows outside
 * the range stay zero, so an MPI caller that sums ranks (src/nbody.cpp:
 * 240-246) gets the complete result.  A cached engine per (thread, device)
 * is reused, so repeated calls allocate nothing after the first.  Copies
 * host->device and back inside the call (the reference contract).
 * precision = NBODY_MIXED: the near/far tile-relative kernel from 32768
 * bodies over the full row range (each call orders the bodies along the
 * Hilbert curve in device memory and returns results in the caller's order),
 * the packed hi/lo kernel below that and for partial row ranges.  The
 * tiling is the heuristic one unless the autotuner has chosen one for the same
 * device, precision and n in this process (nbody_force_calculation_tune, or an
 * engine created with tune = 1); the call itself never runs the autotuner. */
nbody_status nbody_force_calculation(int n, double eps2, int precision, int i_begin, int i_end,
                                     const double* x, const double* y, const double* z,
                                     const double* m, const double* vx, const double* vy,
                                     const double* vz, double* ax, double* ay, double* az,
                                     double* jx, double* jy, double* jz);
/* Optional, once per system size: runs the autotuner for full-row
 * nbody_force_calculation calls of these n bodies (the same arguments as the
 * call's inputs) on the calling thread's cached engine and keeps its choice
 * for the process.  Takes about a second at n = 65536 (tens of trial
 * launches); later calls of this size and precision use the tuned tiling.
 * No reference counterpart: the reference's back end has no tiling. */
nbody_status nbody_force_calculation_tune(int n, double eps2, int precision, const double* x,
                                          const double* y, const double* z, const double* m,
                                          const double* vx, const double* vy, const double* vz);
/* Release the cached drop-in engines of the calling thread. */
nbody_status nbody_force_calculation_release(void);

/* ---- device-pointer entry (zero-copy; used by the torch binding) ----------
 * Same physics on caller-owned device arrays (float64, n each, on the
 * engine's device); work is ordered on `stream` (cudaStream_t, NULL = the
 * engine's stream).  eng supplies eps2, precision, tiling and scratch; n must
 * be <= the engine's n.  It reuses the engine's j-record and partial-sum
 * buffers, so an engine used this way should not be stepping at the same time
 * (between a nbody_predict and its nbody_eval_predicted, say). */
nbody_status nbody_acc_jerk_device(nbody_engine* eng, int n, const double* x, const double* y,
                                   const double* z, const double* m, const double* vx,
                                   const double* vy, const double* vz, double* ax, double* ay,
                                   double* az, double* jx, double* jy, double* jz,
                                   void* stream);

/* ---- allocation-free variant of nbody_acc_jerk_device ----------------------
 * No counterpart in the reference.  For callers that must not allocate
 * device memory (an application that owns the device memory budget through
 * its own pool, a real-time loop where cudaMalloc/cudaFree would stall the
 * device, code running inside someone else's time-step loop): same inputs,
 * outputs and physics as nbody_acc_jerk_device (mixed precision: the packed
 * hi/lo kernel with FP64 accumulators in registers, pair_variant 2), but no
 * engine and no cudaMalloc - its scratch is a 16 MiB static device array
 * inside the library, held by every GPU that loads the library until the
 * process exits.  n must be <= 32768 (NBODY_ERR_INVALID_ARG beyond).  Arrays
 * are float64 on the current device; work is enqueued on `stream`
 * (cudaStream_t, NULL = the legacy default stream) and the call returns
 * without waiting.  Each call on a stream that is not capturing looks up the
 * scratch address (cudaGetSymbolAddress); one on a capturing stream reuses
 * the last lookup, so make the first call on a device before any stream
 * capture.  All calls share the scratch: calls that overlap on the GPU race;
 * order them on one stream.  Because the call does not wait, a bounded-wait
 * timeout of its pair kernel cannot come back as a status: it shows up as NaN
 * in all six outputs.  A CUDA error already pending in the calling thread is
 * reported (NBODY_ERR_CUDA) and left in place; nothing is launched then. */
nbody_status nbody_acc_jerk_noalloc(int n, double eps2, int precision, const double* x,
                                    const double* y, const double* z, const double* m,
                                    const double* vx, const double* vy, const double* vz,
                                    double* ax, double* ay, double* az, double* jx, double* jy,
                                    double* jz, void* stream);

/* ---- batched ensembles -------------------------------------------------------
 * Many independent systems ("clusters") of uneven size, advanced together:
 * each Hermite step is one persistent pair launch over a work list of
 * (cluster, 256-row block, j-tile range) items, captured with the O(N)
 * kernels in one CUDA graph.  No reference counterpart (the reference runs one
 * system); per cluster the physics is exactly the single-system engine's.
 * Each cluster has its own softening and fixed shared step.  State arrays are
 * the clusters' bodies concatenated in cluster order (sum n[c] values each). */
typedef struct nbody_ensemble nbody_ensemble;
typedef struct {
  int nclusters;
  const int* n;          /* bodies per cluster (>= 1)                        */
  const double* eps2;    /* softening^2 per cluster                          */
  const double* dt;      /* fixed shared step per cluster (> 0)              */
  int precision;         /* nbody_precision                                  */
  int device;
  int tiles_per_item;    /* j-tiles per work item; 0 = default 8, or (with the
                            kernel shape) chosen by timing when tune = 1    */
  int tune;
  int pair_variant;      /* mixed only: 0 = automatic (the packed hi/lo
                            kernel, the faster one for clusters of up to a
                            few thousand bodies), 3 = packed hi/lo kernel,
                            4 = near/far tile-relative kernel (each cluster
                            kept in Hilbert order within its segment),
                            5 = tile-relative with every tile taken as far
                            (nbody_config numbering)                       */
  int sort_every;        /* variants 4, 5: re-order every this many steps;
                            0 = 16                                          */
} nbody_ensemble_config;
typedef struct {
  int nclusters, padded_rows, items, tiles_per_item, grid;
  int threads, j_tile;           /* persistent kernel shape in use */
  double interactions_per_step;  /* sum of n[c]^2 */
  long long steps;
  double last_step_ms;           /* CUDA events around the last graph step */
  int record_format;             /* as nbody_timers.record_format          */
  int step_kernels;              /* kernel launches in one captured step   */
  long long reorders;            /* Hilbert re-orderings run by steps       */
  int order_kernels;             /* kernel launches in one re-ordering     */
} nbody_ensemble_info_t;

nbody_status nbody_ensemble_create(nbody_ensemble** out, const nbody_ensemble_config* cfg);
nbody_status nbody_ensemble_destroy(nbody_ensemble* ens);
nbody_status nbody_ensemble_set_state(nbody_ensemble* ens, const double* x, const double* y,
                                      const double* z, const double* m, const double* vx,
                                      const double* vy, const double* vz);
nbody_status nbody_ensemble_get_state(nbody_ensemble* ens, double* x, double* y, double* z,
                                      double* vx, double* vy, double* vz);
nbody_status nbody_ensemble_get_derivs(nbody_ensemble* ens, double* ax, double* ay, double* az,
                                       double* jx, double* jy, double* jz);
nbody_status nbody_ensemble_acc_jerk(nbody_ensemble* ens);
nbody_status nbody_ensemble_step(nbody_ensemble* ens, int nsteps);
nbody_status nbody_ensemble_synchronize(nbody_ensemble* ens);
/* Per-cluster FP64 kinetic and potential energy (arrays of nclusters). */
nbody_status nbody_ensemble_energy(nbody_ensemble* ens, double* T, double* U);
nbody_status nbody_ensemble_info(nbody_ensemble* ens, nbody_ensemble_info_t* out);
nbody_status nbody_ensemble_get_stream(nbody_ensemble* ens, void** stream);

/* ---- adjoint (reverse-mode gradients) -----------------------------------------
 * No reference counterpart.  Gradients of a scalar loss of the final positions
 * and velocities of a fixed-dt Hermite-4 run with respect to the initial
 * positions, velocities and masses.  The forward keeps the state every
 * checkpoint_every steps; the backward recomputes each segment and runs the
 * hand-written adjoint kernels (pair acc/jerk VJP in FP64, reverse corrector
 * and predictor).  All arrays are float64 device pointers of n values on the
 * adjoint's device; work is ordered on `stream` (cudaStream_t, NULL = legacy
 * default stream); the calls return after their work completes. */
typedef struct nbody_adjoint nbody_adjoint;
typedef struct {
  int n;
  double eps2;
  int precision;         /* forward pair loop: NBODY_FP64 or NBODY_MIXED     */
  int device;
  double dt;             /* fixed shared step (> 0)                          */
  int nsteps;
  int checkpoint_every;  /* >= 1                                             */
} nbody_adjoint_config;

nbody_status nbody_adjoint_create(nbody_adjoint** out, const nbody_adjoint_config* cfg);
nbody_status nbody_adjoint_destroy(nbody_adjoint* adj);
/* Runs nsteps from (x, v, m) and writes the final positions and velocities. */
nbody_status nbody_adjoint_forward(nbody_adjoint* adj, const double* x, const double* y,
                                   const double* z, const double* m, const double* vx,
                                   const double* vy, const double* vz, double* x1, double* y1,
                                   double* z1, double* vx1, double* vy1, double* vz1,
                                   void* stream);
/* Given dL/d(final x, v), writes dL/d(initial x, v) and dL/dm.  Needs the
 * preceding nbody_adjoint_forward. */
nbody_status nbody_adjoint_backward(nbody_adjoint* adj, const double* gx, const double* gy,
                                    const double* gz, const double* gvx, const double* gvy,
                                    const double* gvz, double* gx0, double* gy0, double* gz0,
                                    double* gvx0, double* gvy0, double* gvz0, double* gm,
                                    void* stream);
/* One pair VJP: given adjoints (abar, jbar) of acc and jerk at state (x, v, m),
 * writes (xbar, vbar, mbar) = the transposed Jacobian applied to them. */
nbody_status nbody_adjoint_vjp_acc_jerk(nbody_adjoint* adj, const double* x, const double* y,
                                        const double* z, const double* m, const double* vx,
                                        const double* vy, const double* vz, const double* abx,
                                        const double* aby, const double* abz, const double* jbx,
                                        const double* jby, const double* jbz, double* gx,
                                        double* gy, double* gz, double* gvx, double* gvy,
                                        double* gvz, double* gm, void* stream);

/* ---- initial conditions (host, deterministic) ------------------------------
 * Plummer sphere in Henon units (G = M = 1, E = -1/4), equal masses 1/n,
 * centred on the origin in position and velocity; sampled by the
 * Aarseth-Henon-Wielen (1974) method from a seeded xoshiro256** stream. */
nbody_status nbody_plummer(int n, uint64_t seed, double* x, double* y, double* z, double* m,
                           double* vx, double* vy, double* vz);
/* The reference's own initial conditions (src/nbody.cpp:69-114: std::mt19937
 * seed 42, vmax = rmax = mmax = 1, mmin = 0.01, virial rescale with the
 * reference potential at eps2) - the bodies of its `--N 1024` default run. */
nbody_status nbody_reference_ic(int n, double eps2, double* x, double* y, double* z, double* m,
                                double* vx, double* vy, double* vz);

/* ---- state files (host) -----------------------------------------------------
 * Binary SoA snapshot: 64-byte header ("NBODYST1", version 1, n, t, dt, eps2)
 * then x, y, z, m, vx, vy, vz as float64.  Reading with all array pointers
 * NULL returns the header only (n, t, dt, eps2). */
nbody_status nbody_write_state_file(const char* path, int n, double t, double dt, double eps2,
                                    const double* x, const double* y, const double* z,
                                    const double* m, const double* vx, const double* vy,
                                    const double* vz);
nbody_status nbody_read_state_file(const char* path, int n_max, int* n, double* t, double* dt,
                                   double* eps2, double* x, double* y, double* z, double* m,
                                   double* vx, double* vy, double* vz);

/* ---- measured pipe peaks (diagnostic) ---------------------------------------
 * Times FP64 FMA, FP32 FMA and MUFU rsqrt throughput on `device` with
 * dependent-chain-free microkernels; results in op/s (an FMA counts 2 flop
 * in the *_tflops fields). */
typedef struct {
  double fp64_tflops, fp32_tflops, fp32x2_tflops, mufu_rsqrt_gops;
  double sm_clock_mhz; /* cudaDevAttrClockRate at the time of the call */
} nbody_peaks;
nbody_status nbody_measure_peaks(int device, nbody_peaks* out);

/* Failure-path self-test: one kernel waits on a shared-memory barrier that
 * never completes; its bounded wait gives up after limit_ms (0 < limit_ms <=
 * 2000) and reports through the device status word.  Returns
 * NBODY_ERR_TIMEOUT when the path works (the context stays usable). */
nbody_status nbody_selftest_bounded_wait(int device, double limit_ms);

#ifdef __cplusplus
}
#endif
#endif /* NBODY_CUDA_H */
