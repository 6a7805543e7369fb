/*
 * bia_capi.h -- C ABI of libbia_b200.so, the B200 (sm_100a) BIA pair-step library.
 *
 * Two groups of entry points:
 *
 *  1. Drop-in replacements for the reference's Fortran-callable symbols.  Same
 *     names, same gfortran calling convention (scalars by value through %VAL,
 *     arrays as host pointers), same accumulate/overwrite semantics, void return.
 *     Status of the last call on this host thread: bia_last_error().
 *
 *  2. A status-returning API with device-resident state owned by the caller or
 *     by a bia_context (one per host thread, explicit CUDA stream).
 *
 * All arrays are FP64.  State arrays are structure-of-arrays: x, y, z, u, v, w,
 * each of length n.  No function takes or returns a torch type.
 */
#ifndef BIA_CAPI_H
#define BIA_CAPI_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------- */
enum bia_status {
    BIA_OK = 0,
    BIA_ERR_INVALID_ARGUMENT = 1, /* bad n, NULL pointer, unknown method, ... */
    BIA_ERR_NONFINITE = 2,        /* a pair produced a non-finite displacement */
    BIA_ERR_NOT_CONVERGED = 3,    /* reserved: RKF step-size underflow / iteration limit */
    BIA_ERR_DEVICE_TIMEOUT = 4,   /* a bounded device-side wait gave up */
    BIA_ERR_CUDA = 5,             /* a CUDA runtime call failed */
    BIA_ERR_OUT_OF_MEMORY = 6,
    BIA_ERR_NO_DEVICE = 7
};

/* pair solver: the reference's METHOD argument (bia/bia.f90:134-139), plus
   BIA_METHOD_UNIVERSAL, which advances every pair with the universal-variable
   (Stumpff function) solver that ALG uses for near-unit-eccentricity pairs */
enum bia_method {
    BIA_METHOD_RKF = 0,
    BIA_METHOD_ALG = 1,
    BIA_METHOD_UNIVERSAL = 2,
    /* the learned mixed-precision form: attractive ellipses and hyperbolae inside a learned
       head's domain start from the head's guess (BF16 tensor cores, FP32 accumulation), take
       one FP32 Newton correction and one FP64 Halley step; every other pair, and any pair
       whose FP64 step does not settle, takes the universal-variable solver.  Needs the heads
       loaded with bia_context_set_heads. */
    BIA_METHOD_LEARNED = 3
};

typedef struct bia_config {
    int method;        /* BIA_METHOD_ALG (Kepler/Barker solve), BIA_METHOD_RKF or
                          BIA_METHOD_UNIVERSAL */
    int itr;           /* Newton iteration cap, ITR = 18 (bia/bia.f90:52) */
    double eps_th;     /* coupling of r'' = eps r/|r|^3 (bia/bia.f90:37); with charges q
                          the pair coupling is eps_th * q_i * q_j */
    double dt;         /* step length, time_end (bia/bia.f90:35) */
    double err;        /* residual above which a pair counts as not converged, ERR = 1e-12 */
    double rkf_relerr; /* per-pair RKF tolerances (bia/find_dXYUV_RKF.f90:4): 0 ... */
    double rkf_abserr; /* ... and 1e-16 */
    int deterministic; /* 1: fixed-order two-pass reduction (bitwise reproducible);
                          0: FP64 atomics (no scratch, order varies run to run) */
} bia_config;

/* fills cfg with the reference's defaults: ALG, ITR 18, eps_th -6e-7, dt 1,
   ERR 1e-12, RKF 0/1e-16, deterministic reduction */
void bia_config_default(bia_config *cfg);

/* per-step counters (pairs per branch of bia/bia.f90:158-166 and solver work) */
typedef struct bia_stats {
    long long hyperbola, parabola, ellipse, degenerate, rkf;
    long long universal;     /* pairs advanced by the universal-variable solver (ALG pairs
                                with |e^2 - 1| < 0.1, or every pair of BIA_METHOD_UNIVERSAL);
                                degenerate pairs (|g| = 0 or |L| = 0) are counted apart */
    long long iterations;    /* Newton iterations, summed over the classical ALG branches */
    long long iter_hyperbola, iter_ellipse, iter_parabola; /* the same split by branch */
    long long iter_universal; /* Newton iterations of the universal-variable solver */
    long long rkf_steps;     /* accepted RKF steps, summed over RKF pairs */
    long long nonconverged;  /* |residual| > cfg.err (bia/bia.f90:151,167) */
    long long bracket_exits; /* hyperbola iterate left (-theta_0, theta_0) */
    long long fallbacks;     /* classical iteration ended unconverged: bracketed re-solve */
    long long nonfinite;     /* pairs whose displacement was not finite */
    long long learned;       /* BIA_METHOD_LEARNED: pairs started from a learned head */
    long long learned_fallbacks; /* ... of which the FP64 step did not settle: plain solve */
    long long learned_coarse;    /* ... whose head guess was > 1e-2 off in anomaly */
    long long timeouts;      /* bounded tensor-core waits that gave up (the step returns
                                BIA_ERR_DEVICE_TIMEOUT) */
    long long learned_fp32_steps; /* FP32 Newton steps of the learned pairs' first correction
                                     (each learned pair then takes one FP64 Halley step) */
} bia_stats;

typedef struct bia_context bia_context;

/* Create a context on `device` that launches on `stream` (a cudaStream_t, NULL =
   the legacy default stream).  The context owns scratch buffers, grown on demand. */
int bia_context_create(bia_context **ctx, int device, void *stream);
int bia_context_destroy(bia_context *ctx);
/* Autotuner: times the ALG pair-kernel shapes on this device state (the timed launches
   write only scratch; the state is unchanged) and keeps the fastest for this reduction mode
   and floor(log2 n) in the context, which later steps of that size then use.
   Shapes: 0 = 8-warp CTAs, 1 = phase-locked 32-warp CTAs (1 per SM) with per-lane class
   loops, 2 = the same with the balanced class loops (mixed classes; the default from two of
   its CTAs per SM up).  BIA_METHOD_LEARNED: 0 = one kernel, 1 = split (the plain pairs
   in a universal-variable kernel that defers the learned pairs' head inputs to rows and lists
   their warp-blocks, a persistent kernel that evaluates the rows on the tensor cores, and one
   that finishes the listed warp-blocks; the untuned default at every size).  variant (optional) receives the
   choice, ms (optional, 3 floats) the best time of each candidate (-1 when not run).  RKF
   and universal variables have one shape: variant = -1.
   Synchronises the context's stream; not during stream capture.  No counterpart in the
   reference. */
int bia_context_autotune(bia_context *ctx, const bia_config *cfg, int n, double *x, double *y,
                         double *z, double *u, double *v, double *w, const double *q,
                         int *variant, float *ms);
/* Pins the pair-kernel shape that later steps of this context take for `method`
   (BIA_METHOD_ALG or BIA_METHOD_LEARNED), reduction mode `deterministic` and sizes in n's
   floor(log2 n) bucket: what bia_context_autotune stores, for a caller that keeps an earlier
   tuning result; variant -1 restores the default rule.  The shapes of a method compute
   bitwise the same results.  No counterpart in the reference. */
int bia_context_set_shape(bia_context *ctx, int method, int deterministic, int n, int variant);
/* Self-test of the device-side bounded waits: a kernel waits on an mbarrier that nothing
   completes, gives up after its limit and reports it; returns BIA_ERR_DEVICE_TIMEOUT (the
   expected answer) and leaves the context usable.  No counterpart in the reference. */
int bia_selftest_wait_timeout(bia_context *ctx);
/* Loads the two learned Kepler heads of BIA_METHOD_LEARNED from the bytes of
   learned_heads.bin (bia_3d_gpu_b200/train_heads.py writes it: "BIAHEAD1", version 1,
   2 heads of 19472 bytes).  No counterpart in the reference (the learned form is new). */
int bia_context_set_heads(bia_context *ctx, const void *blob, size_t bytes);
/* Evaluates one learned head (0 elliptic, 1 hyperbolic) on n rows of 2 FP32 inputs
   (device arrays, in[2 n] -> out[n]) with the tensor-core kernels the learned step uses;
   for tests of the network path.  No counterpart in the reference. */
int bia_learned_head_eval(bia_context *ctx, int head, int n, const float *in, float *out);
int bia_context_set_stream(bia_context *ctx, void *stream);
/* kernel timing: when on, the pair kernel's launches are bracketed by CUDA events on
   the context's stream; bia_context_kernel_ms returns their summed duration and count
   since the last reset (synchronises the stream). */
int bia_context_set_timing(bia_context *ctx, int on);
int bia_context_kernel_ms(bia_context *ctx, double *ms, long long *launches);

/* Counters of every step enqueued on the context since the last reset (steps called
   with stats == NULL add to them; a call with stats != NULL reports and clears its own
   steps).  Synchronises the context's stream; reset != 0 clears them afterwards. */
int bia_context_stats(bia_context *ctx, bia_stats *stats, int reset);

/* One BIA step on device-resident SoA state (bia/bia.f90:126-204 as one launch
   sequence): all pairs i<j, per-particle reduction, drift, and the update
   X += dX, U += dU in place.  q: optional device array of n charges (NULL: eps_th
   for every pair).  disp: optional device array [6][n] receiving dX..dW (drift
   included, as in the .BIA record, bia/bia.f90:206).  stats: optional, host. */
int bia_step(bia_context *ctx, const bia_config *cfg, int n, double *x, double *y, double *z,
             double *u, double *v, double *w, const double *q, double *disp, bia_stats *stats);

/* nsteps BIA steps.  With use_graph != 0 the step sequence is captured once in a
   CUDA graph and replayed.  stats (optional) are summed over the steps. */
int bia_run(bia_context *ctx, const bia_config *cfg, int n, double *x, double *y, double *z,
            double *u, double *v, double *w, const double *q, int nsteps, int use_graph,
            bia_stats *stats);

/* Host-buffer form of bia_run: copies the host state (6 arrays of n) and charges to
   the device, runs nsteps steps, copies the state back into the same host arrays. */
int bia_run_host(bia_context *ctx, const bia_config *cfg, int n, double *x, double *y,
                 double *z, double *u, double *v, double *w, const double *q, int nsteps,
                 bia_stats *stats);

/* Multi-GPU step by shards (the path's exchange is the per-particle sum: one FP64
   all-reduce of 6n per step).  Shard `shard` of `nshards` owns the pairs (i, j), i < j, whose
   j lies in columns [c0, c1) of 32-particle blocks; bia_shard_columns gives them (about
   equal pair counts; no GPU needed).  bia_step_shard solves the shard's pairs on the context's
   device and writes their sums into the device array sums[6][n] (dX..dW without drift, the
   state unchanged); the caller adds the shards' sums across GPUs (an NCCL all-reduce) and
   then calls bia_apply_update, which adds the drift and updates the state
   (bia/bia.f90:194-204).  The shards of one step partition its pairs, so their sums add up to
   the whole step's (deterministic mode: the same planes in the same order per shard).  No
   counterpart in the reference, which runs on one GPU. */
int bia_shard_columns(int n, int shard, int nshards, int *c0, int *c1);
int bia_step_shard(bia_context *ctx, const bia_config *cfg, int n, double *x, double *y, double *z,
                   double *u, double *v, double *w, const double *q, int shard, int nshards,
                   double *sums, bia_stats *stats);
int bia_apply_update(bia_context *ctx, int n, double dt, double *x, double *y, double *z, double *u,
                     double *v, double *w, const double *sums);

/* Allocation-free form of bia_step, for callers that cannot allocate device memory once
   they run (a framework that owns the GPU's memory pool, a real-time loop that must not
   enter the CUDA allocator).  No counterpart in the reference.  The step's scratch is a
   fixed array inside the library (6 MiB per GPU that loads it, held until exit) instead
   of a bia_context, so n must be <= 2048; larger n returns BIA_ERR_INVALID_ARGUMENT.
   The caller passes device state (updated in place), optional charges q and optional
   disp [6][n]; kernels and one memset are enqueued on `stream` (a cudaStream_t, NULL =
   legacy default stream) and the call returns without synchronising.  The reduction is
   always the deterministic one (cfg->deterministic is ignored); no counters are returned.
   Every call made outside stream capture resolves the array's device address
   (cudaGetSymbolAddress, no allocation); a call during a capture uses the address of the
   last call outside it, so make the first call on a device before any stream capture.  All
   calls share the one array: calls whose work overlaps on the GPU (different streams, or
   host threads) race.  The status (also kept for bia_last_error) comes from the launch
   checks, so an asynchronous error left on the device by earlier work can surface here. */
int bia_step_noalloc(const bia_config *cfg, int n, double *x, double *y, double *z, double *u,
                     double *v, double *w, const double *q, double *disp, void *stream);

/* Invariants of device SoA state (bia/invariance.cu:50-110 semantics, FP64):
   out[11] = {KE, PE, Lx, Ly, Lz, Ua, Va, Wa, Xa, Ya, Za} on the host.
   KE = sum |v|^2, PE = eps_th * sum_{i<j} (q_i q_j) / r_ij. */
int bia_invariance(bia_context *ctx, int n, double eps_th, const double *x, const double *y,
                   const double *z, const double *u, const double *v, const double *w,
                   const double *q, double out[11]);

/* Measured FP64 FMA throughput of `device` in TFLOP/s (FMA = 2 flops): the roofline
   denominator of the FP64-bound pair kernel. */
int bia_measure_fp64_peak(int device, double *tflops);

/* Ensemble of independent systems of uneven size (no counterpart in the reference, which
   runs one system).  The systems are stored back to back in one set of device SoA arrays:
   system s owns particles [off_s, off_s + sizes[s]) with off_s = sizes[0] + ... +
   sizes[s-1], and has pair coupling eps[s] (times q_i q_j when charges are given).
   Create once (host arrays sizes[nsys], eps[nsys]); every step is one pair-kernel launch
   over all systems' 32 x 32 blocks plus one reduction launch, and each system's result
   equals a bia_step of that system alone (same per-block code and summation order). */
typedef struct bia_ensemble bia_ensemble;
int bia_ensemble_create(bia_context *ctx, int nsys, const int *sizes, const double *eps,
                        bia_ensemble **ens);
int bia_ensemble_destroy(bia_ensemble *ens);
long long bia_ensemble_particles(const bia_ensemble *ens);
/* nsteps steps of every system (cfg->eps_th is ignored: each system has its own eps);
   with use_graph != 0 and a non-default stream the sequence is captured in a CUDA graph */
int bia_ensemble_run(bia_context *ctx, bia_ensemble *ens, const bia_config *cfg, double *x,
                     double *y, double *z, double *u, double *v, double *w, const double *q,
                     int nsteps, int use_graph, bia_stats *stats);
/* Autotuner of the ensemble's pair-kernel launch shape for cfg->method, timed on these
   systems (1 warm-up and 3 timed launches per shape; only scratch is written, the state is
   unchanged); the fastest is kept in the ensemble and used by later runs.  Shapes: ALG 0 =
   8-warp CTAs, 1 = phase-locked 32-warp CTAs (1 per SM) with per-lane class loops, 2 = the
   same with the balanced class loops; universal variables 0 = one item per warp, 1 = a persistent grid (2 CTAs per
   SM); learned 0 / 1 = the persistent head kernel (the deferred pairs' rows on the tensor
   cores) at 1 / 2 CTAs per SM.  Every shape gives
   bitwise the same results.  variant (optional): the choice (-1 for RKF, one shape); ms
   (optional, 3 floats): each shape's best time (-1 when not run).  Synchronises the
   context's stream; not during stream capture.  No counterpart in the reference. */
int bia_ensemble_autotune(bia_context *ctx, bia_ensemble *ens, const bia_config *cfg, double *x,
                          double *y, double *z, double *u, double *v, double *w, const double *q,
                          int *variant, float *ms);
/* per-system KE and PE (energy[2 s] = sum |v|^2, energy[2 s + 1] = eps_s sum (q_i q_j)/r_ij),
   host array of 2 nsys doubles; synchronises */
int bia_ensemble_energy(bia_context *ctx, bia_ensemble *ens, const double *x, const double *y,
                        const double *z, const double *u, const double *v, const double *w,
                        const double *q, double *energy);

/* Device trainer of one learned head (0 elliptic, 1 hyperbolic), the training of
   BIA_METHOD_LEARNED's heads on the GPU.  No counterpart in the reference (the learned form
   is new).  Create draws nsamples (eccentricity, mean anomaly) pairs uniformly over the
   head's domain from `seed` (counter-based), solves Kepler's equation for each in FP64 on
   the device, and initialises the FP32 master parameters from `seed` (uniform in
   +-1/sqrt(fan_in)).  Training steps run forward and backward on the tensor cores (BF16
   operands, FP32 accumulation in tensor memory) and Adam on the device; results are the
   same for the same seed.  Parameters (FP32, bia_trainer_param_count() of them) are ordered
   W1[64][2], b1[64], W2[64][64], b2[64], W3[64][64], b3[64], w4[64], b4 (weights
   output-major).  The trainer works on the context's device and on the stream the context
   had when the trainer was created; every call synchronises that stream. */
typedef struct bia_trainer bia_trainer;
int bia_trainer_create(bia_context *ctx, int head, long long nsamples, unsigned long long seed,
                       bia_trainer **trainer);
int bia_trainer_destroy(bia_trainer *trainer);
int bia_trainer_param_count(void);
int bia_trainer_get_params(bia_trainer *trainer, float *params);
/* replaces the parameters (host array) and clears the Adam state */
int bia_trainer_set_params(bia_trainer *trainer, const float *params);
/* gradient of the mean squared error over `rows` device rows x[rows][2] -> y[rows] at the
   current parameters, no update: grad (host, param_count floats), loss (host, optional) */
int bia_trainer_gradient(bia_trainer *trainer, const float *x, const float *y, int rows,
                         float *grad, float *loss);
/* `epochs` passes of Adam (beta 0.9 / 0.999, eps 1e-8) over the samples in batches of
   `batch` rows (a multiple of 128 dividing nsamples, which must be a power of two; each
   epoch visits the samples in its own permuted order), learning rate lr annealed by a
   cosine over the epochs; loss_per_epoch (host, optional): the epoch's mean squared error */
int bia_trainer_train(bia_trainer *trainer, int epochs, int batch, float lr, float *loss_per_epoch);
/* the head as a learned_heads.bin record (19472 bytes: BF16 weights, FP32 vectors) */
int bia_trainer_export(bia_trainer *trainer, void *record);
/* the device arrays of the samples: x[n][2] (the head's inputs), y[n] (target / scale) */
int bia_trainer_samples(bia_trainer *trainer, const float **x, const float **y, long long *n);
/* host copies of samples first .. first + count - 1: x[count][2], y[count] */
int bia_trainer_copy_samples(bia_trainer *trainer, long long first, long long count, float *x, float *y);

/* Direct-integration (DIM) reference solver: rebuilds rkf_c_ (dim/rkf_kernel.cu:194-495).
   y: device state, 6 arrays of n (x, y, z, u, v, w), advanced in place from x0 to xe with
   a_i = eps_th * sum_j (r_i - r_j) / (|r_ij|^2 + 1e-99)^{3/2} (per-particle coupling as in
   dim/dim_3D.f90:9, i.e. half the BIA pair coupling) by adaptive RKF4(5) with step
   doubling (the returned state is the two-half-step track).  BIA_ERR_NOT_CONVERGED when
   ier != 0 (then y holds the last accepted state). */
typedef struct bia_dim_stats {
    long long accepted, rejected; /* steps */
    int nde;                      /* derivative evaluations, as the reference's NDE */
    int ier;                      /* 0, 10000 (too many steps), 20000, 30000 (step underflow) */
    double h_last, x_reached;
} bia_dim_stats;
int bia_dim_integrate(bia_context *ctx, int n, double eps_th, double *y, double x0, double xe,
                      double relerr, double abserr, bia_dim_stats *stats);

const char *bia_status_string(int status);
/* status of the last drop-in call (find_dxyuv_kernel_, invariance_gpu_, rkf_c_) on this
   host thread */
int bia_last_error(void);

/* ---- drop-in replacements of the reference's symbols ----------------------- */

/* Replaces find_dxyuv_kernel_ (bia/find_dXYUV_kernel.cu:526-561), called from
   bia/bia.f90:135,138.  For the fixed particle I (1-based) and every j > I it solves
   the pair given by the host AoS array RXYZUVW[6N] of x_i-x_j, ..., w_i-w_j, writes
   the half-displacements into the host array dXYZUVW[6j..6j+5] (entries j <= I are
   set to 0), and accumulates them into the host arrays: dX[I] += h_j, dX[j] -= h_j
   (likewise dY..dW).  No drift is added (the caller does, bia/bia.f90:194-196).
   METHOD: 0 = RKF, 1 = ALG. */
void find_dxyuv_kernel_(const int METHOD, const int N, const int I, const double EPS,
                        const double DT, const int ITR, double *dX, double *dY, double *dZ,
                        double *dU, double *dV, double *dW, double *RXYZUVW, double *dXYZUVW);

/* Replaces invariance_gpu_ (bia/invariance.cu:50-110), called from bia/bia.f90:67-68:
   host SoA arrays in, the 11 invariants out through scalar pointers. */
void invariance_gpu_(const int N, const double eps_th, double *X, double *Y, double *Z,
                     double *U, double *V, double *W, double *KE, double *PE, double *Lx,
                     double *Ly, double *Lz, double *Ua, double *Va, double *Wa, double *Xa,
                     double *Ya, double *Za);

/* Replaces rkf_c_ (dim/rkf_kernel.cu:194-495), called from dim/dim_3D.f90:30 as
   RKF_C(%VAL(NEQ), %VAL(eps_th), X0, XE, Y0, INIT, RELERR, ABSERR, YN, ESTERR, NDE, IER,
   WK0, WK1, WK2, WK3, WK4): host AoS state YH0[neq] at *X0 is integrated to *XE on the
   device; YHN receives the result, ESE (yln - yhn)/31, NDE the derivative evaluations,
   IER 0 / 10000 / 20000 / 30000, *H the last step, *X0 = *XE, *INIT = 2, YH0 and YL0 the
   final tracks, YLN and ERR the last low-track state and error.  On trouble it returns
   with IER set instead of calling exit(0); WRK is not written. */
void rkf_c_(const int neq, const double eps_th, double *X0, double *XE, double *YH0, int *INIT,
            const double *RELERR, const double *ABSERR, double *YHN, double *ESE, int *NDE,
            int *IER, double *H, double *YL0, double *YLN, double *ERR, double *WRK);

#ifdef __cplusplus
}
#endif
#endif /* BIA_CAPI_H */
