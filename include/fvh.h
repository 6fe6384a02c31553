/*
 * fvh.h -- C ABI of the B200 per-stage update for the compressible Euler
 * equations (high-order finite-volume reconstruction, HLLC/LLF/upwind Riemann
 * fluxes, a-posteriori NAD/PAD troubled-cell detection with a MUSCL fallback,
 * and SSP-RK stage accumulation).
 *
 * The library behind this header replaces the NumPy/CuPy hot path of
 * jpalafou/FVHOE. Each entry point names the reference interface it stands in
 * for (paths inside that project).
 *
 * Conventions
 *  - Every call returns an int status: FVH_OK (0) or a negative FVH_ERR_*.
 *    fvh_last_error() gives the message of the last failure (per handle, or
 *    process-wide for fvh_create). No C++ exception crosses this boundary.
 *  - State arrays are float64, layout (nvars, nx, ny, nz), C order (z
 *    contiguous), exactly the reference's `u` (fvhoe/solver.py:410-420).
 *    Pointers passed to the compute calls are DEVICE pointers; the caller
 *    owns them. The library owns its scratch memory, allocated by fvh_create
 *    and released by fvh_destroy.
 *  - `stream` is a cudaStream_t passed as void*; NULL is the legacy default
 *    stream. All work is ordered on that stream. Only the optional dt/host
 *    read-backs synchronise it.
 *  - A handle is not thread-safe; use one handle per solver and thread.
 */
#ifndef FVH_H
#define FVH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FVH_ABI_VERSION 3

/* status codes */
#define FVH_OK 0
#define FVH_ERR_CONFIG -1    /* invalid or unsupported configuration */
#define FVH_ERR_CUDA -2      /* a CUDA runtime call failed */
#define FVH_ERR_TIMEOUT -3   /* a bounded device-side wait gave up */
#define FVH_ERR_NONFINITE -4 /* the update produced NaN/Inf values */
#define FVH_ERR_ARG -5       /* invalid argument (null pointer, bad enum) */

/* boundary kinds (fvhoe/boundary_conditions.py:357-373) */
#define FVH_BC_PERIODIC 0
#define FVH_BC_OUTFLOW 1 /* mirror */
#define FVH_BC_REFLECTIVE 2 /* mirror, normal momentum negated */
#define FVH_BC_FREE 3 /* repeat the edge cell */
#define FVH_BC_DIRICHLET 4 /* ghost values given by the caller ("dirichlet" and "ic") */
/* "special-case-double-mach-reflection-y=0" (fvhoe/boundary_conditions.py:374-395),
   low y side only: a ghost column whose x index is below dmr_split repeats the
   edge cell (free), the others mirror with the y momentum negated (reflective) */
#define FVH_BC_DMR_Y0 5

/* Riemann solvers (fvhoe/solver.py:185-193) */
#define FVH_RIEMANN_HLLC 0
#define FVH_RIEMANN_LLF 1
#define FVH_RIEMANN_ADVECTION_UPWIND 2

/* slope limiters of the fallback scheme (fvhoe/slope_limiting.py:40-48) */
#define FVH_LIMITER_MINMOD 0
#define FVH_LIMITER_MONCEN 1
#define FVH_LIMITER_NONE 2

/* precision modes */
#define FVH_PREC_FP64 0 /* every operation in float64, reference evaluation order, no FMA contraction */
#define FVH_PREC_FP32 1 /* reconstruction, Riemann fluxes, detection in float32; float64 stage accumulation
                           (SSP-RK3 in the Shu-Osher form, which writes no k-sum) */

/* time integrators (fvhoe/ode.py:245-298) */
#define FVH_INT_EULER 0
#define FVH_INT_SSPRK2 1
#define FVH_INT_SSPRK3 2
#define FVH_INT_RK4 3

typedef struct fvh_config {
  int abi_version;   /* FVH_ABI_VERSION */
  int nvars;         /* 5 + number of passive scalars (<= 16) */
  int n[3];          /* cells along x, y, z; an axis with n = 1 and p = 0 is inactive */
  int p[3];          /* polynomial degree per axis, 0..8 */
  double h[3];       /* cell widths */
  double gamma;      /* specific heat ratio */
  double cfl;        /* Courant number */
  double csq_floor;  /* floor on the squared sound speed */
  int use_fixed_dt;  /* 1: use fixed_dt instead of the CFL step */
  double fixed_dt;
  int riemann;       /* FVH_RIEMANN_* */
  int bc[3][2];      /* FVH_BC_* at the low/high end of each axis */
  int a_posteriori;  /* 1: NAD/PAD detection with the fallback scheme */
  int slope_limiter; /* FVH_LIMITER_* */
  int force_trouble; /* 1: every cell is troubled */
  double nad_eps;    /* NAD tolerance */
  int nad_global;    /* 1: "global" range, 0: "local" */
  int nad_relative;  /* 1: "relative" range, 0: "absolute" */
  int nad_var_mask;  /* bit v (0..4) set: primitive v takes part in NAD */
  int pad_var;       /* primitive index checked by PAD, or -1 for none */
  double pad_lo;
  double pad_hi;
  int sed;           /* 1: smooth-extrema detection relaxes NAD */
  double sed_eps;
  int convex;        /* 1: convex face weights (1D/2D only) */
  int precision;     /* FVH_PREC_* */
  int log_troubles;  /* 1: keep the running trouble / NAD / PAD sums used by snapshots */
  int device;        /* CUDA device ordinal the handle's memory and kernels live on */
  int kernel_path;   /* FVH_PATH_*: which kernel family runs the stage */
  int dmr_split;     /* FVH_BC_DMR_Y0: first x index (ghosts negative) whose cell centre is >= 1/6 */
} fvh_config;

/* kernel families (identical results in FP64) */
#define FVH_PATH_AUTO 0    /* fused 2D tiles when eligible, else the generic passes */
#define FVH_PATH_GENERIC 1 /* generic N-D passes, any configuration */
#define FVH_PATH_FUSED2D 2 /* fused 2D tiles; fvh_create refuses ineligible configurations */

typedef struct fvh_handle fvh_handle;

/* Stage statistics of the last call. */
typedef struct fvh_stats {
  double dt_stage;       /* dt of the last stage (CFL or fixed) */
  double dt_step;        /* dt of the last step after the target clamp */
  unsigned int troubled; /* troubled cells in the last stage */
  unsigned int nonfinite;/* non-finite values written by the last stage */
} fvh_stats;

/* Fills *cfg with the reference's defaults (fvhoe/solver.py:42-84):
 * gamma 5/3, CFL 0.8, HLLC, periodic, NAD 1e-2 global relative on all
 * variables, PAD on P >= 0 (the last key of the default PAD dict), SED on
 * with tolerance 1e-10, minmod, csq_floor 1e-10, FP64. */
void fvh_config_default(fvh_config* cfg);

/* Validates cfg and allocates the scratch memory of one solver on the current
 * CUDA device. Replaces the array allocation of EulerSolver.__init__
 * (fvhoe/solver.py:402-420) for the "cuda" backend. */
int fvh_create(const fvh_config* cfg, fvh_handle** out);

/* Releases a handle and its scratch memory. NULL is accepted. */
int fvh_destroy(fvh_handle* h);

/* Message of the last failure on h, or of the last failed fvh_create when h
 * is NULL. Never NULL. */
const char* fvh_last_error(const fvh_handle* h);

/* Bytes of device scratch memory held by the handle. */
size_t fvh_scratch_bytes(const fvh_handle* h);

/* One right-hand-side evaluation: dudt = L(u) and the CFL time step of this
 * evaluation. Replaces EulerSolver.f / hydrodynamics (fvhoe/solver.py:422-454)
 * including revise_fluxes (:653-732) and euler_equation (:734-751).
 * u, dudt: device arrays of nvars * nx * ny * nz doubles. dt_out: host
 * pointer or NULL; when given, the call synchronises the stream and returns
 * FVH_ERR_NONFINITE (with *dt_out written) when dudt holds NaN/Inf values or
 * dt is not finite or not positive. */
int fvh_rhs(fvh_handle* h, const double* u, double* dudt, double* dt_out, void* stream);

/* One time step of the chosen integrator, updating u in place. The first
 * stage's dt is shortened to target - t when has_target is set and the target
 * is closer (fvhoe/ode.py:11-22). Replaces ODE.take_step with the stepper of
 * ODE.euler/ssprk2/ssprk3/rk4 (fvhoe/ode.py:183-193, 245-298).
 * dt_out: host pointer or NULL (when given, the stream is synchronised and
 * the call returns FVH_ERR_NONFINITE, with *dt_out written, when the step
 * wrote NaN/Inf values or its dt is not finite or, for a CFL dt, not
 * positive; fvh_get_stats reports the count either way). With
 * dt_out = NULL the call makes no host synchronisation and can be captured in
 * a CUDA graph after one uncaptured call of the same handle; each replay
 * computes its own dt on the device and reuses the captured t, target and
 * trouble-log mode, so capture steps without a target (or with a fixed one). */
int fvh_step(fvh_handle* h, double* u, int integrator, double t, int has_target, double target, double* dt_out,
             void* stream);

/* One stage k (0-based) of a step of the chosen integrator, on the caller's
 * stream: the right-hand-side evaluation of the stage's input and its
 * Runge-Kutta combination, as one stage of the steppers of fvhoe/ode.py:245-298
 * (for SSP-RK3, one self.f call of ode.py:274-280 and the sum that follows it).
 * Stage 0 reads u and fixes the step's dt (CFL, then the target clamp, as in
 * fvh_step); stage k > 0 reads the handle's stage buffer written by stage k-1;
 * the last stage writes u in place. Stages of one step must be called in
 * order, with the same integrator and u (a stage 0 call starts a new step);
 * the stages of a step equal one fvh_step call bit for bit. dt_out: the step's
 * dt, as for fvh_step (NULL: no synchronisation). */
int fvh_stage(fvh_handle* h, double* u, int integrator, int k, double t, int has_target, double target,
              double* dt_out, void* stream);

/* fvh_step for a state held in page-locked host memory (cudaHostAlloc or
 * cudaHostRegister), as the reference holds u in host NumPy arrays: the call
 * copies u_host in, steps it and copies the result back to u_host, all queued
 * on the handle's two copy streams and the caller's stream. Both copies run in
 * 16 contiguous chunks, and chunk j of a call's copy-in waits only for chunk j
 * of the previous call's copy-out, so on a full-duplex link one step's
 * copy-out overlaps the next step's copy-in. The call returns once the work is
 * queued (after the step when dt_out is given, which synchronises the caller's
 * stream only); u_host must not be read or written until fvh_host_sync(h)
 * returns. The device copy (nvars * nx * ny * nz doubles) and the streams are
 * made on the first call and counted by fvh_scratch_bytes. No counterpart in
 * the reference, whose state never leaves the host. */
int fvh_step_host(fvh_handle* h, double* u_host, int integrator, double t, int has_target, double target,
                  double* dt_out, void* stream);
/* Waits for the copy-out of the last fvh_step_host call. */
int fvh_host_sync(fvh_handle* h);

/* Finite-volume primitive averages (fv_average = 1) or cell-centre primitives
 * (fv_average = 0) of u over the interior, written to w (same shape).
 * Replaces interpolate_primitives_from_conservatives with gw = 0
 * (fvhoe/solver.py:753-792) as called by snapshot (:840-874). */
int fvh_primitives(fvh_handle* h, const double* u, double* w, int fv_average, void* stream);

/* Allocation-free fvh_primitives, with no counterpart in the reference. For
 * callers that cannot allocate device memory when they convert (a host
 * application owning the device memory pool, or a run that has committed the
 * whole device to its state): no handle, no cudaMalloc; the two sweep buffers
 * come from a 16 MiB static device array that every GPU loading this library
 * holds until exit. cfg is checked as by fvh_create; grids needing more than
 * fvh_primitives_noalloc_max_doubles() doubles per buffer
 * (nvars * prod(n_a + 4 ceil(p_a/2)) over the active axes) are refused with
 * FVH_ERR_CONFIG, and so are Dirichlet and FVH_BC_DMR_Y0 sides, whose
 * ghost values live in a handle. Every refusal is decided on the host before
 * u or w is used. The first call on a device resolves the array's address
 * (make it before any stream capture) and keeps it for the life of the
 * process, so do not use this library across cudaDeviceReset. All calls share
 * the array: calls whose work overlaps on the GPU race.
 * Errors: fvh_primitives_noalloc_error(). */
int fvh_primitives_noalloc(const fvh_config* cfg, const double* u, double* w, int fv_average, void* stream);
size_t fvh_primitives_noalloc_max_doubles(void);
const char* fvh_primitives_noalloc_error(void);

/* Ghost values of a Dirichlet side (FVH_BC_DIRICHLET: the reference's
 * "dirichlet" and "ic" kinds, fvhoe/boundary_conditions.py:18-55, 334-347).
 * The layout of side (axis, side): nvars x ext[0] x ext[1] x ext[2] doubles,
 * ext[axis] = *depth ghost layers ordered outward-in on the low side
 * (cell -depth first) and inward-out on the high side (cell n first), the other
 * active axes spanning their interior plus `depth` ghost layers on each side
 * (ext = n + 2 * depth), inactive axes 1. The reference evaluates its boundary
 * functions at these cells' centres once per step (t = the step's start time);
 * the caller does the same and uploads with fvh_set_boundary_values (host or
 * device pointer) before the step. */
int fvh_boundary_layout(fvh_handle* h, int axis, int side, int* depth, int* ext, size_t* count);
int fvh_set_boundary_values(fvh_handle* h, int axis, int side, const double* values, void* stream);

/* Copies the trouble flags of the last stage (uint8, nx*ny*nz) to the device
 * array flags. Replaces the troubled_cells array of revise_fluxes
 * (fvhoe/solver.py:691-706). */
int fvh_trouble_flags(fvh_handle* h, uint8_t* flags, void* stream);

/* Running trouble / NAD / PAD sums of log_troubles (fvhoe/solver.py:794-833).
 * divide_by > 0 divides the sums in place first (the reset branch of
 * log_troubles); each destination may be NULL. Destinations are device arrays
 * of nx*ny*nz doubles. */
int fvh_trouble_log(fvh_handle* h, double divide_by, double* trouble, double* nad_mag, double* pad_mag,
                    void* stream);

/* Selects how the next stage writes the trouble log: 1 overwrites the sums,
 * 2 adds to them (the two branches of log_troubles, fvhoe/solver.py:821-833). */
int fvh_set_log_mode(fvh_handle* h, int mode);

/* Makes the last stage of the next fvh_step divide the running sums by
 * divisor after adding its values: the reset branch of log_troubles
 * (fvhoe/solver.py:809-820) that the reference runs after every step, done in
 * the detection pass instead of in a separate one (fvh_trouble_log with
 * divide_by). 0 = no division. Applies to one fvh_step. */
int fvh_set_log_divisor(fvh_handle* h, double divisor);

/* Statistics of the last stage; synchronises the stream. */
int fvh_get_stats(fvh_handle* h, fvh_stats* out, void* stream);

/* Kernel kinds reported by fvh_profile_read. The per-launch timing replaces
 * the wall-clock categories of the reference's Timer (fvhoe/timer.py:6-109,
 * categories registered at fvhoe/solver.py:204-218). */
#define FVH_KK_CENTRE 0     /* centre-interpolation sweeps (ghost fill, primitives) */
#define FVH_KK_TRANSVERSE 1 /* transverse-reconstruction sweeps (CFL / extrema reductions) */
#define FVH_KK_FACE 2       /* face states + Riemann solve */
#define FVH_KK_CANDIDATE 3  /* unlimited candidate update */
#define FVH_KK_DETECT 4     /* troubled-cell detection */
#define FVH_KK_FALLBACK 5   /* MUSCL fallback + blend */
#define FVH_KK_FINAL 6      /* flux divergence + Runge-Kutta combination */
#define FVH_KK_SMALL 7      /* stage scalars, convex weights, log arithmetic */
#define FVH_KK_PREDICT 8    /* learned troubled-cell predictor (inference) */
#define FVH_KK_COUNT 9

/* Total kernel launches issued by this library in this process. */
uint64_t fvh_kernel_launches(void);

/* on = 1: time every launch made for h with a CUDA event pair (a few
 * microseconds of overhead per launch); on = 0: stop timing. */
int fvh_profile_enable(fvh_handle* h, int on);

/* Synchronises the stream, then writes per kernel kind (arrays of
 * FVH_KK_COUNT, each may be NULL) the milliseconds, the bytes each launch must
 * move (inputs read once, outputs written once) and the launch counts
 * accumulated since the previous read, and clears them. */
int fvh_profile_read(fvh_handle* h, double* ms, double* bytes, uint64_t* launches, void* stream);

/* ------------------------------------------------------------------------
 * Learned troubled-cell predictor (no counterpart in the reference, whose
 * troubled cells come only from the a-posteriori check,
 * fvhoe/solver.py:653-732). A 100 -> 64 -> 64 -> 1 GELU network over the 5x5
 * neighbourhood of (rho, v_X, v_Y, P) of each cell of a 2D grid, run on the
 * tensor cores (BF16 operands, FP32 accumulation). Attached to a handle, it
 * runs on the stage's primitives before the high-order fluxes; faces next to
 * a predicted cell take the MUSCL fallback flux in the flux pass, the
 * a-posteriori check still runs on every cell and the final pass revises the
 * faces of troubled cells the network missed. The update is then the
 * reference's with the fallback applied on (troubled | predicted) cells.
 * Features: for each variable and offset (a, b) in [-2, 2]^2,
 * d = w(x+a, y+b) - w(x, y), f = sign(d) log1p(|d| / (1e-5 R)) / log1p(1e5),
 * R = the variable's range over the stage (the global NAD extrema), stored as
 * 112 BF16 values per row (12 zero columns). Parameters: FP32, W1[64][100],
 * b1[64], W2[64][64], b2[64], w3[64], b3 (both matrices output-major).
 * ------------------------------------------------------------------------ */
typedef struct fvh_mlp fvh_mlp;

#define FVH_MLP_FEATURES 100
#define FVH_MLP_ROW 112 /* BF16 values per stored feature row */

/* Number of FP32 parameters (10689). */
size_t fvh_mlp_param_count(void);

/* Creates a network on a device with seeded He-normal weights, zero biases. */
int fvh_mlp_create(int device, uint64_t seed, fvh_mlp** out);
int fvh_mlp_destroy(fvh_mlp* m);
/* Message of the last failure on m (or of fvh_mlp_create when m is NULL). */
const char* fvh_mlp_last_error(const fvh_mlp* m);

/* Host copies of the FP32 parameters; set also resets the Adam moments. */
int fvh_mlp_get_params(fvh_mlp* m, float* host, size_t n);
int fvh_mlp_set_params(fvh_mlp* m, const float* host, size_t n);

/* Training rows from a handle's last stage (fused 2D path, a-posteriori with
 * global NAD): X (device, nx*ny rows of FVH_MLP_ROW BF16 bit patterns) and
 * the a-posteriori flags y (device, nx*ny bytes), row-major over (x, y). */
int fvh_mlp_features(fvh_handle* h, uint16_t* X, uint8_t* y, void* stream);

/* One Adam step (beta 0.9 / 0.999, eps 1e-8) on the mean binary cross-entropy
 * with logits over n device rows, positives weighted by pos_weight;
 * loss_out (host, may be NULL) receives the batch mean loss before the
 * update and synchronises the stream. */
int fvh_mlp_train_step(fvh_mlp* m, const uint16_t* X, const uint8_t* y, int n, float lr, float pos_weight,
                       float* loss_out, void* stream);

/* Gradients of that loss (device array of fvh_mlp_param_count() floats) and
 * the loss (host, may be NULL; synchronises), without an update. */
int fvh_mlp_gradients(fvh_mlp* m, const uint16_t* X, const uint8_t* y, int n, float pos_weight, float* grads_out,
                      float* loss_out, void* stream);

/* Logits of n device rows into the device array logits. */
int fvh_mlp_logits(fvh_mlp* m, const uint16_t* X, int n, float* logits, void* stream);

/* Tensor-core completion waits that reached their bound (0 when healthy). */
unsigned int fvh_mlp_errors(fvh_mlp* m);

/* Attaches m to h (NULL detaches); cells whose predicted probability exceeds
 * threshold are flagged. Needs the fused 2D path, a-posteriori limiting with
 * global NAD and a network on h's device; m must outlive the attachment. */
int fvh_set_predictor(fvh_handle* h, fvh_mlp* m, float threshold);

/* Runs the attached predictor every `stages` fused stages (default 1, every
 * stage) and reuses its flags in the stages between; the a-posteriori check
 * still judges every cell of every stage and revises the misses. Attaching a
 * predictor restarts the count. No counterpart in the reference (its detector
 * has no predictor). */
int fvh_set_predictor_interval(fvh_handle* h, int stages);

/* Predictor counts of the last step, summed over its stages. The two face
 * counts are kept by the fused 2D path with or without a predictor: faces
 * whose flux the final pass revised (the faces of troubled cells; with a
 * predictor, those of the cells it missed) and faces that took the fallback
 * flux in the flux pass (those of predicted cells). */
typedef struct fvh_pred_stats {
  unsigned int predicted;   /* cells the network flagged */
  unsigned int troubled;    /* cells the a-posteriori check flagged */
  unsigned int missed;      /* troubled, not predicted */
  unsigned int false_alarm; /* predicted, not troubled */
  unsigned int revised_faces;       /* faces revised by the final pass */
  unsigned int flux_fallback_faces; /* faces given the fallback flux by the flux pass */
} fvh_pred_stats;

/* Synchronises the stream. */
int fvh_get_pred_stats(fvh_handle* h, fvh_pred_stats* out, void* stream);

/* Copies the predicted flags of the last stage (uint8, nx*ny*nz) to the device
 * array flags. */
int fvh_pred_flags(fvh_handle* h, uint8_t* flags, void* stream);

/* ------------------------------------------------------------------------
 * Batched ensemble (no counterpart in the reference, which advances one
 * problem per EulerSolver, fvhoe/ode.py:94-174): independent 2D problems that
 * share every setting of cfg except the grid advance together, one
 * cooperative persistent launch per SSP-RK3 stage over a work list of
 * (problem, tile) entries, a whole step captured in a CUDA graph. Each member
 * takes its own CFL dt, clamped to the common target, and stops when it
 * reaches it, exactly as EulerSolver.ssprk3(t_end) does (fvhoe/ode.py:11-22,
 * 94-112); an FP64 member equals the same problem run alone, bit for bit.
 * cfg: the shared settings (cfg.n and cfg.h[0..1] are ignored; x and y must
 * be active, five variables, equal p in 1..8 on x and y, no convex weights,
 * no Dirichlet or FVH_BC_DMR_Y0 sides).
 * ------------------------------------------------------------------------ */
typedef struct fvh_ensemble fvh_ensemble;

int fvh_ensemble_create(const fvh_config* cfg, int nprob, const int* nx, const int* ny, const double* hx,
                        const double* hy, fvh_ensemble** out);
int fvh_ensemble_destroy(fvh_ensemble* e);
const char* fvh_ensemble_last_error(const fvh_ensemble* e);
/* Device memory held by the ensemble (states and scratch). */
size_t fvh_ensemble_bytes(const fvh_ensemble* e);
/* Device pointer of member q's state, float64 (5, nx, ny); NULL for a bad q.
 * Fill it before fvh_ensemble_reset / fvh_ensemble_step. */
double* fvh_ensemble_state(fvh_ensemble* e, int q);
/* Copies member q's state from src / to dst (host or device pointers of
 * 5 * nx * ny doubles); store synchronises the stream. */
int fvh_ensemble_load(fvh_ensemble* e, int q, const double* src, void* stream);
int fvh_ensemble_store(fvh_ensemble* e, int q, double* dst, void* stream);
/* Every member to time t0 with target t_end (active while t < t_end);
 * synchronises the stream. */
int fvh_ensemble_reset(fvh_ensemble* e, double t0, double t_end, void* stream);
/* nsteps SSP-RK3 steps of every active member, stream-ordered after the
 * caller's prior work on stream; no host synchronisation. */
int fvh_ensemble_step(fvh_ensemble* e, int nsteps, void* stream);
/* Per-member times and step counts (host arrays of nprob, each may be NULL),
 * the number of active members and the non-finite values written since the
 * reset; synchronises. FVH_ERR_TIMEOUT when a grid-barrier wait ran out. */
int fvh_ensemble_status(fvh_ensemble* e, double* t, int* steps, int* active, unsigned int* nonfinite,
                        void* stream);
/* Tile shape variant (0..2 of fvh_ensemble_variant_info), resident blocks per
 * SM of the persistent kernel (0 = as many as fit) and whether steps replay a
 * captured CUDA graph. */
int fvh_ensemble_configure(fvh_ensemble* e, int variant, int blocks_per_sm, int use_graph);
int fvh_ensemble_variant_info(fvh_ensemble* e, int variant, int* tx, int* ty, int* max_blocks_per_sm,
                              size_t* smem_bytes);
/* Bound of the grid-barrier waits between the phases of a stage, in polls of
 * about 64 ns each (0 restores the default, 2^24 polls). A wait that runs out
 * raises an abort flag that every block checks at its next barrier, so all
 * blocks return; fvh_ensemble_status then reports FVH_ERR_TIMEOUT until
 * fvh_ensemble_reset clears it. Used by tests to show that a stalled stage
 * ends with a status instead of a hang. */
int fvh_ensemble_set_wait_limit(fvh_ensemble* e, unsigned int polls);
/* Times `steps` steps of every variant and block count on the ensemble's own
 * data (restoring states and times after each trial) and keeps the fastest. */
int fvh_ensemble_autotune(fvh_ensemble* e, int steps, int* variant_out, int* blocks_out, double* ms_per_step,
                          void* stream);
/* Whether steps replay a CUDA graph, and why not when capture failed. */
int fvh_ensemble_graph_info(const fvh_ensemble* e, int* in_use, const char** error);

#ifdef __cplusplus
}
#endif

#endif /* FVH_H */
