/*
 * ibpm_b200.h -- C ABI of libibpm_b200.so, a CUDA (sm_100a) implementation of
 * ImmersedBodies.jl's CNAB/IBPM time step.
 *
 * The entry points are what a Julia `AbstractSolver` (src/solver.jl:6-28)
 * binds with `ccall` (the module immersedbodies.jl_b200/julia/ImmersedBodiesCUDA.jl).
 *
 *   reference interface                         replaced by
 *   ------------------------------------------  -------------------------------
 *   CnabSolver(state; fftw, cg)                 ibpm_create + ibpm_set_state
 *     src/solver.jl:84-150, 152
 *   advance!(::CnabSolver) src/solver.jl:155    ibpm_advance
 *   getstate(::CnabSolver) src/solver.jl:153    ibpm_get_state (lazy copy-back)
 *   update_vars!/boundary_total_force           ibpm_get_forces
 *     src/problem.jl:676-685, 853-856
 *   error("Panel index=... outside allowed      IBPM_ERR_REGION + ibpm_last_error
 *     region") src/coupling.jl:39-41
 *   save_state/load_state src/io/io.jl:14-71    ibpm_get_state/ibpm_set_state
 *                                               (same arrays, same layouts)
 *
 * Arrays are FP64 in the reference's Julia layouts (column-major, x fastest):
 *   q, q0      : nq x nlevel, nq = (nx+1)*ny + nx*(ny+1)  (u block, then v block)
 *   gamma, psi : ng x nlevel, ng = (nx-1)*(ny-1)
 *   nonlin1/2  : ng x nlevel   (state.nonlin[1], state.nonlin[2])
 *   xb, ub     : npanel x 2,  ds : npanel,  fbt : 2*npanel (state.F̃b),  fb : npanel x 2
 * Caller buffers are copied in or out during the call and never retained.
 * The library owns all device memory and one CUDA stream per handle.
 * One host thread may use a handle at a time; handles are independent.
 *
 * Every call returns IBPM_OK (0), a positive warning, or a negative error.
 * The message of the last error is kept per handle (ibpm_last_error).
 */
#ifndef IBPM_B200_H
#define IBPM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IBPM_ABI_VERSION 1

/* status codes */
#define IBPM_OK 0
#define IBPM_WARN_CG_MAXITER 1      /* CG hit maxiter (the reference's cg! is silent) */
#define IBPM_ERR_INVALID (-1)       /* bad argument or unsupported problem */
#define IBPM_ERR_CUDA (-2)          /* CUDA runtime error or no device */
#define IBPM_ERR_REGION (-3)        /* panel outside allowed region (coupling.jl:39-41) */
#define IBPM_ERR_NOMEM (-4)         /* device allocation failed */
#define IBPM_ERR_NONFINITE (-5)     /* NaN/Inf met in the CG residual */

/* body kinds (src/problem.jl:226-258) */
#define IBPM_BODY_STATIC 0          /* StaticBody */
#define IBPM_BODY_MOVING_RIGID 1    /* MovingRigidBody */

/* precision modes */
#define IBPM_FP64 0                 /* plain FP64 drop-in path */
#define IBPM_FP32 1                 /* mixed precision: FP32 fields and transforms; FP64 scans, boundary
                                       values, CG, force sums and B^-1 (no counterpart in the reference) */
#define IBPM_MIXED_L1 2             /* mixed precision by level: level 1 (the body's level) stored and
                                       solved in FP64, the coarser levels in FP32 fields and transforms;
                                       FP64 scans, CG, force sums and B^-1; static bodies only (no
                                       counterpart in the reference) */

typedef struct ibpm_problem {
    int32_t nx, ny, nlevel;     /* MultiDomainGrid base.n and nlevel (problem.jl:398-409) */
    double h, x0, y0;           /* base.h, base.x0 */
    double Re;                  /* Fluid.Re */
    double dt;                  /* CNAB.dt */
    int32_t npanel;             /* n_panels(bodies) */
    int32_t nbody;              /* number of preset bodies, in Bodies order */
    const int32_t *body_kind;   /* nbody entries, IBPM_BODY_* */
    const int32_t *body_start;  /* nbody+1 panel offsets (0-based), panel_range of each body */
    const double *body_xb;      /* bodypanels(body).xb stacked, npanel x 2 column-major */
    const double *body_ds;      /* bodypanels(body).ds stacked, npanel */
    int32_t grid_moving;        /* 0: StaticGrid, 1: MovingGrid (fluid.jl:22-67) */
} ibpm_problem;

typedef struct ibpm_options {
    int32_t precision;          /* IBPM_FP64, IBPM_FP32 or IBPM_MIXED_L1 */
    int32_t device;             /* CUDA device ordinal */
    int32_t cg_maxiter;         /* cg kwargs (solver.jl:137): maxiter, default 5000 */
    double cg_reltol;           /* default 1e-12 */
    double cg_abstol;           /* default 0 */
} ibpm_options;

/* Host-callback results for one step, evaluated by the caller at that step's t. */
typedef struct ibpm_step_params {
    double freestream[2];       /* fluid.freestream_vel(t) */
    double grid_motion[6];      /* GridVelocity: center(2), vel(2), angle, angular_vel */
    const double *body_motion;  /* nbody x 6 row-major: RigidBodyTransform pos(2), vel(2),
                                   angle, angular_vel; entries of static bodies are ignored;
                                   may be NULL when no body moves */
} ibpm_step_params;

/* A view of State (src/problem.jl:626-639).  NULL array pointers are skipped. */
typedef struct ibpm_state_view {
    int64_t index;
    double t0;
    double *q, *q0, *gamma, *psi, *nonlin1, *nonlin2;
    double *xb, *ds, *ub, *fbt;
    double freestream[2];
} ibpm_state_view;

typedef struct ibpm_info {
    int64_t nq, ng, nbc;        /* GridIndices sizes (problem.jl:374-388) */
    int32_t static_bodies;      /* 1: precomputed B^-1, 0: CG every step */
    int32_t last_cg_iters;      /* iterations of the last step's CG (0 for static bodies) */
    double last_cg_residual;    /* final ||r|| of that CG */
    int64_t device_bytes;       /* device memory held by the handle */
    double first_cg_residual;   /* ||r0|| of the last step's CG, from its initial guess */
    double warm_start_coef[2];  /* the last step's warm-start Galerkin coefficients: along
                                   F1 - F2, then along the network's correction (the
                                   projected mode: directions kept, then 0) */
} ibpm_info;

typedef struct ibpm_handle ibpm_handle;

/* Fills the reference defaults: FP64, device 0, maxiter 5000, reltol 1e-12, abstol 0. */
void ibpm_default_options(ibpm_options *opt);

/* CnabSolver(State(prob)) (solver.jl:84-150): allocates, computes the panel weights
 * of static bodies (errors with IBPM_ERR_REGION like coupling.jl:39-41), the
 * A/Ainv operators and, for static bodies, B and B^-1 on the device.  The state
 * starts as State(prob) (problem.jl:640-665): zeros, index 0, t0 = 0.
 * On failure *out is NULL and ibpm_last_error(NULL) gives the message. */
int ibpm_create(const ibpm_problem *prob, const ibpm_options *opt, ibpm_handle **out);
void ibpm_destroy(ibpm_handle *h);

/* Upload/download State arrays.  set_state recomputes t from index and t0
 * (set_time_index!, problem.jl:705-708) and fb (update_vars!). */
int ibpm_set_state(ibpm_handle *h, const ibpm_state_view *st);
int ibpm_get_state(ibpm_handle *h, ibpm_state_view *st);

/* advance!(solver) nsteps times; params[k] holds the callbacks at step k.  Returns
 * after the device finished the steps.  IBPM_WARN_CG_MAXITER if any CG stopped at maxiter. */
int ibpm_advance(ibpm_handle *h, int64_t nsteps, const ibpm_step_params *params);

/* The reference's output accessors vorticity!, x_velocity!, y_velocity!
 * (src/problem.jl:715-866) for one level (1-based), computed on the device so that
 * only that level is copied back: Γ / hc² ((nx-1) x (ny-1)), (q + q0)_u / hc
 * ((nx+1) x ny) or (q + q0)_v / hc (nx x (ny+1)), column-major, hc the level's
 * grid step. */
#define IBPM_FIELD_VORTICITY 0
#define IBPM_FIELD_X_VELOCITY 1
#define IBPM_FIELD_Y_VELOCITY 2
int ibpm_get_field(ibpm_handle *h, int32_t field, int32_t level, double *out);

/* state.fb (npanel x 2) and boundary_total_force over all panels (2); NULL skips. */
int ibpm_get_forces(ibpm_handle *h, double *fb, double *total_force);

/* Ensembles: independent cases (handles of any sizes, bodies and precisions)
 * stepped together.  No counterpart in the reference, which steps one case per
 * solver.  Static-body, static-grid cases of one precision with equal nx, ny,
 * levels, grid step and time step form a batched group: their fields are
 * stacked in one allocation, every line pass, nonlinear term, curl and
 * coarsening runs as one launch over all cases of the group, and so does the
 * coupling (E, B^-1, E^T), each case on its own panels; a group's whole step
 * is one CUDA graph.  Other cases step on their own streams.  All of them are
 * enqueued before any is waited for; params[k * n + c] holds step k of case c.
 * Each case's results are the bits of stepping it alone.  While grouped, a
 * case's handle reads and writes its slot of the group's fields (its own
 * field buffers are freed); destroying the ensemble copies every live case
 * back into buffers of its own.  Handles and ensemble may be destroyed in
 * either order: a handle destroyed first is dropped from its groups, and the
 * ensemble then refuses to advance (IBPM_ERR_INVALID).  A handle may appear
 * once.  The ensemble does not own the handles.  The
 * environment variable IBPM_ENSEMBLE_BATCH=0 at creation disables grouping
 * (every case on its own stream). */
typedef struct ibpm_ensemble ibpm_ensemble;
int ibpm_ensemble_create(ibpm_handle *const *cases, int32_t n, ibpm_ensemble **out);
int ibpm_ensemble_advance(ibpm_ensemble *e, int64_t nsteps, const ibpm_step_params *params);
void ibpm_ensemble_destroy(ibpm_ensemble *e);
const char *ibpm_ensemble_last_error(const ibpm_ensemble *e);
/* The number of batched groups and of the cases they hold (NULL skips). */
int ibpm_ensemble_groups(const ibpm_ensemble *e, int32_t *ngroups, int32_t *nbatched);

/* Pass-shape autotuner (no counterpart in the reference).  The Y pass of the
 * DST-diagonalised solves runs with NG line pairs (2 NG columns) per block, NG
 * in {1, 2, 4, 8}; every NG gives the same bits.  With the environment variable
 * IBPM_TUNE=1, engines (and ensemble groups) time every NG on the device for
 * each (GPU, transform length, precision, batch bucket) they launch, before
 * their first step, and keep the fastest; IBPM_TUNE_CACHE=<file> reads the table
 * from that file at first use and appends new choices to it.  Untuned keys use
 * NG = 2 (4 from 16 fields per launch).  IBPM_TUNE_FORCE_NG=<n> forces one NG.
 * ibpm_tune_table writes the table as text lines "key NG" into out (len bytes,
 * NUL-terminated) and returns the length it needs. */
int ibpm_tune_table(char *out, int32_t len);

int ibpm_get_time(ibpm_handle *h, int64_t *index, double *t);
int ibpm_get_info(ibpm_handle *h, ibpm_info *info);
const char *ibpm_last_error(const ibpm_handle *h);

/* The library's CUDA stream (cudaStream_t) for callers that time on it. */
void *ibpm_stream(ibpm_handle *h);
/* Number of kernels this handle launched so far (instrumentation). */
int64_t ibpm_kernel_launches(const ibpm_handle *h);

/* Kernel timing (instrumentation for roofline reports): when enabled, every
 * launch of the classes below is bracketed by CUDA events on the handle's
 * stream.  ibpm_profile(h, 1) clears the counters; ibpm_profile_read gives the
 * launches, summed device time (ms) and algorithmic bytes (one read of each
 * input field and one write of each output field) of a class. */
#define IBPM_KCLASS_XPASS 0         /* DST along x (row pass) */
#define IBPM_KCLASS_YPASS 1         /* DST along y, spectral multiply, DST along y */
#define IBPM_KCLASS_NONLINEAR 2     /* nonlinear advection term */
#define IBPM_KCLASS_CURL 3          /* curl of the streamfunction */
#define IBPM_KCLASS_XTRIAL 4        /* trial solve, first X pass (all levels) */
#define IBPM_KCLASS_YTRIAL 5        /* trial solve, Y pass with the A/Ainv multiplies (all levels) */
#define IBPM_KCLASS_TCDST 6         /* the four tensor-core passes of a batched 2D solve; its third value
                                       counts algorithmic flops (4 nprod P^3 per field), not bytes */
#define IBPM_KCLASS_TCLINES 7       /* the FP64 prologue of a tensor-core solve into BF16 lines */
#define IBPM_KCLASS_COUNT 8
int ibpm_profile(ibpm_handle *h, int enable);
int ibpm_profile_read(ibpm_handle *h, int kclass, int64_t *launches, double *ms, double *bytes);

/* Diagnostics: single operators of the step on caller host buffers, for
 * operator-level parity tests.
 *   ibpm_diag_solve: x = S(S(b) scale / Lambda) on one (nx-1) x (ny-1) field with
 *     op 0: Lambda = lap_eigs (Δinv_operator, fluid.jl:117-119),
 *     op 1: A at `level`, op 2: Ainv at `level` (A_operator, fluid.jl:121-134);
 *     op 3..5: ops 0..2 with the tensor-core transforms of one BF16 product,
 *     op 6..8: with three products (split BF16); nx = ny in {256, 512}, FP64
 *     engine only (see ibpm_set_rebuild_transform).
 *   ibpm_diag_apply_B: x = B z (B_operator, coupling.jl:163-176), 2*npanel.
 *   ibpm_diag_binv: the precomputed B^-1 (2np x 2np, column-major); static bodies only. */
int ibpm_diag_solve(ibpm_handle *h, int op, int level, const double *b, double *x);
int ibpm_diag_apply_B(ibpm_handle *h, const double *z, double *x);
int ibpm_diag_binv(ibpm_handle *h, double *out);
/* vort2flux (fluid.jl:178-205) on host buffers: gamma (ng x L) is coarsified in
 * place (as in the reference), psi (ng x L) and q (nq x L) are outputs. */
int ibpm_diag_vort2flux(ibpm_handle *h, double *gamma, double *psi, double *q);
/* rot!(reg!(f)) (fluid.jl:101-111 after coupling.jl:72-85) into gamma1 (ng), and
 * regT!(f, q1) (coupling.jl:57-69) from a level-1 flux q1 (nq); NULL skips either. */
int ibpm_diag_reg(ibpm_handle *h, const double *f, double *gamma1, const double *q1, double *fout);

/* Learned CG warm start for moving bodies.  No counterpart in the reference:
 * cg! (src/coupling.jl:194-202) starts from the previous F~b.  Here the start
 * can first move along the last change of the solution (a Galerkin step in the
 * B-energy norm), and then along a network's correction computed from that
 * guess's residual; plain CG then runs to the same tolerance, so only the
 * iteration count changes.
 *
 * The network is a 1D convolutional net over the body points: `layers`
 * convolutions of odd width `kernel` with zero padding, `width` channels
 * between them, tanh after every layer but the last.  Inputs are normalised per
 * channel ((x - in_mean) / in_std) and the last layer's output is the
 * normalised prediction (prediction = out_mean + out_std * y).  Parameters are
 * one FP32 vector: per layer W [out][in][kernel], then b [out].  Samples are
 * arrays [batch][channels][n], n body points per sample.  The warm start uses
 * 10 input channels per point -- the residual r = b - B x_e of the
 * extrapolated guess x_e (x, y), the previous solution F1 (x, y), its last
 * change d = F1 - F2 (x, y), ub (x, y), cos and sin of the body angle, with r and
 * d divided by their RMS over the sample -- and 2 outputs, the correction of x_e
 * (x, y) in units of r's RMS.  A network lives on one device and owns a stream. */
typedef struct ibpm_net ibpm_net;
int ibpm_net_create(int32_t cin, int32_t width, int32_t kernel, int32_t layers, int32_t cout, uint64_t seed,
                    int32_t device, ibpm_net **out);
void ibpm_net_destroy(ibpm_net *net);
int64_t ibpm_net_num_params(const ibpm_net *net);
int ibpm_net_get_params(ibpm_net *net, float *params);
int ibpm_net_set_params(ibpm_net *net, const float *params);   /* also resets the optimiser state */
int ibpm_net_set_normalisation(ibpm_net *net, const float *in_mean, const float *in_std, const float *out_mean,
                               const float *out_std);
int ibpm_net_get_normalisation(ibpm_net *net, float *in_mean, float *in_std, float *out_mean, float *out_std);
/* Prediction in solver units for raw host samples x [batch][cin][n] -> y [batch][cout][n]. */
int ibpm_net_forward(ibpm_net *net, const float *x, int64_t batch, int32_t n, float *y);
/* Loss of the normalised prediction against the normalised raw targets
 * t [batch][cout][n], and its gradient with respect to the parameters.  With e
 * the error of one sequence of n points and E its running sum along the points
 * divided by sqrt(n), the loss is (sum e^2 + sum E^2) / (batch cout n): the
 * running-sum term weighs the smooth error components, the ones that dominate
 * the CG residual, about n/3 times more. */
int ibpm_net_loss_grad(ibpm_net *net, const float *x, const float *t, int64_t batch, int32_t n, float *loss,
                       float *grad);
/* Adam (lr, betas 0.9 / 0.999, eps 1e-8) on shuffled full batches of the raw
 * samples, `epochs` passes; epoch_loss[e] (may be NULL) is the mean batch loss. */
int ibpm_net_train(ibpm_net *net, const float *x, const float *t, int64_t nsamples, int32_t n, int32_t epochs,
                   int32_t batch, float lr, uint64_t seed, float *epoch_loss);
const char *ibpm_net_last_error(const ibpm_net *net);   /* NULL: the last failed create */
/* Chooses the CG initial guess of a moving-body handle.  F1, F2 are the last two
 * solutions:
 *   IBPM_WS_PREVIOUS      F1 (the reference; net and depth ignored)
 *   IBPM_WS_EXTRAPOLATED  x_e = F1 + y (F1 - F2)
 *   IBPM_WS_LEARNED       x_e + a p, p the network's correction from x_e's residual
 *                         (net: 10 -> 2 channels on the handle's device, kept alive
 *                         while installed)
 *   IBPM_WS_PROJECTED     the combination of the last `depth` (1 .. 16) solutions
 *                         (projection for successive right-hand sides); the history
 *                         restarts from the current solution when the mode or the
 *                         state is set
 *   IBPM_WS_DIRECT        B^-1 b: B assembled for the step's body position from its
 *                         2 npanel columns (batched applications, as the static-body
 *                         B^-1 of src/coupling.jl:187-192) and inverted on the GPU,
 *                         every `depth` (1 .. 1048576) steps, the first on the next
 *                         step; between rebuilds the last inverse gives the guess.
 *                         FP64 handles only; keeps a (2 npanel)^2 matrix and the
 *                         column-batch work buffers (up to about 16 GB)
 *   IBPM_WS_PRECONDITIONED  as IBPM_WS_DIRECT, and CG is preconditioned by the same
 *                         inverse (z = B_k^-1 r, B_k of the last rebuild): between
 *                         rebuilds CG needs a few iterations instead of hundreds.
 *                         Not the reference's iteration (it passes no
 *                         preconditioner); the stopping rule on ||r|| is the same
 * where the coefficients minimise the B-energy norm of the error over their
 * directions (Galerkin steps with B of the current step, applied in batched
 * passes; CG reuses B x0).  CG then runs from the guess to the reference's
 * tolerance in every mode: max(reltol ||b - B F1||, abstol), the relative part
 * taken from the residual at the reference's own start F1 (the direct and
 * preconditioned modes apply B to F1 once more for it when reltol > 0), so a
 * better guess changes only the iteration count. */
#define IBPM_WS_PREVIOUS 0
#define IBPM_WS_LEARNED 1
#define IBPM_WS_EXTRAPOLATED 2
#define IBPM_WS_PROJECTED 3
#define IBPM_WS_DIRECT 4
#define IBPM_WS_PRECONDITIONED 5
/* IBPM_WS_PRECONDITIONED with a better start between rebuilds: B^-1 b plus this
 * step's stale error F - B^-1 b extrapolated in time from the last (up to
 * three) steps' stale errors, which change smoothly with the body's motion. */
#define IBPM_WS_PRECOND_EXTRAP 6
int ibpm_set_warm_start(ibpm_handle *h, int32_t mode, ibpm_net *net, int32_t depth);
/* How IBPM_WS_PRECONDITIONED and IBPM_WS_PRECOND_EXTRAP assemble the B they
 * invert (the preconditioner; no counterpart in the reference).  products 0: the
 * FP64 transforms of the step (the default); 1 or 3: every 2D solve of the
 * assembly as four dense DST-I passes on the tensor cores (tcgen05) with BF16
 * operands and FP32 accumulation (each pass two half-length products by the
 * transform's even/odd symmetry), one product S_hi x_hi or three
 * (S_hi x_hi + S_hi x_lo + S_lo x_hi, each operand split as hi = bf16(v),
 * lo = bf16(v - hi)).  The preconditioner is then close to, not equal to, the
 * inverse; CG still runs to the same tolerance, so forces are unchanged to
 * that tolerance and only the iteration count can differ.  Moving bodies, FP64
 * engine, nx = ny in {256, 512}, an sm_100 device; other modes ignore it. */
int ibpm_set_rebuild_transform(ibpm_handle *h, int32_t products);
/* The last step's warm-start features (10 x npanel floats), target (2 x
 * npanel: the converged F~b minus the extrapolated guess x_e) and, in the
 * learned mode, the network's correction as the step used it (zeros
 * otherwise); the target is in units of the RMS of x_e's residual.  Needs the extrapolated or learned mode; NULL skips an output. */
int ibpm_warm_start_sample(ibpm_handle *h, float *features, float *target, float *prediction);

/* Laplacian-inverse solve x = Δ⁻¹ b (the operator of src/fluid.jl:117-119) for callers
 * that cannot allocate device memory.  No counterpart in the reference: it exists
 * for code running inside another framework's memory pool or a fixed arena, or a
 * host loop that must not allocate between steps.  b and x are caller-owned
 * device buffers of (nx-1) x (ny-1) doubles, column-major; x may be b (the
 * first pass reads b into scratch, the last writes x, in stream order).
 * The scratch fields and transform tables live in one static device array of
 * about 4.3 MB that each GPU loading the library keeps until exit; it limits
 * (nx-1)(ny-1) to 262144 cells (nx, ny even, <= 1024, of the form 2^a 3^b 5^c).
 * Larger sizes return IBPM_ERR_INVALID.  The first call on a device (and the
 * first after a change of nx, ny) writes the tables: make it outside stream
 * capture, which such a call rejects with IBPM_ERR_INVALID.  All calls share the array, so
 * calls that overlap on the GPU race.  stream is a cudaStream_t (NULL: default).
 * On error ibpm_noalloc_last_error() gives the message. */
int ibpm_lap_inv_noalloc(int nx, int ny, const double *b, double *x, void *stream);
const char *ibpm_noalloc_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
