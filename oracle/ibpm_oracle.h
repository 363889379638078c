/*
 * ibpm_oracle.h -- CPU restatement of ImmersedBodies.jl's CNAB/IBPM time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle that the CUDA path is checked
 * against.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * may load it.  The product library (libibpm_b200.so) never links it.
 *
 * Pinning status: the reference (Julia) cannot run in this container, so the
 * full time step is "parity unpinned" against the reference itself.  What is
 * pinned: the DST-I against scipy.fft.dst(type=1) (the FFTW RODFT00 definition
 * used by src/fluid.jl:113-115), the Yang3 delta partition of unity, the
 * save_state byte layout (src/io/io.jl:14-25), the time-index rule
 * (src/problem.jl:703-708) and the "outside allowed region" error
 * (src/coupling.jl:39-41, test/solver.jl:66-79).  The whole step is also
 * cross-checked against an independent numpy/scipy transcription
 * (tests/golden/make_golden.py).
 *
 * All arrays use the reference's Julia layouts (column-major, x fastest):
 *   q, q0      : nq x nlevel,  nq = (nx+1)*ny + nx*(ny+1)   (u block then v block)
 *   Gamma, psi : ng x nlevel,  ng = (nx-1)*(ny-1)
 *   nonlin[2]  : ng x nlevel each
 *   xb, ub     : npanel x 2;  ds : npanel;  Fb : 2*npanel;  fb : npanel x 2
 */
#ifndef IBPM_ORACLE_H
#define IBPM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Body kinds (src/problem.jl:226-258). */
#define ORC_BODY_STATIC 0
#define ORC_BODY_MOVING_RIGID 1

typedef struct orc_problem {
    int32_t nx, ny, nlevel;     /* base grid cells and number of levels */
    double h, x0, y0;           /* base grid step and lower-left corner */
    double Re, dt;              /* Reynolds number, CNAB time step */
    int32_t npanel;             /* total panels over all bodies */
    int32_t nbody;
    const int32_t *body_kind;   /* nbody entries */
    const int32_t *body_start;  /* nbody+1 offsets into the panel arrays (0-based) */
    const double *body_xb;      /* reference panel positions, npanel x 2 column-major */
    const double *body_ds;      /* reference panel lengths, npanel */
    int32_t grid_moving;        /* 0 StaticGrid, 1 MovingGrid */
    int32_t cg_maxiter;         /* IterativeSolvers cg! kwargs (src/solver.jl:137) */
    double cg_reltol;
    double cg_abstol;
    int32_t timing_only;        /* 1: skip building B^-1 (static bodies) -- for CPU timing
                                   samples only; the step then applies a zero B^-1 */
} orc_problem;

/* Per-step host callback results, evaluated by the caller at the step's t. */
typedef struct orc_step_params {
    double freestream[2];       /* fluid.freestream_vel(t) */
    const double *body_motion;  /* nbody x 6: pos.x pos.y vel.x vel.y angle angular_vel */
    double grid_motion[6];      /* center.x center.y vel.x vel.y angle angular_vel */
} orc_step_params;

typedef struct orc_solver orc_solver;

/* CnabSolver(state) (src/solver.jl:84-150).  Returns NULL and fills err on failure. */
orc_solver *orc_create(const orc_problem *p, char *err, int errlen);
void orc_destroy(orc_solver *s);
int orc_nthreads(int n);  /* set OpenMP threads (<=0: leave), returns the count in use */

/* advance!(solver) (src/solver.jl:155-190).  Returns 0, or -1 with err filled. */
int orc_advance(orc_solver *s, const orc_step_params *prm, char *err, int errlen);

/* Direct access to the state arrays (reference layouts, see header comment). */
double *orc_q(orc_solver *s);
double *orc_q0(orc_solver *s);
double *orc_gamma(orc_solver *s);
double *orc_psi(orc_solver *s);
double *orc_nonlin(orc_solver *s, int k);  /* k = 0,1 -> state.nonlin[1], [2] */
double *orc_xb(orc_solver *s);
double *orc_ds(orc_solver *s);
double *orc_ub(orc_solver *s);
double *orc_fbt(orc_solver *s);            /* state.F̃b */
double *orc_fb(orc_solver *s);             /* state.fb */
double *orc_freestream(orc_solver *s);     /* 2 doubles */
int64_t orc_get_index(orc_solver *s);
void orc_set_index(orc_solver *s, int64_t index); /* set_time_index! */
double orc_get_t(orc_solver *s);
double orc_get_t0(orc_solver *s);
void orc_set_t0(orc_solver *s, double t0);
int orc_last_cg_iters(orc_solver *s);
/* Copy of the precomputed B^-1 (2np x 2np column-major) for static bodies; returns 0 if absent. */
int orc_binv(orc_solver *s, double *out);
/* Replaces the precomputed B^-1 of static bodies (2np x 2np, column-major), e.g.
 * in a timing_only solver that skipped building it; 0 when there is none. */
int orc_set_binv(orc_solver *s, const double *in);
/* Apply the Schur complement B (src/coupling.jl:150-177) with the current weights. */
void orc_apply_B(orc_solver *s, double *x, const double *z);
/* vort2flux! on caller arrays (src/fluid.jl:175-206); Gamma is coarsified in place. */
void orc_vort2flux(orc_solver *s, double *psi, double *q, double *gamma);
/* rot!(Gamma, reg!(q, f)) (fluid.jl:101-111, coupling.jl:72-85) and regT! (coupling.jl:57-69) */
void orc_reg_rot(orc_solver *s, const double *f, double *gamma1);
void orc_regT(orc_solver *s, const double *q1, double *f);
/* update_vars! (src/problem.jl:676-685) */
void orc_update_vars(orc_solver *s);

/* ---- kernels exposed for known-answer tests ---- */
/* Unnormalised 1D DST-I (FFTW RODFT00): y_k = 2 sum_j x_j sin(pi (j+1)(k+1)/(n+1)). */
void orc_dst1(int n, const double *x, double *y);
/* 2D DST-I over an (n1 x n2) column-major array, both dimensions. */
void orc_dst2(int n1, int n2, const double *x, double *y);
/* _lap_inv_operator with a given eigenvalue array (src/fluid.jl:145-166). */
void orc_lap_inv(int nx, int ny, const double *lam, const double *b, double *x);
/* _lap_eigs (src/fluid.jl:168-173), (nx-1) x (ny-1). */
void orc_lap_eigs(int nx, int ny, double *lam);
/* Yang3 smoothed delta times h (src/coupling.jl:91-148). */
double orc_delta_h(double rf, double rb, double dr);

#ifdef __cplusplus
}
#endif
#endif
