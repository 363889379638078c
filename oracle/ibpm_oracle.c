/*
 * ibpm_oracle.c -- CPU FP64 restatement of ImmersedBodies.jl's CnabSolver.
 *
 * TEST INFRASTRUCTURE ONLY (see ibpm_oracle.h).  The product CUDA path never
 * links or calls this file.
 *
 * Every function names the reference file:line it restates.  Loops keep the
 * reference's 1-based index ranges through the accessor macros below, so the
 * transcription can be read side by side with src/fluid.jl and
 * src/coupling.jl.  The DST-I is computed here with its own mixed-radix FFT of
 * the odd extension (length 2(n+1)); FFTW is not available, and the CUDA path
 * uses a different (length n+1, pre-twiddled) algorithm, so the two are
 * independent.
 */
#include "ibpm_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

/* ------------------------------------------------------------------------- */
/* FFT (mixed radix, iterative Stockham autosort, precomputed twiddles)       */
/* ------------------------------------------------------------------------- */
/* Forward transform X_k = sum_j x_j exp(-2 pi i j k / n).  n is factored into
 * stages of radix 4, 2, 3 and then any other prime; stage s (radix p, Ns the
 * product of the earlier radices) maps x to y by
 *   y[q Ns p + k + r Ns] = sum_t W_p^{r t} W_{Ns p}^{t k} x[q Ns + k + t n/p]
 * for q < n/(Ns p), k < Ns.  Every twiddle W_{Ns p}^{t k} and every root
 * W_p^{r t} is tabulated when the plan is made (long double), so the transform
 * does no index modulo and evaluates no trigonometric function. */

#define FFT_MAX_STAGES 40

typedef struct fft_plan {
    int n;
    int nst;
    int radix[FFT_MAX_STAGES];
    cplx *tw[FFT_MAX_STAGES];   /* tw[s][k (p-1) + t - 1] = W_{Ns p}^{t k}, k < Ns, 1 <= t < p */
    cplx *root[FFT_MAX_STAGES]; /* root[s][r p + t] = W_p^{r t} */
} fft_plan;

static cplx cexpm(long double num, long double den) { /* exp(-2 pi i num / den) */
    const long double a = -2.0L * 3.14159265358979323846264338327950288L * num / den;
    return (double)cosl(a) + I * (double)sinl(a);
}

static fft_plan *fft_plan_new(int n) {
    fft_plan *pl = (fft_plan *)calloc(1, sizeof(fft_plan));
    pl->n = n;
    int m = n, Ns = 1;
    while (m > 1) {
        int p;
        if (m % 4 == 0)
            p = 4;
        else if (m % 2 == 0)
            p = 2;
        else {
            p = m;
            for (int f = 3; f * f <= m; f += 2)
                if (m % f == 0) {
                    p = f;
                    break;
                }
        }
        const int s = pl->nst++;
        pl->radix[s] = p;
        pl->tw[s] = (cplx *)malloc(sizeof(cplx) * (size_t)Ns * (size_t)(p - 1));
        for (int k = 0; k < Ns; k++)
            for (int t = 1; t < p; t++) pl->tw[s][(size_t)k * (p - 1) + t - 1] = cexpm((long double)t * k, (long double)Ns * p);
        pl->root[s] = (cplx *)malloc(sizeof(cplx) * (size_t)p * p);
        for (int r = 0; r < p; r++)
            for (int t = 0; t < p; t++) pl->root[s][(size_t)r * p + t] = cexpm((long double)((r * t) % p), (long double)p);
        Ns *= p;
        m /= p;
    }
    return pl;
}

static void fft_plan_free(fft_plan *p) {
    if (!p) return;
    for (int s = 0; s < p->nst; s++) {
        free(p->tw[s]);
        free(p->root[s]);
    }
    free(p);
}

/* Forward FFT of x (length pl->n); w is scratch of the same length.  The result
 * is in x on return. */
static void fft_exec(const fft_plan *pl, cplx *x, cplx *w) {
    const int n = pl->n;
    cplx *src = x, *dst = w;
    int Ns = 1;
    for (int s = 0; s < pl->nst; s++) {
        const int p = pl->radix[s], stride = n / p, nq = n / (Ns * p);
        const cplx *tw = pl->tw[s], *rt = pl->root[s];
        for (int q = 0; q < nq; q++) {
            for (int k = 0; k < Ns; k++) {
                const int j = q * Ns + k;
                const cplx *twk = tw + (size_t)k * (p - 1);
                cplx *out = dst + (size_t)q * Ns * p + k;
                if (p == 4) {
                    const cplx a = src[j], b = src[j + stride] * (k ? twk[0] : 1.0);
                    const cplx c = src[j + 2 * stride] * (k ? twk[1] : 1.0);
                    const cplx d = src[j + 3 * stride] * (k ? twk[2] : 1.0);
                    const cplx t0 = a + c, t1 = a - c, t2 = b + d, t3 = -I * (b - d);
                    out[0] = t0 + t2;
                    out[Ns] = t1 + t3;
                    out[2 * Ns] = t0 - t2;
                    out[3 * Ns] = t1 - t3;
                } else if (p == 2) {
                    const cplx a = src[j], b = src[j + stride] * (k ? twk[0] : 1.0);
                    out[0] = a + b;
                    out[Ns] = a - b;
                } else {
                    cplx v[64];
                    cplx *vb = p <= 64 ? v : (cplx *)malloc(sizeof(cplx) * (size_t)p);
                    vb[0] = src[j];
                    for (int t = 1; t < p; t++) vb[t] = src[j + t * stride] * twk[t - 1];
                    for (int r = 0; r < p; r++) {
                        cplx acc = 0;
                        const cplx *rr = rt + (size_t)r * p;
                        for (int t = 0; t < p; t++) acc += vb[t] * rr[t];
                        out[(size_t)r * Ns] = acc;
                    }
                    if (vb != v) free(vb);
                }
            }
        }
        cplx *tmp = src;
        src = dst;
        dst = tmp;
        Ns *= p;
    }
    if (src != x) memcpy(x, src, sizeof(cplx) * (size_t)n);
}

/* Pairwise DST-I of two real lines a, b of length n (FFTW RODFT00 definition):
 * the odd extension of z = a + i b has FFT -i DST(a) + DST(b). */
static void dst1_pair(int n, const double *a, int as, const double *b, int bs, double *ya, int yas, double *yb,
                      int ybs, const fft_plan *pl, cplx *z, cplx *Z) {
    const int M = n + 1, N = 2 * M;
    z[0] = 0;
    z[M] = 0;
    for (int j = 1; j <= n; j++) {
        double av = a[(size_t)(j - 1) * as];
        double bv = b ? b[(size_t)(j - 1) * bs] : 0.0;
        z[j] = av + I * bv;
        z[N - j] = -(av + I * bv);
    }
    fft_exec(pl, z, Z);
    for (int k = 1; k <= n; k++) {
        ya[(size_t)(k - 1) * yas] = -cimag(z[k]);
        if (yb) yb[(size_t)(k - 1) * ybs] = creal(z[k]);
    }
}

void orc_dst1(int n, const double *x, double *y) {
    fft_plan *pl = fft_plan_new(2 * (n + 1));
    cplx *z = (cplx *)malloc(sizeof(cplx) * 2 * (size_t)(n + 1));
    cplx *Z = (cplx *)malloc(sizeof(cplx) * 2 * (size_t)(n + 1));
    dst1_pair(n, x, 1, NULL, 0, y, 1, NULL, 0, pl, z, Z);
    free(z);
    free(Z);
    fft_plan_free(pl);
}

/* 2D DST-I over dims 1 and 2 of a column-major n1 x n2 array (src/fluid.jl:113-115). */
static void dst2_plans(int n1, int n2, const double *x, double *y, const fft_plan *p1, const fft_plan *p2) {
    double *t = (double *)malloc(sizeof(double) * (size_t)n1 * n2);
    /* along dim 1: lines are columns j (contiguous) */
#pragma omp parallel
    {
        cplx *z = (cplx *)malloc(sizeof(cplx) * 2 * (size_t)(n1 + 1));
        cplx *Z = (cplx *)malloc(sizeof(cplx) * 2 * (size_t)(n1 + 1));
#pragma omp for schedule(static)
        for (int j = 0; j < n2; j += 2) {
            const double *a = x + (size_t)j * n1;
            const double *b = (j + 1 < n2) ? x + (size_t)(j + 1) * n1 : NULL;
            double *ya = t + (size_t)j * n1;
            double *yb = (j + 1 < n2) ? t + (size_t)(j + 1) * n1 : NULL;
            dst1_pair(n1, a, 1, b, 1, ya, 1, yb, 1, p1, z, Z);
        }
        free(z);
        free(Z);
    }
#pragma omp parallel
    {
        cplx *z = (cplx *)malloc(sizeof(cplx) * 2 * (size_t)(n2 + 1));
        cplx *Z = (cplx *)malloc(sizeof(cplx) * 2 * (size_t)(n2 + 1));
#pragma omp for schedule(static)
        for (int i = 0; i < n1; i += 2) {
            const double *a = t + i;
            const double *b = (i + 1 < n1) ? t + i + 1 : NULL;
            double *ya = y + i;
            double *yb = (i + 1 < n1) ? y + i + 1 : NULL;
            dst1_pair(n2, a, n1, b, n1, ya, n1, yb, n1, p2, z, Z);
        }
        free(z);
        free(Z);
    }
    free(t);
}

void orc_dst2(int n1, int n2, const double *x, double *y) {
    fft_plan *p1 = fft_plan_new(2 * (n1 + 1));
    fft_plan *p2 = fft_plan_new(2 * (n2 + 1));
    dst2_plans(n1, n2, x, y, p1, p2);
    fft_plan_free(p1);
    fft_plan_free(p2);
}

/* ------------------------------------------------------------------------- */
/* Solver state                                                               */
/* ------------------------------------------------------------------------- */

struct orc_solver {
    orc_problem p;
    int32_t *body_kind, *body_start;
    double *ref_xb, *ref_ds;
    int nx, ny, L, nu, nv, nq, ng, nbc, np;
    int bL, bR, bB, bT;
    fft_plan *plx, *ply;
    /* State (src/problem.jl:626-665) */
    int64_t index;
    double t0, t;
    double *q, *q0, *G, *psi, *nonlin[2], *xb, *ds, *ub, *Fbt, *fb;
    double fs[2];
    /* CnabSolver buffers (src/solver.jl:93-106) */
    double *qs, *Gs, *Gbc, *Gtmp, *psitmp, *qtmp, *Ftmp, *Gtmp1, *Gtmp2, *Gtmp3, *qtmp1, *qtmp2, *Gdst1, *Gdst2;
    double *lam;
    double **Lexpl, **Limpl;
    /* Regularization (src/coupling.jl:3-18) */
    int *pc;   /* np x 2 panel_coords */
    double *w; /* np x 2 x 7 x 7 weights, layout [(p*2+c)*49 + b*7 + a] */
    double *Binv;
    int last_cg_iters;
    int any_moving;
};

#define REG_SUPPORT 3
#define NSUPP 7

/* 1-based accessors in the reference's column-major layouts */
#define GAM(a, i, j) (a)[(size_t)((i)-1) + (size_t)(s->nx - 1) * (size_t)((j)-1)]
#define QX(a, i, j) (a)[(size_t)((i)-1) + (size_t)(s->nx + 1) * (size_t)((j)-1)]
#define QY(a, i, j) (a)[(size_t)s->nu + (size_t)((i)-1) + (size_t)(s->nx) * (size_t)((j)-1)]
#define BC(a, k) (a)[(k)-1]

static double *dalloc(size_t n) { return (double *)calloc(n ? n : 1, sizeof(double)); }

static double gridstep(const orc_solver *s, int lev) { return ldexp(1.0, lev - 1) * s->p.h; } /* problem.jl:417 */

/* ---- fluid.jl ---- */

/* rot! (src/fluid.jl:101-111) */
static void rot(const orc_solver *s, double *G, const double *q) {
    const int nx = s->nx, ny = s->ny;
#pragma omp parallel for schedule(static)
    for (int j = 2; j <= ny; j++)
        for (int i = 2; i <= nx; i++) GAM(G, i - 1, j - 1) = (QX(q, i, j - 1) - QX(q, i, j)) + (QY(q, i, j) - QY(q, i - 1, j));
}

/* 4-argument curl! (src/fluid.jl:230-276) */
static void curl(const orc_solver *s, double *q, const double *psi, const double *pbc) {
    const int nx = s->nx, ny = s->ny, T = s->bT, B = s->bB, L = s->bL, R = s->bR;
#pragma omp parallel for schedule(static)
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 2; i <= nx; i++) QX(q, i, j) = GAM(psi, i - 1, j) - GAM(psi, i - 1, j - 1);
    for (int i = 2; i <= nx; i++) QX(q, i, 1) = GAM(psi, i - 1, 1) - BC(pbc, B + i);
    for (int i = 2; i <= nx; i++) QX(q, i, ny) = BC(pbc, i + T) - GAM(psi, i - 1, ny - 1);
    for (int j = 1; j <= ny; j++) QX(q, 1, j) = BC(pbc, (L + 1) + j) - BC(pbc, L + j);
    for (int j = 1; j <= ny; j++) QX(q, nx + 1, j) = BC(pbc, (R + 1) + j) - BC(pbc, R + j);

#pragma omp parallel for schedule(static)
    for (int j = 2; j <= ny; j++)
        for (int i = 2; i <= nx - 1; i++) QY(q, i, j) = GAM(psi, i - 1, j - 1) - GAM(psi, i, j - 1);
    for (int j = 2; j <= ny; j++) QY(q, 1, j) = BC(pbc, L + j) - GAM(psi, 1, j - 1);
    for (int j = 2; j <= ny; j++) QY(q, nx, j) = GAM(psi, nx - 1, j - 1) - BC(pbc, R + j);
    for (int i = 1; i <= nx; i++) QY(q, i, 1) = BC(pbc, B + i) - BC(pbc, (B + 1) + i);
    for (int i = 1; i <= nx; i++) QY(q, i, ny + 1) = BC(pbc, T + i) - BC(pbc, (T + 1) + i);
}

/* get_bc! (src/fluid.jl:278-306) */
static void get_bc(const orc_solver *s, double *rbc, const double *r) {
    const int nx = s->nx, ny = s->ny, T = s->bT, B = s->bB, L = s->bL, R = s->bR;
    for (int k = 0; k <= nx / 2; k++) {
        int i = nx / 4 + k, ibc = 1 + 2 * k;
        BC(rbc, B + ibc) = GAM(r, i, ny / 4);
        BC(rbc, T + ibc) = GAM(r, i, 3 * ny / 4);
    }
    for (int k = 1; k <= nx / 2; k++) {
        int i = nx / 4 + k, ibc = 2 * k;
        BC(rbc, B + ibc) = 0.5 * (GAM(r, i, ny / 4) + GAM(r, i - 1, ny / 4));
        BC(rbc, T + ibc) = 0.5 * (GAM(r, i, 3 * ny / 4) + GAM(r, i - 1, 3 * ny / 4));
    }
    for (int k = 0; k <= ny / 2; k++) {
        int j = ny / 4 + k, jbc = 1 + 2 * k;
        BC(rbc, L + jbc) = GAM(r, nx / 4, j);
        BC(rbc, R + jbc) = GAM(r, 3 * nx / 4, j);
    }
    for (int k = 1; k <= ny / 2; k++) {
        int j = ny / 4 + k, jbc = 2 * k;
        BC(rbc, L + jbc) = 0.5 * (GAM(r, nx / 4, j) + GAM(r, nx / 4, j - 1));
        BC(rbc, R + jbc) = 0.5 * (GAM(r, 3 * nx / 4, j) + GAM(r, 3 * nx / 4, j - 1));
    }
}

/* apply_bc! (src/fluid.jl:308-338) */
static void apply_bc(const orc_solver *s, double *r, const double *rbc, double fac) {
    const int nx = s->nx, ny = s->ny, T = s->bT, B = s->bB, L = s->bL, R = s->bR;
    for (int i = 1; i <= nx - 1; i++) {
        GAM(r, i, 1) += fac * BC(rbc, (B + 1) + i);
        GAM(r, i, ny - 1) += fac * BC(rbc, (T + 1) + i);
    }
    for (int j = 1; j <= ny - 1; j++) {
        GAM(r, 1, j) += fac * BC(rbc, (L + 1) + j);
        GAM(r, nx - 1, j) += fac * BC(rbc, (R + 1) + j);
    }
}

/* coarsify! (src/fluid.jl:208-228); zip() stops at the shorter index range */
static void coarsify(const orc_solver *s, double *Gc, const double *G) {
    const int nx = s->nx, ny = s->ny;
    const int ni = (nx / 2 - 2 - (-nx / 2 + 2)) / 2 + 1, nic = (nx / 4 - 1) - (-nx / 4 + 1) + 1;
    const int nj = (ny / 2 - 2 - (-ny / 2 + 2)) / 2 + 1, njc = (ny / 4 - 1) - (-ny / 4 + 1) + 1;
    const int ci = ni < nic ? ni : nic, cj = nj < njc ? nj : njc;
    for (int b = 0; b < cj; b++) {
        int j = ny / 2 + (-ny / 2 + 2) + 2 * b, jc = ny / 2 + (-ny / 4 + 1) + b;
        for (int a = 0; a < ci; a++) {
            int i = nx / 2 + (-nx / 2 + 2) + 2 * a, ic = nx / 2 + (-nx / 4 + 1) + a;
            GAM(Gc, ic, jc) = GAM(G, i, j) +
                              0.5 * (GAM(G, i + 1, j) + GAM(G, i, j + 1) + GAM(G, i - 1, j) + GAM(G, i, j - 1)) +
                              0.25 * (GAM(G, i + 1, j + 1) + GAM(G, i + 1, j - 1) + GAM(G, i - 1, j - 1) +
                                      GAM(G, i - 1, j + 1));
        }
    }
}

/* _lap_eigs (src/fluid.jl:168-173) */
void orc_lap_eigs(int nx, int ny, double *lam) {
    for (int j = 1; j <= ny - 1; j++)
        for (int i = 1; i <= nx - 1; i++)
            lam[(size_t)(i - 1) + (size_t)(nx - 1) * (j - 1)] = -2 * ((cos(M_PI * i / nx) + cos(M_PI * j / ny)) - 2);
}

/* _lap_inv_operator closure body (src/fluid.jl:157-165) */
static void lap_inv(const orc_solver *s, const double *Lam, double *x, const double *b) {
    const size_t ng = (size_t)s->ng;
    const double scale = 1.0 / (double)(4 * (long)s->nx * (long)s->ny);
    memcpy(s->Gdst1, b, ng * sizeof(double));
    dst2_plans(s->nx - 1, s->ny - 1, s->Gdst1, s->Gdst2, s->plx, s->ply);
#pragma omp parallel for schedule(static)
    for (size_t k = 0; k < ng; k++) s->Gdst2[k] *= scale / Lam[k];
    dst2_plans(s->nx - 1, s->ny - 1, s->Gdst2, s->Gdst1, s->plx, s->ply);
    memcpy(x, s->Gdst1, ng * sizeof(double));
}

void orc_lap_inv(int nx, int ny, const double *lam, const double *b, double *x) {
    const size_t ng = (size_t)(nx - 1) * (ny - 1);
    const double scale = 1.0 / (double)(4 * (long)nx * (long)ny);
    double *t = dalloc(ng);
    orc_dst2(nx - 1, ny - 1, b, t);
    for (size_t k = 0; k < ng; k++) t[k] *= scale / lam[k];
    orc_dst2(nx - 1, ny - 1, t, x);
    free(t);
}

/* vort2flux closure body (src/fluid.jl:178-205); Gamma is coarsified in place */
void orc_vort2flux(orc_solver *s, double *psi, double *q, double *G) {
    const int L = s->L;
    const size_t ng = (size_t)s->ng, nq = (size_t)s->nq;
    for (int lev = 2; lev <= L; lev++) coarsify(s, G + ng * (lev - 1), G + ng * (lev - 2));
    memset(psi, 0, sizeof(double) * ng * L);
    memset(s->Gbc, 0, sizeof(double) * s->nbc);
    lap_inv(s, s->lam, psi + ng * (L - 1), G + ng * (L - 1));
    curl(s, q + nq * (L - 1), psi + ng * (L - 1), s->Gbc);
    for (int lev = L - 1; lev >= 1; lev--) {
        memcpy(s->Gtmp1, G + ng * (lev - 1), ng * sizeof(double));
        get_bc(s, s->Gbc, psi + ng * lev);
        apply_bc(s, s->Gtmp1, s->Gbc, 1.0);
        lap_inv(s, s->lam, psi + ng * (lev - 1), s->Gtmp1);
        curl(s, q + nq * (lev - 1), psi + ng * (lev - 1), s->Gbc);
    }
}

/* avg_flux! (src/fluid.jl:352-370) */
static void avg_flux(const orc_solver *s, double *Q, int lev) {
    const int nx = s->nx, ny = s->ny;
    const size_t nq = (size_t)s->nq;
    const double *q = s->q + nq * (lev - 1), *q0 = s->q0 + nq * (lev - 1);
    memset(Q, 0, sizeof(double) * nq);
#pragma omp parallel for schedule(static)
    for (int j = 2; j <= ny; j++)
        for (int i = 1; i <= nx + 1; i++)
            QX(Q, i, j) = (QX(q, i, j) + QX(q, i, j - 1) + QX(q0, i, j) + QX(q0, i, j - 1)) / 2;
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= ny + 1; j++)
        for (int i = 2; i <= nx; i++)
            QY(Q, i, j) = (QY(q, i, j) + QY(q, i - 1, j) + QY(q0, i, j) + QY(q0, i - 1, j)) / 2;
}

/* direct_product! / direct_product_loops! (src/fluid.jl:372-439) */
static void direct_product(const orc_solver *s, double *fq, const double *Q, const double *G, const double *Gbc) {
    const int nx = s->nx, ny = s->ny, T = s->bT, B = s->bB, L = s->bL, R = s->bR;
    memset(fq, 0, sizeof(double) * (size_t)s->nq);
#pragma omp parallel for schedule(static)
    for (int j = 2; j <= ny - 1; j++)
        for (int i = 2; i <= nx; i++)
            QX(fq, i, j) = (QY(Q, i, j + 1) * GAM(G, i - 1, j) + QY(Q, i, j) * GAM(G, i - 1, j - 1)) / 2;
    for (int i = 2; i <= nx; i++) QX(fq, i, 1) = (QY(Q, i, 2) * GAM(G, i - 1, 1) + QY(Q, i, 1) * BC(Gbc, B + i)) / 2;
    for (int i = 2; i <= nx; i++)
        QX(fq, i, ny) = (QY(Q, i, ny) * GAM(G, i - 1, ny - 1) + QY(Q, i, ny + 1) * BC(Gbc, T + i)) / 2;
#pragma omp parallel for schedule(static)
    for (int j = 2; j <= ny; j++)
        for (int i = 2; i <= nx - 1; i++)
            QY(fq, i, j) = -(QX(Q, i + 1, j) * GAM(G, i, j - 1) + QX(Q, i, j) * GAM(G, i - 1, j - 1)) / 2;
    for (int j = 2; j <= ny; j++) QY(fq, 1, j) = -(QX(Q, 2, j) * GAM(G, 1, j - 1) + QX(Q, 1, j) * BC(Gbc, L + j)) / 2;
    for (int j = 2; j <= ny; j++)
        QY(fq, nx, j) = -(QX(Q, nx, j) * GAM(G, nx - 1, j - 1) + QX(Q, nx + 1, j) * BC(Gbc, R + j)) / 2;
}

/* nonlinear closure body (src/fluid.jl:441-455) with rhs_force (340-350) */
static void nonlinear(orc_solver *s, double *nl, const double *Gbc, int lev) {
    const size_t ng = (size_t)s->ng;
    avg_flux(s, s->qtmp1, lev);
    direct_product(s, s->qtmp2, s->qtmp1, s->G + ng * (lev - 1), Gbc);
    rot(s, nl, s->qtmp2);
    const double hc = gridstep(s, lev);
    const double f = 1 / (hc * hc);
#pragma omp parallel for schedule(static)
    for (size_t k = 0; k < ng; k++) nl[k] *= f;
}

/* base_flux! (src/fluid.jl:22-67) */
static void base_flux(orc_solver *s, const orc_step_params *prm) {
    const int nx = s->nx, ny = s->ny;
    const size_t nq = (size_t)s->nq;
    for (int lev = 1; lev <= s->L; lev++) {
        double *q0 = s->q0 + nq * (lev - 1);
        const double hc = gridstep(s, lev);
        if (!s->p.grid_moving) {
            const double u = s->fs[0], v = s->fs[1];
            for (int j = 1; j <= ny; j++)
                for (int i = 1; i <= nx + 1; i++) QX(q0, i, j) = u * hc;
            for (int j = 1; j <= ny + 1; j++)
                for (int i = 1; i <= nx; i++) QY(q0, i, j) = v * hc;
        } else {
            const double *gm = prm->grid_motion;
            const double cx = gm[0], cy = gm[1], u0x = gm[2], u0y = gm[3], th = gm[4], Om = gm[5];
            const double ct = cos(th), st = sin(th);
            const double Rv11 = Om * -st, Rv12 = Om * -ct, Rv21 = Om * ct, Rv22 = Om * -st;
            /* subdomain origin (src/problem.jl:424-429) */
            const double hb = s->p.h;
            const double x0 = s->p.x0 + nx * (hb - hc) / 2, y0 = s->p.y0 + ny * (hb - hc) / 2;
            const double ux = s->fs[0], uy = s->fs[1];
            for (int j = 1; j <= ny; j++) {
                const double y = y0 + hc / 2 + hc * (j - 1);
                for (int i = 1; i <= nx + 1; i++) {
                    const double x = x0 + hc * (i - 1);
                    const double dx = x - cx, dy = y - cy;
                    const double wx = ux - u0x - (Rv11 * dx + Rv12 * dy);
                    const double wy = uy - u0y - (Rv21 * dx + Rv22 * dy);
                    QX(q0, i, j) = hc * (ct * wx + st * wy);
                }
            }
            for (int j = 1; j <= ny + 1; j++) {
                const double y = y0 + hc * (j - 1);
                for (int i = 1; i <= nx; i++) {
                    const double x = x0 + hc / 2 + hc * (i - 1);
                    const double dx = x - cx, dy = y - cy;
                    const double wx = ux - u0x - (Rv11 * dx + Rv12 * dy);
                    const double wy = uy - u0y - (Rv21 * dx + Rv22 * dy);
                    QY(q0, i, j) = hc * (-st * wx + ct * wy);
                }
            }
        }
    }
}

/* ---- coupling.jl ---- */

/* δh, Yang3 smoothed delta (src/coupling.jl:91-148); returns delta * h */
double orc_delta_h(double rf, double rb, double dr) {
    const double r = fabs(rf - rb);
    const double r1 = r / dr;
    const double r2 = r1 * r1;
    const double r3 = r2 * r1;
    const double r4 = r3 * r1;
    if (r1 <= 1.0) {
        const double a5 = asin((1.0 / 2.0) * sqrt(3.0) * (2.0 * r1 - 1.0));
        const double a8 = sqrt(1.0 - 12.0 * r2 + 12.0 * r1);
        return 4.166666667e-2 * r4 + (-0.1388888889 + 3.472222222e-2 * a8) * r3 +
               (-7.121664902e-2 - 5.208333333e-2 * a8 + 0.2405626122 * a5) * r2 +
               (-0.2405626122 * a5 - 0.3792313933 + 0.1012731481 * a8) * r1 + 8.0187537413e-2 * a5 -
               4.195601852e-2 * a8 + 0.6485698427;
    } else if (r1 <= 2.0) {
        const double a6 = asin((1.0 / 2.0) * sqrt(3.0) * (-3.0 + 2.0 * r1));
        const double a9 = sqrt(-23.0 + 36.0 * r1 - 12.0 * r2);
        return -6.250000000e-2 * r4 + (0.4861111111 - 1.736111111e-2 * a9) * r3 +
               (-1.143175026 + 7.812500000e-2 * a9 - 0.1202813061 * a6) * r2 +
               (0.8751991178 + 0.3608439183 * a6 - 0.1548032407 * a9) * r1 - 0.2806563809 * a6 + 8.22848104e-3 +
               0.1150173611 * a9;
    } else if (r1 <= 3.0) {
        const double a1 = asin((1.0 / 2.0 * (2.0 * r1 - 5.0)) * sqrt(3.0));
        const double a7 = sqrt(-71.0 - 12.0 * r2 + 60.0 * r1);
        return 2.083333333e-2 * r4 + (3.472222222e-3 * a7 - 0.2638888889) * r3 +
               (1.214391675 - 2.604166667e-2 * a7 + 2.405626122e-2 * a1) * r2 +
               (-0.1202813061 * a1 - 2.449273192 + 7.262731481e-2 * a7) * r1 + 0.1523563211 * a1 + 1.843201677 -
               7.306134259e-2 * a7;
    }
    return 0.0;
}

/* Julia's shortest round-trip float printing, approximately (used in the error text). */
static void fmt_julia_double(char *buf, size_t n, double v) {
    for (int prec = 1; prec <= 17; prec++) {
        snprintf(buf, n, "%.*g", prec, v);
        if (strtod(buf, NULL) == v) break;
    }
    if (!strpbrk(buf, ".eni")) strncat(buf, ".0", n - strlen(buf) - 1);
}

/* _update!(reg, index, point) (src/coupling.jl:27-54); index is 1-based */
static int reg_update_one(orc_solver *s, int index, double xb, double yb, char *err, int errlen) {
    const double h = s->p.h, x0 = s->p.x0, y0 = s->p.y0;
    const int nx = s->nx, ny = s->ny;
    const int n[2] = {nx, ny};
    const double p0[2] = {x0, y0}, pb[2] = {xb, yb};
    int ix[2];
    for (int d = 0; d < 2; d++) {
        double v = nearbyint((pb[d] - p0[d]) / h + 1.0 - 0.25); /* round(Int, ...), ties to even */
        int i = (int)v;
        if (!(REG_SUPPORT < i && i <= n[d] - REG_SUPPORT)) {
            if (err) {
                char bx[40], by[40];
                fmt_julia_double(bx, sizeof bx, xb);
                fmt_julia_double(by, sizeof by, yb);
                snprintf(err, errlen, "Panel index=%d at (%s, %s) outside allowed region", index, bx, by);
            }
            return -1;
        }
        ix[d] = i;
    }
    const int p = index - 1;
    s->pc[2 * p] = ix[0];
    s->pc[2 * p + 1] = ix[1];
    double x[NSUPP], y[NSUPP];
    for (int k = -REG_SUPPORT; k <= REG_SUPPORT; k++) {
        x[k + REG_SUPPORT] = x0 + h * ((ix[0] + k) - 1);
        y[k + REG_SUPPORT] = y0 + h * ((ix[1] + k) - 1);
    }
    for (int b = 0; b < NSUPP; b++)
        for (int a = 0; a < NSUPP; a++) {
            s->w[((size_t)(p * 2 + 0)) * 49 + b * 7 + a] = orc_delta_h(x[a], xb, h) * orc_delta_h(y[b] + h / 2, yb, h);
            s->w[((size_t)(p * 2 + 1)) * 49 + b * 7 + a] = orc_delta_h(x[a] + h / 2, xb, h) * orc_delta_h(y[b], yb, h);
        }
    return 0;
}

/* regT! (src/coupling.jl:57-69): interpolation onto the panels; q is a level-1 flux */
static void regT(const orc_solver *s, double *fb, const double *q) {
    const int np = s->np;
    for (int p = 0; p < np; p++) {
        const int i0 = s->pc[2 * p] - REG_SUPPORT, j0 = s->pc[2 * p + 1] - REG_SUPPORT;
        const double *wu = s->w + (size_t)(p * 2) * 49, *wv = s->w + (size_t)(p * 2 + 1) * 49;
        double su = 0.0, sv = 0.0; /* LinearAlgebra.dot generic loop, column-major order */
        for (int b = 0; b < NSUPP; b++)
            for (int a = 0; a < NSUPP; a++) {
                su += QX(q, i0 + a, j0 + b) * wu[b * 7 + a];
                sv += QY(q, i0 + a, j0 + b) * wv[b * 7 + a];
            }
        fb[p] = su;
        fb[np + p] = sv;
    }
}

/* reg! (src/coupling.jl:72-85): regularization onto the fluid, panels in order */
static void reg(const orc_solver *s, double *q, const double *fb) {
    const int np = s->np;
    memset(q, 0, sizeof(double) * (size_t)s->nq);
    for (int p = 0; p < np; p++) {
        const int i0 = s->pc[2 * p] - REG_SUPPORT, j0 = s->pc[2 * p + 1] - REG_SUPPORT;
        const double *wu = s->w + (size_t)(p * 2) * 49, *wv = s->w + (size_t)(p * 2 + 1) * 49;
        for (int b = 0; b < NSUPP; b++)
            for (int a = 0; a < NSUPP; a++) {
                QX(q, i0 + a, j0 + b) += wu[b * 7 + a] * fb[p];
                QY(q, i0 + a, j0 + b) += wv[b * 7 + a] * fb[np + p];
            }
    }
}

/* B_operator closure body (src/coupling.jl:163-176) */
void orc_apply_B(orc_solver *s, double *x, const double *z) {
    const size_t ng = (size_t)s->ng;
    memset(s->Gtmp, 0, sizeof(double) * ng * s->L);
    reg(s, s->qtmp2, z);
    rot(s, s->Gtmp2, s->qtmp2);
    lap_inv(s, s->Limpl[0], s->Gtmp, s->Gtmp2);
    orc_vort2flux(s, s->psitmp, s->qtmp, s->Gtmp);
    regT(s, x, s->qtmp);
}

/* LU with partial pivoting, then inverse (stands in for LinearAlgebra.inv = getrf+getri) */
static int invert(int n, double *A) {
    int *piv = (int *)malloc(sizeof(int) * (size_t)n);
    for (int k = 0; k < n; k++) {
        int pr = k;
        double mx = fabs(A[k + (size_t)n * k]);
        for (int i = k + 1; i < n; i++)
            if (fabs(A[i + (size_t)n * k]) > mx) {
                mx = fabs(A[i + (size_t)n * k]);
                pr = i;
            }
        piv[k] = pr;
        if (mx == 0.0) {
            free(piv);
            return -1;
        }
        if (pr != k)
            for (int j = 0; j < n; j++) {
                double t = A[k + (size_t)n * j];
                A[k + (size_t)n * j] = A[pr + (size_t)n * j];
                A[pr + (size_t)n * j] = t;
            }
        const double d = A[k + (size_t)n * k];
        for (int i = k + 1; i < n; i++) A[i + (size_t)n * k] /= d;
#pragma omp parallel for schedule(static)
        for (int j = k + 1; j < n; j++) {
            const double f = A[k + (size_t)n * j];
            if (f != 0.0)
                for (int i = k + 1; i < n; i++) A[i + (size_t)n * j] -= A[i + (size_t)n * k] * f;
        }
    }
    /* inverse: solve A X = I column by column (X overwrites a copy) */
    double *LU = (double *)malloc(sizeof(double) * (size_t)n * n);
    memcpy(LU, A, sizeof(double) * (size_t)n * n);
#pragma omp parallel for schedule(static)
    for (int c = 0; c < n; c++) {
        double *x = A + (size_t)n * c;
        for (int i = 0; i < n; i++) x[i] = 0.0;
        /* apply the row permutation to e_c */
        int pos = c;
        double *e = (double *)calloc((size_t)n, sizeof(double));
        e[pos] = 1.0;
        for (int k = 0; k < n; k++)
            if (piv[k] != k) {
                double t = e[k];
                e[k] = e[piv[k]];
                e[piv[k]] = t;
            }
        for (int i = 0; i < n; i++) {
            double v = e[i];
            for (int k = 0; k < i; k++) v -= LU[i + (size_t)n * k] * x[k];
            x[i] = v;
        }
        for (int i = n - 1; i >= 0; i--) {
            double v = x[i];
            for (int k = i + 1; k < n; k++) v -= LU[i + (size_t)n * k] * x[k];
            x[i] = v / LU[i + (size_t)n * i];
        }
        free(e);
    }
    free(LU);
    free(piv);
    return 0;
}

static double dot(int n, const double *a, const double *b) {
    double s = 0.0;
    for (int i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}

/* IterativeSolvers.jl cg! (plain CG, x is the initial guess; stop when
 * ||r|| <= max(reltol*||r0||, abstol) or after maxiter iterations).  Called at
 * src/coupling.jl:198-201. */
static int cg_solve(orc_solver *s, double *x, const double *b) {
    const int n = 2 * s->np;
    double *u = dalloc(n), *r = dalloc(n), *c = dalloc(n);
    memcpy(r, b, sizeof(double) * n);
    orc_apply_B(s, c, x);
    for (int i = 0; i < n; i++) r[i] -= c[i];
    double residual = sqrt(dot(n, r, r));
    const double tol = fmax(s->p.cg_reltol * residual, s->p.cg_abstol);
    double prev = 1.0;
    int it = 0;
    while (!(it >= s->p.cg_maxiter || residual <= tol)) {
        const double beta = residual * residual / (prev * prev);
        for (int i = 0; i < n; i++) u[i] = r[i] + beta * u[i];
        orc_apply_B(s, c, u);
        const double alpha = residual * residual / dot(n, u, c);
        for (int i = 0; i < n; i++) x[i] += alpha * u[i];
        for (int i = 0; i < n; i++) r[i] -= alpha * c[i];
        prev = residual;
        residual = sqrt(dot(n, r, r));
        it++;
    }
    free(u);
    free(r);
    free(c);
    return it;
}

/* ---- bodies.jl ---- */

/* _init_body_motion! (src/bodies.jl:33-41) with _init! (1-11) */
static int init_body_motion(orc_solver *s, char *err, int errlen) {
    for (int b = 0; b < s->p.nbody; b++) {
        if (s->body_kind[b] != ORC_BODY_STATIC) continue; /* _init!(::MovingRigidBody) = false */
        for (int p = s->body_start[b]; p < s->body_start[b + 1]; p++) {
            s->xb[p] = s->ref_xb[p];
            s->xb[s->np + p] = s->ref_xb[s->np + p];
            s->ds[p] = s->ref_ds[p];
            s->ub[p] = 0.0;
            s->ub[s->np + p] = 0.0;
        }
        for (int p = s->body_start[b]; p < s->body_start[b + 1]; p++)
            if (reg_update_one(s, p + 1, s->xb[p], s->xb[s->np + p], err, errlen)) return -1;
    }
    return 0;
}

/* _update_body_motion! (src/bodies.jl:43-51) with _update!(::MovingRigidBody) (12-31) */
static int update_body_motion(orc_solver *s, const orc_step_params *prm, char *err, int errlen) {
    for (int b = 0; b < s->p.nbody; b++) {
        if (s->body_kind[b] != ORC_BODY_MOVING_RIGID) continue;
        const double *m = prm->body_motion + 6 * b;
        const double r0x = m[0], r0y = m[1], v0x = m[2], v0y = m[3], ang = m[4], Om = m[5];
        const double c = cos(ang), sn = sin(ang);
        const double Rv11 = Om * -sn, Rv12 = Om * -c, Rv21 = Om * c, Rv22 = Om * -sn;
        for (int p = s->body_start[b]; p < s->body_start[b + 1]; p++) {
            const double rx = s->ref_xb[p], ry = s->ref_xb[s->np + p];
            s->xb[p] = r0x + (c * rx + -sn * ry);
            s->xb[s->np + p] = r0y + (sn * rx + c * ry);
            s->ub[p] = v0x + (Rv11 * rx + Rv12 * ry);
            s->ub[s->np + p] = v0y + (Rv21 * rx + Rv22 * ry);
        }
        for (int p = s->body_start[b]; p < s->body_start[b + 1]; p++)
            if (reg_update_one(s, p + 1, s->xb[p], s->xb[s->np + p], err, errlen)) return -1;
    }
    return 0;
}

/* ---- solver.jl ---- */

int orc_nthreads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

void orc_destroy(orc_solver *s) {
    if (!s) return;
    double *bufs[] = {s->q,      s->q0,    s->G,     s->psi,   s->nonlin[0], s->nonlin[1], s->xb,    s->ds,
                      s->ub,     s->Fbt,   s->fb,    s->qs,    s->Gs,        s->Gbc,       s->Gtmp,  s->psitmp,
                      s->qtmp,   s->Ftmp,  s->Gtmp1, s->Gtmp2, s->Gtmp3,     s->qtmp1,     s->qtmp2, s->Gdst1,
                      s->Gdst2,  s->lam,   s->w,     s->Binv,  s->ref_xb,    s->ref_ds};
    for (size_t i = 0; i < sizeof(bufs) / sizeof(bufs[0]); i++) free(bufs[i]);
    if (s->Lexpl)
        for (int l = 0; l < s->L; l++) {
            free(s->Lexpl[l]);
            free(s->Limpl[l]);
        }
    free(s->Lexpl);
    free(s->Limpl);
    free(s->pc);
    free(s->body_kind);
    free(s->body_start);
    fft_plan_free(s->plx);
    fft_plan_free(s->ply);
    free(s);
}

/* CnabSolver(state) (src/solver.jl:84-150) on a fresh State(prob) (problem.jl:640-665) */
orc_solver *orc_create(const orc_problem *p, char *err, int errlen) {
    if (p->nx < 8 || p->ny < 8 || p->nlevel < 1 || p->npanel < 1) {
        if (err) snprintf(err, errlen, "invalid problem sizes");
        return NULL;
    }
    orc_solver *s = (orc_solver *)calloc(1, sizeof(orc_solver));
    s->p = *p;
    s->nx = p->nx;
    s->ny = p->ny;
    s->L = p->nlevel;
    s->np = p->npanel;
    s->nu = (s->nx + 1) * s->ny;
    s->nv = s->nx * (s->ny + 1);
    s->nq = s->nu + s->nv;
    s->ng = (s->nx - 1) * (s->ny - 1);
    s->nbc = 2 * (s->nx + 1) + 2 * (s->ny + 1);
    s->bL = 0;
    s->bR = s->ny + 1;
    s->bB = 2 * (s->ny + 1);
    s->bT = 2 * (s->ny + 1) + s->nx + 1;
    s->body_kind = (int32_t *)malloc(sizeof(int32_t) * p->nbody);
    s->body_start = (int32_t *)malloc(sizeof(int32_t) * (p->nbody + 1));
    memcpy(s->body_kind, p->body_kind, sizeof(int32_t) * p->nbody);
    memcpy(s->body_start, p->body_start, sizeof(int32_t) * (p->nbody + 1));
    s->ref_xb = dalloc(2 * (size_t)s->np);
    s->ref_ds = dalloc(s->np);
    memcpy(s->ref_xb, p->body_xb, sizeof(double) * 2 * s->np);
    memcpy(s->ref_ds, p->body_ds, sizeof(double) * s->np);
    s->p.body_kind = s->body_kind;
    s->p.body_start = s->body_start;
    s->p.body_xb = s->ref_xb;
    s->p.body_ds = s->ref_ds;
    const size_t nq = s->nq, ng = s->ng, L = s->L, np = s->np;
    s->q = dalloc(nq * L);
    s->q0 = dalloc(nq * L);
    s->G = dalloc(ng * L);
    s->psi = dalloc(ng * L);
    s->nonlin[0] = dalloc(ng * L);
    s->nonlin[1] = dalloc(ng * L);
    s->xb = dalloc(2 * np);
    s->ds = dalloc(np);
    s->ub = dalloc(2 * np);
    s->Fbt = dalloc(2 * np);
    s->fb = dalloc(2 * np);
    s->t0 = 0.0;
    orc_set_index(s, 0);
    s->qs = dalloc(nq * L);
    s->Gs = dalloc(ng * L);
    s->Gbc = dalloc(s->nbc);
    s->Gtmp = dalloc(ng * L);
    s->psitmp = dalloc(ng * L);
    s->qtmp = dalloc(nq * L);
    s->Ftmp = dalloc(2 * np);
    s->Gtmp1 = dalloc(ng);
    s->Gtmp2 = dalloc(ng);
    s->Gtmp3 = dalloc(ng);
    s->qtmp1 = dalloc(nq);
    s->qtmp2 = dalloc(nq);
    s->Gdst1 = dalloc(ng);
    s->Gdst2 = dalloc(ng);
    s->plx = fft_plan_new(2 * s->nx);
    s->ply = fft_plan_new(2 * s->ny);
    s->lam = dalloc(ng);
    orc_lap_eigs(s->nx, s->ny, s->lam);
    s->pc = (int *)calloc(2 * np, sizeof(int));
    s->w = dalloc(np * 2 * 49);
    for (int b = 0; b < p->nbody; b++)
        if (s->body_kind[b] != ORC_BODY_STATIC) s->any_moving = 1;
    if (init_body_motion(s, err, errlen)) {
        orc_destroy(s);
        return NULL;
    }
    /* A_operators (src/fluid.jl:121-143) */
    s->Lexpl = (double **)calloc(L, sizeof(double *));
    s->Limpl = (double **)calloc(L, sizeof(double *));
    for (int lev = 1; lev <= s->L; lev++) {
        const double hc = gridstep(s, lev), dt = p->dt, Re = p->Re;
        s->Lexpl[lev - 1] = dalloc(ng);
        s->Limpl[lev - 1] = dalloc(ng);
        for (size_t k = 0; k < ng; k++) {
            s->Lexpl[lev - 1][k] = 1.0 / (1 - s->lam[k] * dt / (2 * Re * (hc * hc)));
            s->Limpl[lev - 1][k] = 1 + s->lam[k] * dt / (2 * Re * (hc * hc));
        }
    }
    /* Binv_operator (src/coupling.jl:179-192): static bodies precompute inv(B) */
    if (!s->any_moving && p->timing_only) {
        s->Binv = dalloc((size_t)(2 * s->np) * (2 * s->np));
    } else if (!s->any_moving) {
        const int n = 2 * s->np;
        s->Binv = dalloc((size_t)n * n);
        double *x = dalloc(n);
        for (int i = 0; i < n; i++) { /* _linear_op_matrix (coupling.jl:204-215) */
            x[i] = 1;
            if (i > 0) x[i - 1] = 0;
            orc_apply_B(s, s->Binv + (size_t)n * i, x);
        }
        free(x);
        if (invert(n, s->Binv)) {
            if (err) snprintf(err, errlen, "B is singular");
            orc_destroy(s);
            return NULL;
        }
    }
    return s;
}

/* get_trial_state closure body (src/fluid.jl:467-506) */
static void get_trial_state(orc_solver *s) {
    const size_t ng = (size_t)s->ng;
    const double dt = s->p.dt, Re = s->p.Re;
    const double beta[2] = {1.5, -0.5};
    double *bc = s->Gbc, *rhsbc = s->Gtmp2, *rhs = s->Gtmp3;
    for (int lev = s->L; lev >= 1; lev--) {
        memset(bc, 0, sizeof(double) * s->nbc);
        memset(rhsbc, 0, sizeof(double) * ng);
        const double hc = gridstep(s, lev);
        if (lev < s->L) {
            get_bc(s, bc, s->G + ng * lev);
            apply_bc(s, rhsbc, bc, 0.25 * dt / (Re * (hc * hc)));
        }
        for (int k = 0; k < s->nbc; k++) bc[k] *= 0.25;
        nonlinear(s, s->nonlin[0] + ng * (lev - 1), bc, lev);
        lap_inv(s, s->Lexpl[lev - 1], rhs, s->G + ng * (lev - 1));
        for (int n = 0; n < 2; n++) {
            const double *nl = s->nonlin[n] + ng * (lev - 1);
            const double f = dt * beta[n];
            for (size_t k = 0; k < ng; k++) rhs[k] += f * nl[k];
        }
        for (size_t k = 0; k < ng; k++) rhs[k] += rhsbc[k];
        lap_inv(s, s->Limpl[lev - 1], s->Gs + ng * (lev - 1), rhs);
    }
    double *t = s->nonlin[0]; /* _cycle! (src/fluid.jl:510) */
    s->nonlin[0] = s->nonlin[1];
    s->nonlin[1] = t;
    orc_vort2flux(s, s->psi, s->qs, s->Gs);
}

/* couple_surface_rigid closure body (src/coupling.jl:236-250) */
static void couple_surface(orc_solver *s) {
    const size_t nq = (size_t)s->nq;
    const int n = 2 * s->np;
    for (size_t k = 0; k < nq; k++) s->qtmp1[k] = s->qs[k] + s->q0[k];
    regT(s, s->Ftmp, s->qtmp1);
    const double h = s->p.h;
    for (int k = 0; k < n; k++) s->Ftmp[k] -= s->ub[k] * h;
    if (s->Binv) {
        for (int i = 0; i < n; i++) {
            double acc = 0.0;
            for (int j = 0; j < n; j++) acc += s->Binv[i + (size_t)n * j] * s->Ftmp[j];
            s->Fbt[i] = acc;
        }
        s->last_cg_iters = 0;
    } else {
        s->last_cg_iters = cg_solve(s, s->Fbt, s->Ftmp);
    }
}

/* project_circ closure body (src/coupling.jl:218-230) */
static void project_circ(orc_solver *s) {
    const size_t ng = (size_t)s->ng;
    memcpy(s->G, s->Gs, sizeof(double) * ng * s->L);
    reg(s, s->qtmp1, s->Fbt);
    rot(s, s->Gtmp2, s->qtmp1);
    lap_inv(s, s->Limpl[0], s->Gs, s->Gtmp2);
    for (size_t k = 0; k < ng; k++) s->G[k] -= s->Gs[k];
}

void orc_reg_rot(orc_solver *s, const double *f, double *gamma1) {
    reg(s, s->qtmp2, f);
    rot(s, gamma1, s->qtmp2);
}

void orc_regT(orc_solver *s, const double *q1, double *f) { regT(s, f, q1); }

void orc_update_vars(orc_solver *s) {
    const double dt = s->p.dt, h = s->p.h;
    for (int k = 0; k < 2 * s->np; k++) s->fb[k] = s->Fbt[k] * h / dt;
}

/* advance!(::CnabSolver) (src/solver.jl:155-190) */
int orc_advance(orc_solver *s, const orc_step_params *prm, char *err, int errlen) {
    orc_set_index(s, s->index + 1);
    s->fs[0] = prm->freestream[0];
    s->fs[1] = prm->freestream[1];
    if (update_body_motion(s, prm, err, errlen)) return -1;
    base_flux(s, prm);
    get_trial_state(s);
    couple_surface(s);
    project_circ(s);
    orc_vort2flux(s, s->psi, s->q, s->G);
    orc_update_vars(s);
    return 0;
}

/* ---- accessors ---- */
double *orc_q(orc_solver *s) { return s->q; }
double *orc_q0(orc_solver *s) { return s->q0; }
double *orc_gamma(orc_solver *s) { return s->G; }
double *orc_psi(orc_solver *s) { return s->psi; }
double *orc_nonlin(orc_solver *s, int k) { return s->nonlin[k ? 1 : 0]; }
double *orc_xb(orc_solver *s) { return s->xb; }
double *orc_ds(orc_solver *s) { return s->ds; }
double *orc_ub(orc_solver *s) { return s->ub; }
double *orc_fbt(orc_solver *s) { return s->Fbt; }
double *orc_fb(orc_solver *s) { return s->fb; }
double *orc_freestream(orc_solver *s) { return s->fs; }
int64_t orc_get_index(orc_solver *s) { return s->index; }
/* set_time_index! (src/problem.jl:705-708) */
void orc_set_index(orc_solver *s, int64_t index) {
    s->index = index;
    s->t = s->t0 + s->p.dt * (double)(index - 1);
}
double orc_get_t(orc_solver *s) { return s->t; }
double orc_get_t0(orc_solver *s) { return s->t0; }
void orc_set_t0(orc_solver *s, double t0) {
    s->t0 = t0;
    orc_set_index(s, s->index);
}
int orc_last_cg_iters(orc_solver *s) { return s->last_cg_iters; }
int orc_binv(orc_solver *s, double *out) {
    if (!s->Binv) return 0;
    const size_t n = 2 * (size_t)s->np;
    memcpy(out, s->Binv, sizeof(double) * n * n);
    return 1;
}

int orc_set_binv(orc_solver *s, const double *in) {
    if (!s->Binv) return 0;
    const size_t n = 2 * (size_t)s->np;
    memcpy(s->Binv, in, sizeof(double) * n * n);
    return 1;
}
