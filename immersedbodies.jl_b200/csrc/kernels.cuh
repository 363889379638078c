// kernels.cuh -- FP64 device kernels of the IBPM time step.
//
// Index helpers use the reference's 1-based (i, j) so each kernel reads like
// the loop it restates.  Layouts (column-major, x fastest):
//   Gamma-like field  (nx-1) x (ny-1):  GI(i,j) = (i-1) + (nx-1)(j-1)
//   x flux  (nx+1) x ny:                UI(i,j) = (i-1) + (nx+1)(j-1)
//   y flux  nx x (ny+1):                VI(i,j) = nu + (i-1) + nx(j-1)
// A "batch" index b selects a field: either the level (b = lev-1, the trial
// solves) or an independent right-hand side (the B^-1 setup columns).
#pragma once
#include "fft_dst.cuh"

namespace ibpm {

struct Grid {
    int nx, ny, L;
    double h, x0, y0, Re, dt;
    int grid_moving;
};

// Per-step host-callback values, resident in device memory.
struct StepDev {
    double fs[2];   // freestream velocity
    double gm[6];   // grid motion: center(2), vel(2), angle, angular_vel
};

#define GI(i, j) ((long long)((i)-1) + (long long)(g.nx - 1) * (long long)((j)-1))
#define UI(i, j) ((long long)((i)-1) + (long long)(g.nx + 1) * (long long)((j)-1))
#define VI(i, j) (nu + (long long)((i)-1) + (long long)g.nx * (long long)((j)-1))

enum { SIDE_B = 0, SIDE_T = 1, SIDE_L = 2, SIDE_R = 3 };

__device__ __forceinline__ double gridstep(const Grid &g, int lev) { return ldexp(g.h, lev - 1); }

// get_bc! (src/fluid.jl:278-306), one entry: rbc[side offset + ibc] from the
// coarser level's field r.  r == nullptr means zero boundary values.
__device__ __forceinline__ double getbc(const double *__restrict__ r, const Grid &g, int side, int ibc) {
    if (r == nullptr) return 0.0;
    const int nx = g.nx, ny = g.ny;
    if (side == SIDE_B || side == SIDE_T) {
        const int row = side == SIDE_B ? ny / 4 : 3 * ny / 4;
        if (ibc & 1) return r[GI(nx / 4 + (ibc - 1) / 2, row)];
        const int i = nx / 4 + ibc / 2;
        return 0.5 * (r[GI(i, row)] + r[GI(i - 1, row)]);
    }
    const int col = side == SIDE_L ? nx / 4 : 3 * nx / 4;
    if (ibc & 1) return r[GI(col, ny / 4 + (ibc - 1) / 2)];
    const int j = ny / 4 + ibc / 2;
    return 0.5 * (r[GI(col, j)] + r[GI(col, j - 1)]);
}

// apply_bc! contribution at (i, j) (src/fluid.jl:308-338), accumulated in the
// reference's order (bottom/top rows first, then left/right columns).
__device__ __forceinline__ double apply_bc_at(double v, const double *__restrict__ r, const Grid &g, int i, int j,
                                              double fac) {
    if (j == 1) v += fac * getbc(r, g, SIDE_B, i + 1);
    if (j == g.ny - 1) v += fac * getbc(r, g, SIDE_T, i + 1);
    if (i == 1) v += fac * getbc(r, g, SIDE_L, j + 1);
    if (i == g.nx - 1) v += fac * getbc(r, g, SIDE_R, j + 1);
    return v;
}

__device__ __forceinline__ bool on_ring(const Grid &g, int i, int j) {
    return j == 1 || j == g.ny - 1 || i == 1 || i == g.nx - 1;
}

// base_flux! (src/fluid.jl:22-67), evaluated per face instead of stored.
__device__ __forceinline__ double base_flux_x(const Grid &g, const StepDev *__restrict__ prm, int lev, int i, int j) {
    const double hc = gridstep(g, lev);
    if (!g.grid_moving) return prm->fs[0] * hc;
    const double cx = prm->gm[0], cy = prm->gm[1], th = prm->gm[4], Om = prm->gm[5];
    double st, ct;
    sincos(th, &st, &ct);
    const double x0 = g.x0 + g.nx * (g.h - hc) / 2, y0 = g.y0 + g.ny * (g.h - hc) / 2;
    const double x = x0 + hc * (i - 1), y = y0 + hc / 2 + hc * (j - 1);
    const double dx = x - cx, dy = y - cy;
    const double wx = prm->fs[0] - prm->gm[2] - ((Om * -st) * dx + (Om * -ct) * dy);
    const double wy = prm->fs[1] - prm->gm[3] - ((Om * ct) * dx + (Om * -st) * dy);
    return hc * (ct * wx + st * wy);
}

__device__ __forceinline__ double base_flux_y(const Grid &g, const StepDev *__restrict__ prm, int lev, int i, int j) {
    const double hc = gridstep(g, lev);
    if (!g.grid_moving) return prm->fs[1] * hc;
    const double cx = prm->gm[0], cy = prm->gm[1], th = prm->gm[4], Om = prm->gm[5];
    double st, ct;
    sincos(th, &st, &ct);
    const double x0 = g.x0 + g.nx * (g.h - hc) / 2, y0 = g.y0 + g.ny * (g.h - hc) / 2;
    const double x = x0 + hc / 2 + hc * (i - 1), y = y0 + hc * (j - 1);
    const double dx = x - cx, dy = y - cy;
    const double wx = prm->fs[0] - prm->gm[2] - ((Om * -st) * dx + (Om * -ct) * dy);
    const double wy = prm->fs[1] - prm->gm[3] - ((Om * ct) * dx + (Om * -st) * dy);
    return hc * (-st * wx + ct * wy);
}

// ---------------------------------------------------------------------------
// Line-pass kernels
// ---------------------------------------------------------------------------

// Prologue: plain field
struct InPlain {
    const double *p;
    long long bs;
    int ld;
    __device__ __forceinline__ double operator()(int b, int i, int j) const {
        return p[b * bs + (long long)(i - 1) + (long long)ld * (j - 1)];
    }
};

// Prologue of vort2flux's telescoping solve (src/fluid.jl:194-197):
// Gamma_tmp = Gamma[:, lev]; apply_bc!(Gamma_tmp, get_bc(psi[:, lev+1]); fac=1)
struct InBC {
    const double *gam;
    const double *coarse;
    long long bs, cbs;
    Grid g;
    __device__ __forceinline__ double operator()(int b, int i, int j) const {
        const double *G = gam + b * bs;
        double v = G[GI(i, j)];
        if (on_ring(g, i, j)) v = apply_bc_at(v, coarse + b * cbs, g, i, j, 1.0);
        return v;
    }
};

// Regularised flux on the panels' bounding box (compact patch):
// patch[(i - i0) + pw (j - j0)] for x faces, offset pw*ph for y faces.
struct Patch {
    const double *p;
    const int *bbox;      // device: i0, i1, j0, j1 (1-based face indices)
    long long bs;
    __device__ __forceinline__ double get(int b, int comp, int i, int j) const {
        const int i0 = bbox[0], i1 = bbox[1], j0 = bbox[2], j1 = bbox[3];
        if (i < i0 || i > i1 || j < j0 || j > j1) return 0.0;
        const int pw = i1 - i0 + 1, ph = j1 - j0 + 1;
        return p[b * bs + (long long)comp * pw * ph + (i - i0) + (long long)pw * (j - j0)];
    }
};

// Prologue rot!(Gamma, reg!(q, f)) (src/fluid.jl:101-111 after src/coupling.jl:72-85),
// evaluated from the regularised patch.
struct InRegRot {
    Patch pt;
    __device__ __forceinline__ double operator()(int b, int I, int J) const {
        return (pt.get(b, 0, I + 1, J) - pt.get(b, 0, I + 1, J + 1)) + (pt.get(b, 1, I + 1, J + 1) - pt.get(b, 1, I, J + 1));
    }
};

// Epilogue: plain store
struct OutPlain {
    double *p;
    long long bs;
    int ld;
    __device__ __forceinline__ void operator()(int b, int i, int j, double v) const {
        p[b * bs + (long long)(i - 1) + (long long)ld * (j - 1)] = v;
    }
};

// Epilogue of project_circ (src/coupling.jl:227): Gamma[:, 1] .-= x
struct OutSub {
    double *p;
    long long bs;
    int ld;
    __device__ __forceinline__ void operator()(int b, int i, int j, double v) const {
        double *q = p + b * bs + (long long)(i - 1) + (long long)ld * (j - 1);
        *q = *q - v;
    }
};

// Epilogue of rhs = A Gamma in get_trial_state (src/fluid.jl:485-493):
// rhs = ((A Gamma + dt b1 N1) + dt b2 N2) + rhsbc, rhsbc = apply_bc!(0, get_bc(Gamma[:, lev+1]); fac)
struct OutTrialRhs {
    double *rhs;
    const double *n1, *n2;
    const double *gam_old;  // Gamma at all levels (level stride bs)
    long long bs;
    Grid g;
    __device__ __forceinline__ void operator()(int b, int i, int j, double v) const {
        const int lev = b + 1;
        const long long k = b * bs + GI(i, j);
        const double f1 = g.dt * 1.5, f2 = g.dt * -0.5;
        double r = (v + f1 * n1[k]) + f2 * n2[k];
        if (lev < g.L && on_ring(g, i, j)) {
            const double hc = gridstep(g, lev);
            const double fac = 0.25 * g.dt / (g.Re * (hc * hc));
            r = r + apply_bc_at(0.0, gam_old + (b + 1) * bs, g, i, j, fac);
        }
        rhs[k] = r;
    }
};

// Spectral multipliers scale / Lambda (src/fluid.jl:117-134)
enum { MULT_LAPINV = 0, MULT_AEXPL = 1, MULT_AIMPL = 2 };
struct Mult {
    int mode;
    const double *cx;   // cos(pi i / nx), i = 0..nx
    const double *cy;   // cos(pi j / ny), j = 0..ny
    double scale;       // 1 / (4 nx ny)
    double h, Re, dt;
    int lev0, levstep;  // level of batch b: lev0 + b * levstep
    __device__ __forceinline__ double operator()(int b, int i, int j) const {
        const double lam = -2 * ((__ldg(&cx[i]) + __ldg(&cy[j])) - 2);
        if (mode == MULT_LAPINV) return scale / lam;
        const int lev = lev0 + b * levstep;
        const double hc = ldexp(h, lev - 1);
        const double den = 2 * Re * (hc * hc);
        if (mode == MULT_AEXPL) {
            const double Lam = 1.0 / (1 - lam * dt / den);
            return scale / Lam;
        }
        const double Lam = 1 + lam * dt / den;
        return scale / Lam;
    }
};

// X pass: DST along x of rows (ja, jb) = (2p+1, 2p+2) of each batch field.
template <int NG, class In, class Out>
__global__ void __launch_bounds__(kTPF *NG) xpass_kernel(In in, Out out, Plan pl, int nrows) {
    extern __shared__ double2 smem[];
    const int M = pl.M;
    const int g = threadIdx.x / kTPF, t = threadIdx.x % kTPF;
    double2 *buf = smem + g * (M + 1);
    double2 *wt = smem + NG * (M + 1) + 2 * g;
    const int b = blockIdx.y;
    const int pair = blockIdx.x * NG + g;
    const int ja = 2 * pair + 1, jb = 2 * pair + 2;
    const bool va = ja <= nrows, vb = jb <= nrows;
    for (int i = t; i <= M; i += kTPF) {
        double2 z = make_double2(0.0, 0.0);
        if (i >= 1 && i < M) {
            if (va) z.x = in(b, i, ja);
            if (vb) z.y = in(b, i, jb);
        }
        buf[i] = z;
    }
    __syncthreads();
    dst_inplace(buf, pl, t, wt);
    for (int i = 1 + t; i < M; i += kTPF) {
        const double2 y = buf[i];
        if (va) out(b, i, ja, y.x);
        if (vb) out(b, i, jb, y.y);
    }
}

// Y pass: for each column i, x[i, :] = DST_y(mult(i, :) * DST_y(in[i, :])).
// A block owns 2*NG adjacent columns; loads and stores are row-coalesced.
template <int NG>
__global__ void __launch_bounds__(kTPF *NG) ypass_kernel(const double *__restrict__ in, double *__restrict__ out,
                                                         long long bs, int ncols, Plan pl, Mult mult) {
    extern __shared__ double2 smem[];
    const int M = pl.M;
    const int g = threadIdx.x / kTPF, t = threadIdx.x % kTPF;
    double2 *buf = smem + g * (M + 1);
    double2 *wt = smem + NG * (M + 1) + 2 * g;
    const int b = blockIdx.y;
    const int c0 = blockIdx.x * 2 * NG;  // 0-based first column of the block
    const double *src = in + b * bs;
    double *dst = out + b * bs;
    constexpr int W = 2 * NG;
    for (int e = threadIdx.x; e < W * (M + 1); e += blockDim.x) {
        const int c = e % W, jj = e / W;
        const int col = c0 + c;
        double v = 0.0;
        if (jj >= 1 && jj < M && col < ncols) v = src[col + (long long)ncols * (jj - 1)];
        double *slot = reinterpret_cast<double *>(smem + (c >> 1) * (M + 1) + jj) + (c & 1);
        *slot = v;
    }
    __syncthreads();
    dst_inplace(buf, pl, t, wt);
    {
        const int ia = c0 + 2 * g + 1, ib = c0 + 2 * g + 2;  // 1-based columns
        for (int jj = 1 + t; jj < M; jj += kTPF) {
            double2 y = buf[jj];
            y.x *= (ia <= ncols) ? mult(b, ia, jj) : 0.0;
            y.y *= (ib <= ncols) ? mult(b, ib, jj) : 0.0;
            buf[jj] = y;
        }
    }
    __syncthreads();
    dst_inplace(buf, pl, t, wt);
    for (int e = threadIdx.x; e < W * (M + 1); e += blockDim.x) {
        const int c = e % W, jj = e / W;
        const int col = c0 + c;
        if (jj >= 1 && jj < M && col < ncols) {
            const double *slot = reinterpret_cast<const double *>(smem + (c >> 1) * (M + 1) + jj) + (c & 1);
            dst[col + (long long)ncols * (jj - 1)] = *slot;
        }
    }
}

// ---------------------------------------------------------------------------
// Stencil kernels
// ---------------------------------------------------------------------------

// nonlinear (src/fluid.jl:441-455) = rot(direct_product(avg_flux(q + q0), Gamma, Gamma_bc)) / hc^2,
// with Gamma_bc = 0.25 get_bc(Gamma[:, lev+1]) (src/fluid.jl:473-483).  Batch b = level - 1.
struct NonlinArgs {
    const double *q;      // nq x L
    const double *gam;    // ng x L
    double *out;          // ng x L (state.nonlin[1])
    const StepDev *prm;
    Grid g;
};

__device__ __forceinline__ double avg_qx(const NonlinArgs &a, const double *q, int lev, int i, int j) {
    const Grid &g = a.g;
    return (q[UI(i, j)] + q[UI(i, j - 1)] + base_flux_x(g, a.prm, lev, i, j) + base_flux_x(g, a.prm, lev, i, j - 1)) / 2;
}
__device__ __forceinline__ double avg_qy(const NonlinArgs &a, const double *q, long long nu, int lev, int i, int j) {
    const Grid &g = a.g;
    return (q[VI(i, j)] + q[VI(i - 1, j)] + base_flux_y(g, a.prm, lev, i, j) + base_flux_y(g, a.prm, lev, i - 1, j)) / 2;
}

__global__ void nonlinear_kernel(NonlinArgs a) {
    const Grid &g = a.g;
    const int nx = g.nx, ny = g.ny;
    const int I = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int J = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int b = blockIdx.z, lev = b + 1;
    if (I > nx - 1 || J > ny - 1) return;
    const long long nq = (long long)(nx + 1) * ny + (long long)nx * (ny + 1), ng = (long long)(nx - 1) * (ny - 1);
    const long long nu = (long long)(nx + 1) * ny;
    const double *q = a.q + b * nq;
    const double *G = a.gam + b * ng;
    const double *C = lev < g.L ? a.gam + (b + 1) * ng : nullptr;
    // x-flux product at (i, j), i in 2..nx  (direct_product_loops!, fluid.jl:396-415)
    auto fqx = [&](int i, int j) -> double {
        if (j == 1)
            return (avg_qy(a, q, nu, lev, i, 2) * G[GI(i - 1, 1)] +
                    avg_qy(a, q, nu, lev, i, 1) * (getbc(C, g, SIDE_B, i) * 0.25)) / 2;
        if (j == ny)
            return (avg_qy(a, q, nu, lev, i, ny) * G[GI(i - 1, ny - 1)] +
                    avg_qy(a, q, nu, lev, i, ny + 1) * (getbc(C, g, SIDE_T, i) * 0.25)) / 2;
        return (avg_qy(a, q, nu, lev, i, j + 1) * G[GI(i - 1, j)] + avg_qy(a, q, nu, lev, i, j) * G[GI(i - 1, j - 1)]) / 2;
    };
    // y-flux product at (i, j), j in 2..ny  (fluid.jl:417-436)
    auto fqy = [&](int i, int j) -> double {
        if (i == 1)
            return -(avg_qx(a, q, lev, 2, j) * G[GI(1, j - 1)] + avg_qx(a, q, lev, 1, j) * (getbc(C, g, SIDE_L, j) * 0.25)) / 2;
        if (i == nx)
            return -(avg_qx(a, q, lev, nx, j) * G[GI(nx - 1, j - 1)] +
                     avg_qx(a, q, lev, nx + 1, j) * (getbc(C, g, SIDE_R, j) * 0.25)) / 2;
        return -(avg_qx(a, q, lev, i + 1, j) * G[GI(i, j - 1)] + avg_qx(a, q, lev, i, j) * G[GI(i - 1, j - 1)]) / 2;
    };
    // rot! at Gamma(I, J) with i = I+1, j = J+1 (fluid.jl:106-108)
    const double r = (fqx(I + 1, J) - fqx(I + 1, J + 1)) + (fqy(I + 1, J + 1) - fqy(I, J + 1));
    const double hc = gridstep(g, lev);
    a.out[b * ng + GI(I, J)] = r * (1 / (hc * hc));
}

// 4-argument curl! (src/fluid.jl:230-276) with psi_bc = get_bc(psi_coarse) (zero if null).
// One thread per face; batch b uses psi + b*bs, q + b*qbs, coarse + b*cbs.
__global__ void curl_kernel(double *__restrict__ qout, long long qbs, const double *__restrict__ psi, long long bs,
                            const double *__restrict__ coarse, long long cbs, Grid g) {
    const int nx = g.nx, ny = g.ny;
    const long long nu = (long long)(nx + 1) * ny, nq = nu + (long long)nx * (ny + 1);
    const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int b = blockIdx.y;
    if (f >= nq) return;
    const double *P = psi + b * bs;
    const double *C = coarse ? coarse + b * cbs : nullptr;
    double v;
    if (f < nu) {
        const int i = (int)(f % (nx + 1)) + 1, j = (int)(f / (nx + 1)) + 1;
        if (i == 1)
            v = getbc(C, g, SIDE_L, j + 1) - getbc(C, g, SIDE_L, j);
        else if (i == nx + 1)
            v = getbc(C, g, SIDE_R, j + 1) - getbc(C, g, SIDE_R, j);
        else if (j == 1)
            v = P[GI(i - 1, 1)] - getbc(C, g, SIDE_B, i);
        else if (j == ny)
            v = getbc(C, g, SIDE_T, i) - P[GI(i - 1, ny - 1)];
        else
            v = P[GI(i - 1, j)] - P[GI(i - 1, j - 1)];
    } else {
        const long long k = f - nu;
        const int i = (int)(k % nx) + 1, j = (int)(k / nx) + 1;
        if (j == 1)
            v = getbc(C, g, SIDE_B, i) - getbc(C, g, SIDE_B, i + 1);
        else if (j == ny + 1)
            v = getbc(C, g, SIDE_T, i) - getbc(C, g, SIDE_T, i + 1);
        else if (i == 1)
            v = getbc(C, g, SIDE_L, j) - P[GI(1, j - 1)];
        else if (i == nx)
            v = P[GI(nx - 1, j - 1)] - getbc(C, g, SIDE_R, j);
        else
            v = P[GI(i - 1, j - 1)] - P[GI(i, j - 1)];
    }
    qout[b * qbs + f] = v;
}

// coarsify! (src/fluid.jl:208-228): fine level -> central block of the next coarser level.
__global__ void coarsify_kernel(double *__restrict__ coarse, const double *__restrict__ fine, long long bs, Grid g) {
    const int nx = g.nx, ny = g.ny;
    const int ni = (nx / 2 - 2 - (-nx / 2 + 2)) / 2 + 1, nic = (nx / 4 - 1) - (-nx / 4 + 1) + 1;
    const int nj = (ny / 2 - 2 - (-ny / 2 + 2)) / 2 + 1, njc = (ny / 4 - 1) - (-ny / 4 + 1) + 1;
    const int ci = ni < nic ? ni : nic, cj = nj < njc ? nj : njc;
    const int a = blockIdx.x * blockDim.x + threadIdx.x, bb = blockIdx.y * blockDim.y + threadIdx.y;
    if (a >= ci || bb >= cj) return;
    const double *G = fine + blockIdx.z * bs;
    double *Gc = coarse + blockIdx.z * bs;
    const int i = nx / 2 + (-nx / 2 + 2) + 2 * a, ic = nx / 2 + (-nx / 4 + 1) + a;
    const int j = ny / 2 + (-ny / 2 + 2) + 2 * bb, jc = ny / 2 + (-ny / 4 + 1) + bb;
    Gc[GI(ic, jc)] = G[GI(i, j)] + 0.5 * (G[GI(i + 1, j)] + G[GI(i, j + 1)] + G[GI(i - 1, j)] + G[GI(i, j - 1)]) +
                     0.25 * (G[GI(i + 1, j + 1)] + G[GI(i + 1, j - 1)] + G[GI(i - 1, j - 1)] + G[GI(i - 1, j + 1)]);
}

// ---------------------------------------------------------------------------
// Coupling kernels (src/coupling.jl)
// ---------------------------------------------------------------------------

// Yang3 smoothed delta times h (src/coupling.jl:91-148), the published
// polynomial of Yang et al., JCP 2009, with the reference's constants.
__device__ __forceinline__ double delta_h(double rf, double rb, double dr) {
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

struct Panels {
    int np;
    double *xb;        // np x 2 (current positions)
    double *ub;        // np x 2
    int *pc;           // np x 2 panel_coords (ix, iy)
    double *w;         // np x 2 x 49, [(p*2+c)*49 + bb*7 + a]
    int *bbox;         // i0, i1, j0, j1 of the support union (face indices)
    int *err;          // err[0]: 0 or 1-based panel index outside the region
};

// _update!(reg, index, point) (src/coupling.jl:27-54) for panels [p0, p1).
// One block of 49 x 2 threads per panel.
__global__ void reg_weights_kernel(Panels P, int p0, Grid g) {
    const int p = p0 + blockIdx.x;
    const int a = threadIdx.x % 7, bb = threadIdx.x / 7, c = threadIdx.y;
    const double h = g.h, x0 = g.x0, y0 = g.y0;
    const double xb = P.xb[p], yb = P.xb[P.np + p];
    const int ix = (int)rint((xb - x0) / h + 1.0 - 0.25);
    const int iy = (int)rint((yb - y0) / h + 1.0 - 0.25);
    const bool ok = (3 < ix && ix <= g.nx - 3) && (3 < iy && iy <= g.ny - 3);
    if (!ok) {
        if (threadIdx.x == 0 && threadIdx.y == 0) atomicCAS(P.err, 0, p + 1);
        return;
    }
    if (threadIdx.x == 0 && c == 0) {
        P.pc[2 * p] = ix;
        P.pc[2 * p + 1] = iy;
    }
    const double x = x0 + h * ((ix + (a - 3)) - 1);
    const double y = y0 + h * ((iy + (bb - 3)) - 1);
    double wv;
    if (c == 0)
        wv = delta_h(x, xb, h) * delta_h(y + h / 2, yb, h);
    else
        wv = delta_h(x + h / 2, xb, h) * delta_h(y, yb, h);
    P.w[(long long)(p * 2 + c) * 49 + bb * 7 + a] = wv;
}

// Union of the panels' 7x7 supports (one block).
__global__ void bbox_kernel(Panels P, Grid g) {
    __shared__ int s[4][32];
    int i0 = 1 << 30, i1 = -(1 << 30), j0 = 1 << 30, j1 = -(1 << 30);
    for (int p = threadIdx.x; p < P.np; p += blockDim.x) {
        const int ix = P.pc[2 * p], iy = P.pc[2 * p + 1];
        i0 = min(i0, ix - 3);
        i1 = max(i1, ix + 3);
        j0 = min(j0, iy - 3);
        j1 = max(j1, iy + 3);
    }
    for (int o = 16; o > 0; o >>= 1) {
        i0 = min(i0, __shfl_xor_sync(0xffffffffu, i0, o));
        i1 = max(i1, __shfl_xor_sync(0xffffffffu, i1, o));
        j0 = min(j0, __shfl_xor_sync(0xffffffffu, j0, o));
        j1 = max(j1, __shfl_xor_sync(0xffffffffu, j1, o));
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        s[0][w] = i0;
        s[1][w] = i1;
        s[2][w] = j0;
        s[3][w] = j1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) {
            i0 = min(i0, s[0][k]);
            i1 = max(i1, s[1][k]);
            j0 = min(j0, s[2][k]);
            j1 = max(j1, s[3][k]);
        }
        P.bbox[0] = max(i0, 1);
        P.bbox[1] = i1;
        P.bbox[2] = max(j0, 1);
        P.bbox[3] = j1;
    }
}

// reg! (src/coupling.jl:72-85) as a deterministic gather over a 16x16 tile of
// faces: the block lists, in panel order, the panels whose support meets the
// tile, then every face sums w * f over that list in panel order -- the same
// accumulation order as the reference's sequential loop over panels.
// f: 2np per batch (x block then y block); patch output per batch.
constexpr int kTile = 16;
__global__ void __launch_bounds__(256) reg_patch_kernel(Panels P, const double *__restrict__ f, long long fbs,
                                                        double *__restrict__ patch, long long pbs) {
    __shared__ int list[1024];
    __shared__ int warp_cnt[8];
    __shared__ int total;
    const int i0 = P.bbox[0], i1 = P.bbox[1], j0 = P.bbox[2], j1 = P.bbox[3];
    const int pw = i1 - i0 + 1, ph = j1 - j0 + 1;
    const int ti0 = i0 + blockIdx.x * kTile, tj0 = j0 + blockIdx.y * kTile;
    if (ti0 > i1 || tj0 > j1) return;
    const int ti1 = min(ti0 + kTile - 1, i1), tj1 = min(tj0 + kTile - 1, j1);
    const int b = blockIdx.z;
    const double *fb = f + b * fbs;
    double *out = patch + b * pbs;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int li = tid % kTile, lj = tid / kTile;
    const int i = ti0 + li, j = tj0 + lj;
    double accx = 0.0, accy = 0.0;
    int base = 0;
    for (int c0 = 0; c0 < P.np; c0 += 256) {
        if (tid == 0) total = 0;
        const int p = c0 + tid;
        bool hit = false;
        if (p < P.np) {
            const int ix = P.pc[2 * p], iy = P.pc[2 * p + 1];
            hit = ix + 3 >= ti0 && ix - 3 <= ti1 && iy + 3 >= tj0 && iy - 3 <= tj1;
        }
        const unsigned m = __ballot_sync(0xffffffffu, hit);
        if (lane == 0) warp_cnt[w] = __popc(m);
        __syncthreads();
        int off = 0;
        for (int k = 0; k < w; ++k) off += warp_cnt[k];
        if (hit) list[off + __popc(m & ((1u << lane) - 1))] = p;
        if (tid == 255) {
            int s = 0;
            for (int k = 0; k < 8; ++k) s += warp_cnt[k];
            total = s;
        }
        __syncthreads();
        (void)base;
        const int n = total;
        if (i <= ti1 && j <= tj1) {
            for (int k = 0; k < n; ++k) {
                const int q = list[k];
                const int ix = P.pc[2 * q], iy = P.pc[2 * q + 1];
                const int da = i - ix + 3, db = j - iy + 3;
                if (da >= 0 && da < 7 && db >= 0 && db < 7) {
                    accx = accx + P.w[(long long)(q * 2) * 49 + db * 7 + da] * fb[q];
                    accy = accy + P.w[(long long)(q * 2 + 1) * 49 + db * 7 + da] * fb[P.np + q];
                }
            }
        }
        __syncthreads();
    }
    if (i <= ti1 && j <= tj1) {
        out[(i - i0) + (long long)pw * (j - j0)] = accx;
        out[(long long)pw * ph + (i - i0) + (long long)pw * (j - j0)] = accy;
    }
}

// regT! (src/coupling.jl:57-69): fb[p, c] = dot(q_c[7x7 at p], w[p, c]) in
// column-major order.  With add_q0 it is couple_surface_rigid's
// Ftmp = E (qs + q0) - ub h (src/coupling.jl:239-244).
__global__ void regT_kernel(Panels P, const double *__restrict__ q, long long qbs, double *__restrict__ out,
                            long long obs, int nbatch, int add_q0, const StepDev *__restrict__ prm, Grid g) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int np = P.np;
    if (t >= 2 * np * nbatch) return;
    const int b = t / (2 * np), pcomp = t % (2 * np);
    const int c = pcomp / np, p = pcomp % np;
    const long long nu = (long long)(g.nx + 1) * g.ny;
    const double *Q = q + b * qbs;
    const int i0 = P.pc[2 * p] - 3, j0 = P.pc[2 * p + 1] - 3;
    const double *w = P.w + (long long)(p * 2 + c) * 49;
    double s = 0.0;
    for (int bb = 0; bb < 7; ++bb)
        for (int a = 0; a < 7; ++a) {
            const int i = i0 + a, j = j0 + bb;
            double v = c == 0 ? Q[UI(i, j)] : Q[VI(i, j)];
            if (add_q0) v = v + (c == 0 ? base_flux_x(g, prm, 1, i, j) : base_flux_y(g, prm, 1, i, j));
            s += v * w[bb * 7 + a];
        }
    if (add_q0) s = s - P.ub[c * np + p] * g.h;
    out[b * obs + c * np + p] = s;
}

// x = Binv z for the precomputed B^-1 (src/coupling.jl:187-192), column-major n x n.
// Grid (ceil(n/64), ceil(n/64)); partial sums part[chunk * n + row], summed in
// chunk order by binv_reduce_kernel (deterministic).
__global__ void __launch_bounds__(256) binv_gemv_kernel(const double *__restrict__ A, const double *__restrict__ z,
                                                        double *__restrict__ part, int n) {
    __shared__ double red[4][64];
    const int r = threadIdx.x % 64, s = threadIdx.x / 64;
    const int row = blockIdx.x * 64 + r;
    const int cbeg = blockIdx.y * 64;
    double acc = 0.0;
    if (row < n) {
        for (int c = cbeg + s; c < min(cbeg + 64, n); c += 4) acc += A[row + (long long)n * c] * __ldg(&z[c]);
    }
    red[s][r] = acc;
    __syncthreads();
    if (s == 0 && row < n) part[(long long)blockIdx.y * n + row] = ((red[0][r] + red[1][r]) + red[2][r]) + red[3][r];
}

// F~b = sum of the chunk partials; update_vars! fb = F~b h / dt (problem.jl:676-685);
// total force sum over panels (problem.jl:853-856).  One block.
__global__ void binv_reduce_kernel(const double *__restrict__ part, int nchunk, int n, double *__restrict__ fbt,
                                   double *__restrict__ fb, double *__restrict__ total, double h, double dt,
                                   int from_part) {
    __shared__ double sx[32], sy[32];
    const int np = n / 2;
    double tx = 0.0, ty = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        double v;
        if (from_part) {
            v = 0.0;
            for (int c = 0; c < nchunk; ++c) v += part[(long long)c * n + k];
            fbt[k] = v;
        } else {
            v = fbt[k];
        }
        const double f = v * h / dt;
        fb[k] = f;
        if (k < np)
            tx += f;
        else
            ty += f;
    }
    for (int o = 16; o > 0; o >>= 1) {
        tx += __shfl_xor_sync(0xffffffffu, tx, o);
        ty += __shfl_xor_sync(0xffffffffu, ty, o);
    }
    if ((threadIdx.x & 31) == 0) {
        sx[threadIdx.x >> 5] = tx;
        sy[threadIdx.x >> 5] = ty;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ax = 0.0, ay = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            ax += sx[k];
            ay += sy[k];
        }
        total[0] = ax;
        total[1] = ay;
    }
}

// _update!(panels, ::MovingRigidBody, t) (src/bodies.jl:12-31) for panels [p0, p1)
// with motion m = pos(2), vel(2), angle, angular_vel.
__global__ void rigid_motion_kernel(Panels P, const double *__restrict__ ref_xb, const double *__restrict__ motion,
                                    int p0, int p1) {
    const int p = p0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= p1) return;
    const double r0x = motion[0], r0y = motion[1], v0x = motion[2], v0y = motion[3], ang = motion[4], Om = motion[5];
    double sn, c;
    sincos(ang, &sn, &c);
    const double rx = ref_xb[p], ry = ref_xb[P.np + p];
    P.xb[p] = r0x + (c * rx + -sn * ry);
    P.xb[P.np + p] = r0y + (sn * rx + c * ry);
    P.ub[p] = v0x + ((Om * -sn) * rx + (Om * -c) * ry);
    P.ub[P.np + p] = v0y + ((Om * c) * rx + (Om * -sn) * ry);
}

// In-place Gauss-Jordan inversion of a symmetric positive definite matrix
// (stands in for LinearAlgebra.inv at src/coupling.jl:190).  Step k, part 1:
// save the pivot row/column.
__global__ void gj_save_kernel(const double *__restrict__ A, int n, int k, double *__restrict__ rowk,
                               double *__restrict__ colk, int *err) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const double p = A[k + (long long)n * k];
    if (t == 0 && !(p > 0.0)) atomicCAS(err, 0, k + 1);
    rowk[t] = A[k + (long long)n * t] / p;
    colk[t] = A[t + (long long)n * k];
}
// part 2: rank-1 update of every element
__global__ void gj_update_kernel(double *__restrict__ A, int n, int k, const double *__restrict__ rowk,
                                 const double *__restrict__ colk) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= n) return;
    const double p = colk[k];
    double v;
    if (i == k && j == k)
        v = 1.0 / p;
    else if (i == k)
        v = rowk[j];
    else if (j == k)
        v = -colk[i] / p;
    else
        v = A[i + (long long)n * j] - colk[i] * rowk[j];
    A[i + (long long)n * j] = v;
}

// Identity columns [c0, c0+nb) of a 2np-length basis, one per batch.
__global__ void unit_columns_kernel(double *__restrict__ f, int n, int c0, int nb) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * nb) return;
    const int b = t / n, k = t % n;
    f[t] = (k == c0 + b) ? 1.0 : 0.0;
}

}  // namespace ibpm
