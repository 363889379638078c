// common.cuh -- types and device helpers shared by the IBPM kernels.
//
// Index helpers use the reference's 1-based (i, j) so each kernel reads like
// the loop it restates.  Layouts (column-major, x fastest):
//   Gamma-like field  (nx-1) x (ny-1):  GI(i,j) = (i-1) + (nx-1)(j-1)
//   x flux  (nx+1) x ny:                UI(i,j) = (i-1) + (nx+1)(j-1)
//   y flux  nx x (ny+1):                VI(i,j) = nu + (i-1) + nx(j-1)
// A "batch" index b selects a field: either the level (b = lev-1, the trial
// solves) or an independent right-hand side (the B^-1 setup columns).
//
// Fields have element type T: double for the plain FP64 path, float for the
// mixed-precision path.  Boundary values, base fluxes and coupling sums are
// always accumulated in double.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ibpm {

// complex type of a real type
template <class T>
struct Cx;
template <>
struct Cx<double> {
    using type = double2;
    static __host__ __device__ __forceinline__ double2 make(double a, double b) { return make_double2(a, b); }
};
template <>
struct Cx<float> {
    using type = float2;
    static __host__ __device__ __forceinline__ float2 make(float a, float b) { return make_float2(a, b); }
};

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
template <class T>
__device__ __forceinline__ double getbc(const T *__restrict__ r, const Grid &g, int side, int ibc) {
    if (r == nullptr) return 0.0;
    const int nx = g.nx, ny = g.ny;
    if (side == SIDE_B || side == SIDE_T) {
        const int row = side == SIDE_B ? ny / 4 : 3 * ny / 4;
        if (ibc & 1) return (double)r[GI(nx / 4 + (ibc - 1) / 2, row)];
        const int i = nx / 4 + ibc / 2;
        return 0.5 * ((double)r[GI(i, row)] + (double)r[GI(i - 1, row)]);
    }
    const int col = side == SIDE_L ? nx / 4 : 3 * nx / 4;
    if (ibc & 1) return (double)r[GI(col, ny / 4 + (ibc - 1) / 2)];
    const int j = ny / 4 + ibc / 2;
    return 0.5 * ((double)r[GI(col, j)] + (double)r[GI(col, j - 1)]);
}

// apply_bc! contribution at (i, j) (src/fluid.jl:308-338), accumulated in the
// reference's order (bottom/top rows first, then left/right columns).
template <class T>
__device__ __forceinline__ double apply_bc_at(double v, const T *__restrict__ r, const Grid &g, int i, int j,
                                              double fac) {
    if (j == 1) v += fac * getbc(r, g, SIDE_B, i + 1);
    if (j == g.ny - 1) v += fac * getbc(r, g, SIDE_T, i + 1);
    if (i == 1) v += fac * getbc(r, g, SIDE_L, j + 1);
    if (i == g.nx - 1) v += fac * getbc(r, g, SIDE_R, j + 1);
    return v;
}

// One element global -> shared memory without passing through registers
// (cp.async, 4 or 8 bytes; both addresses naturally aligned).  Completed by
// cp_async_wait_all() in the issuing thread, then a barrier for the block.
template <class T>
__device__ __forceinline__ void cp_async_elem(T *sdst, const T *gsrc) {
    static_assert(sizeof(T) == 4 || sizeof(T) == 8, "4- or 8-byte elements");
    const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
    if constexpr (sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

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

struct Panels {
    int np;
    double *xb;        // np x 2 (current positions)
    double *ub;        // np x 2
    int *pc;           // np x 2 panel_coords (ix, iy)
    double *w;         // np x 2 x 49, [(p*2+c)*49 + bb*7 + a]
    int *bbox;         // i0, i1, j0, j1 of the support union (face indices)
    int *err;          // err[0]: 0 or 1-based panel index outside the region
};

// One case of a batched ensemble group, as the multi-case coupling kernels see
// it: its panels and the buffers of its force solve and regularisation patch.
struct CaseView {
    Panels P;
    double *Ftmp, *part, *Fbt, *fb, *total;
    const double *Binv;
    void *patch;  // element type of the group's fields
    long long patch_stride;
};

// Regularised flux on the panels' bounding box (compact patch):
// patch[(i - i0) + pw (j - j0)] for x faces, offset pw*ph for y faces.
template <class T>
struct Patch {
    const T *p;
    const int *bbox;      // device: i0, i1, j0, j1 (1-based face indices)
    long long bs;
    __device__ __forceinline__ double get(int b, int comp, int i, int j) const {
        const int i0 = bbox[0], i1 = bbox[1], j0 = bbox[2], j1 = bbox[3];
        if (i < i0 || i > i1 || j < j0 || j > j1) return 0.0;
        const int pw = i1 - i0 + 1, ph = j1 - j0 + 1;
        return (double)p[b * bs + (long long)comp * pw * ph + (i - i0) + (long long)pw * (j - j0)];
    }
};

}  // namespace ibpm
