// coupling.cu -- the regularised-delta coupling kernels (src/coupling.jl,
// src/bodies.jl), compiled with -fmad=false.
//
// The reference evaluates the grid coordinates x0 + h (i - 1), the Yang3
// polynomial and the E / E^T sums without fused multiply-adds.  The Yang3 delta
// is discontinuous at r = 3h by ~1e-9 (its published constants carry 10
// digits), and panels lying exactly 3h from a grid line fall on one side of
// that branch or the other depending on the rounding of x0 + h (i - 1); an
// FMA-contracted coordinate changes the weights by ~1e-9.  This file is
// therefore compiled without contraction so every rounding matches the
// reference's.
#include "coupling.h"

namespace ibpm {


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
// f: 2np per batch (x block then y block); patch output per batch; (bx, by): the
// tile's place in the bounding box.
template <class T>
__device__ __forceinline__ void reg_patch_tile(const Panels &P, const double *__restrict__ fb, T *__restrict__ out,
                                               int bx, int by) {
    __shared__ int list[1024];
    __shared__ int warp_cnt[8];
    __shared__ int total;
    const int i0 = P.bbox[0], i1 = P.bbox[1], j0 = P.bbox[2], j1 = P.bbox[3];
    const int pw = i1 - i0 + 1, ph = j1 - j0 + 1;
    const int ti0 = i0 + bx * kTile, tj0 = j0 + by * kTile;
    if (ti0 > i1 || tj0 > j1) return;
    const int ti1 = min(ti0 + kTile - 1, i1), tj1 = min(tj0 + kTile - 1, j1);
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
        out[(i - i0) + (long long)pw * (j - j0)] = (T)accx;
        out[(long long)pw * ph + (i - i0) + (long long)pw * (j - j0)] = (T)accy;
    }
}

template <class T>
__global__ void __launch_bounds__(256) reg_patch_kernel(Panels P, const double *__restrict__ f, long long fbs,
                                                        T *__restrict__ patch, long long pbs) {
    const int b = blockIdx.z;
    // the blocks walk the tiles of the bounding box (its size is known on the device only)
    const int pw = P.bbox[1] - P.bbox[0] + 1, ph = P.bbox[3] - P.bbox[2] + 1;
    for (int by = blockIdx.y; by * kTile < ph; by += gridDim.y)
        for (int bx = blockIdx.x; bx * kTile < pw; bx += gridDim.x) reg_patch_tile<T>(P, f + b * fbs, patch + b * pbs, bx, by);
}

// reg_patch_kernel for the cases of a batched ensemble group (case = blockIdx.z):
// each case's E^T F~b onto its own patch.
template <class T>
__global__ void __launch_bounds__(256) reg_patch_multi_kernel(const CaseView *__restrict__ tab) {
    const CaseView &cv = tab[blockIdx.z];
    const int pw = cv.P.bbox[1] - cv.P.bbox[0] + 1, ph = cv.P.bbox[3] - cv.P.bbox[2] + 1;
    for (int by = blockIdx.y; by * kTile < ph; by += gridDim.y)
        for (int bx = blockIdx.x; bx * kTile < pw; bx += gridDim.x)
            reg_patch_tile<T>(cv.P, cv.Fbt, static_cast<T *>(cv.patch), bx, by);
}

// regT! (src/coupling.jl:57-69): fb[p, c] = dot(q_c[7x7 at p], w[p, c]) in
// column-major order.  With add_q0 it is couple_surface_rigid's
// Ftmp = E (qs + q0) - ub h (src/coupling.jl:239-244).
// One warp per output: the lanes form the 49 products w q of the support in
// parallel; lane 0 adds them in the reference's order (column-major over the
// support, from 0), so the sum rounds as a sequential dot product.
constexpr int kRegTWarps = 4;
template <class T>
__device__ __forceinline__ void regT_warp(const Panels &P, const T *__restrict__ Q, double *__restrict__ outb,
                                          int pcomp, int add_q0, const StepDev *__restrict__ prm, const Grid &g,
                                          double (*prod)[49]) {
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int np = P.np;
    const int c = pcomp / np, p = pcomp % np;
    const long long nu = (long long)(g.nx + 1) * g.ny;
    const int i0 = P.pc[2 * p] - 3, j0 = P.pc[2 * p + 1] - 3;
    const double *w = P.w + (long long)(p * 2 + c) * 49;
    for (int k = lane; k < 49; k += 32) {
        const int bb = k / 7, a = k % 7;
        const int i = i0 + a, j = j0 + bb;
        double v = c == 0 ? (double)Q[UI(i, j)] : (double)Q[VI(i, j)];
        if (add_q0) v = v + (c == 0 ? base_flux_x(g, prm, 1, i, j) : base_flux_y(g, prm, 1, i, j));
        prod[wid][k] = v * w[k];
    }
    __syncwarp();
    if (lane == 0) {
        double s = 0.0;
        for (int k = 0; k < 49; ++k) s += prod[wid][k];
        if (add_q0) s = s - P.ub[c * np + p] * g.h;
        outb[c * np + p] = s;
    }
}

template <class T>
__global__ void __launch_bounds__(32 * kRegTWarps) regT_kernel(Panels P, const T *__restrict__ q, long long qbs,
                                                                double *__restrict__ out, long long obs, int nbatch,
                                                                int add_q0, const StepDev *__restrict__ prm, Grid g) {
    __shared__ double prod[kRegTWarps][49];
    const int t = blockIdx.x * kRegTWarps + (threadIdx.x >> 5);
    const int np = P.np;
    if (t >= 2 * np * nbatch) return;  // the whole warp leaves together
    const int b = t / (2 * np), pcomp = t % (2 * np);
    regT_warp<T>(P, q + b * qbs, out + b * obs, pcomp, add_q0, prm, g, prod);
}

// couple_surface_rigid's Ftmp = E (qs + q0) - ub h for the cases of a batched
// ensemble group (case = blockIdx.y; flux stride qbs; callback values prm[case]).
template <class T>
__global__ void __launch_bounds__(32 * kRegTWarps) regT_multi_kernel(const CaseView *__restrict__ tab,
                                                                      const T *__restrict__ q, long long qbs,
                                                                      const StepDev *__restrict__ prm, Grid g) {
    __shared__ double prod[kRegTWarps][49];
    const int cs = blockIdx.y;
    const CaseView &cv = tab[cs];
    const int t = blockIdx.x * kRegTWarps + (threadIdx.x >> 5);
    if (t >= 2 * cv.P.np) return;  // the whole warp leaves together
    regT_warp<T>(cv.P, q + cs * qbs, cv.Ftmp, t, 1, prm + cs, g, prod);
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


// ---- launchers ----
void launch_reg_weights(const Panels &P, int p0, int p1, const Grid &g, cudaStream_t st) {
    if (p1 > p0) reg_weights_kernel<<<p1 - p0, dim3(49, 2), 0, st>>>(P, p0, g);
}
void launch_bbox(const Panels &P, const Grid &g, cudaStream_t st) { bbox_kernel<<<1, 256, 0, st>>>(P, g); }
// Blocks per dimension for the patch kernels: with many batches, enough for a
// bounding box of 128 faces in one sweep (a larger box takes more sweeps); with
// a few, the tiles of the whole grid, each block at most one tile.
static int patch_grid(int n, int nbatch) {
    const int whole = (n + 1 + kTile - 1) / kTile + 1;
    return nbatch > 4 && whole > 8 ? 8 : whole;
}

template <class T>
void launch_reg_patch(const Panels &P, const double *f, long long fbs, T *patch, long long pbs, int nbatch,
                      const Grid &g, cudaStream_t st) {
    reg_patch_kernel<T><<<dim3(patch_grid(g.nx, nbatch), patch_grid(g.ny, nbatch), nbatch), 256, 0, st>>>(P, f, fbs, patch, pbs);
}
template <class T>
void launch_regT(const Panels &P, const T *q, long long qbs, double *out, long long obs, int nbatch, int add_q0,
                 const StepDev *prm, const Grid &g, cudaStream_t st) {
    const int nt = 2 * P.np * nbatch;
    regT_kernel<T><<<(nt + kRegTWarps - 1) / kRegTWarps, 32 * kRegTWarps, 0, st>>>(P, q, qbs, out, obs, nbatch,
                                                                                  add_q0, prm, g);
}
template <class T>
void launch_reg_patch_multi(const CaseView *tab, int ncase, const Grid &g, cudaStream_t st) {
    reg_patch_multi_kernel<T><<<dim3(patch_grid(g.nx, ncase), patch_grid(g.ny, ncase), ncase), 256, 0, st>>>(tab);
}
template <class T>
void launch_regT_multi(const CaseView *tab, int ncase, int np_max, const T *q, long long qbs, const StepDev *prm,
                       const Grid &g, cudaStream_t st) {
    regT_multi_kernel<T><<<dim3((2 * np_max + kRegTWarps - 1) / kRegTWarps, ncase), 32 * kRegTWarps, 0, st>>>(
        tab, q, qbs, prm, g);
}
template void launch_reg_patch_multi<double>(const CaseView *, int, const Grid &, cudaStream_t);
template void launch_reg_patch_multi<float>(const CaseView *, int, const Grid &, cudaStream_t);
template void launch_regT_multi<double>(const CaseView *, int, int, const double *, long long, const StepDev *,
                                        const Grid &, cudaStream_t);
template void launch_regT_multi<float>(const CaseView *, int, int, const float *, long long, const StepDev *,
                                       const Grid &, cudaStream_t);
template void launch_reg_patch<double>(const Panels &, const double *, long long, double *, long long, int,
                                       const Grid &, cudaStream_t);
template void launch_reg_patch<float>(const Panels &, const double *, long long, float *, long long, int,
                                      const Grid &, cudaStream_t);
template void launch_regT<double>(const Panels &, const double *, long long, double *, long long, int, int,
                                  const StepDev *, const Grid &, cudaStream_t);
template void launch_regT<float>(const Panels &, const float *, long long, double *, long long, int, int,
                                 const StepDev *, const Grid &, cudaStream_t);
void launch_rigid_motion(const Panels &P, const double *ref_xb, const double *motion, int p0, int p1,
                         cudaStream_t st) {
    if (p1 > p0) rigid_motion_kernel<<<(p1 - p0 + 127) / 128, 128, 0, st>>>(P, ref_xb, motion, p0, p1);
}

}  // namespace ibpm
