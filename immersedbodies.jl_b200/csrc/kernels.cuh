// kernels.cuh -- device kernels of the IBPM time step (line passes, stencils,
// B^-1 algebra).  Field element type T is double (plain FP64 path) or float
// (mixed-precision path); arithmetic on boundary values, multipliers and
// coupling sums is done in double.  Included by ibpm.cu only.
#pragma once
#include <type_traits>
#include "common.cuh"
#include "fft_pow2.cuh"

namespace ibpm {

// ---------------------------------------------------------------------------
// Line-pass kernels
// ---------------------------------------------------------------------------

// Shared-memory layout of a pass kernel: nbuf line buffers of D::C, then the
// double2 scan scratch at a 16-byte boundary.
template <class D>
__host__ __device__ constexpr size_t scratch_offset(int M, int nbuf) {
    return ((size_t)nbuf * D::smem_len(M) * sizeof(typename D::C) + 15) / 16 * 16;
}
template <class D>
__host__ __device__ constexpr size_t pass_smem(int M, int nbuf, int ngroups) {
    return scratch_offset<D>(M, nbuf) + (size_t)D::NWARP * ngroups * sizeof(double2);
}

// Prologue: plain field
template <class T>
struct InPlain {
    const T *p;
    long long bs;
    int ld;
    __device__ __forceinline__ double operator()(int b, int i, int j) const {
        return (double)p[b * bs + (long long)(i - 1) + (long long)ld * (j - 1)];
    }
};

// Prologue of vort2flux's telescoping solve (src/fluid.jl:194-197):
// Gamma_tmp = Gamma[:, lev]; apply_bc!(Gamma_tmp, get_bc(psi[:, lev+1]); fac=1)
// (the coarser level's psi may be of another element type TC)
template <class T, class TC = T>
struct InBC {
    const T *gam;
    const TC *coarse;
    long long bs, cbs;
    Grid g;
    __device__ __forceinline__ double operator()(int b, int i, int j) const {
        const T *G = gam + b * bs;
        double v = (double)G[GI(i, j)];
        if (on_ring(g, i, j)) v = apply_bc_at(v, coarse + b * cbs, g, i, j, 1.0);
        return v;
    }
    // The compile-time X pass loads the field alone (plain()) and then adds the
    // boundary values to the ring elements (ring()), so the loads of a line are
    // not held up behind the boundary reads; the sum is the one operator() forms.
    static constexpr bool kSplitRing = true;
    __device__ __forceinline__ double plain(int b, int i, int j) const { return (double)gam[b * bs + GI(i, j)]; }
    __device__ __forceinline__ bool ring_row(int j) const { return j == 1 || j == g.ny - 1; }
    __device__ __forceinline__ double ring(double v, int b, int i, int j) const {
        return apply_bc_at(v, coarse + b * cbs, g, i, j, 1.0);
    }
};

// detects the split prologue of InBC
template <class In, class = void>
struct SplitRing {
    static constexpr bool value = false;
};
template <class In>
struct SplitRing<In, std::void_t<decltype(In::kSplitRing)>> {
    static constexpr bool value = In::kSplitRing;
};

// A prologue over a field that is zero outside the block i0..i1 x j0..j1: there
// the field reads as zero without a load (the boundary values on the ring are
// still added).  The coarse levels of a B application are such fields: their
// vorticity is the finer level's coarsified into the central block
// (coarsify!, src/fluid.jl:208-228), and zero elsewhere.
template <class In>
struct InCentral {
    In in;
    int i0, i1, j0, j1;
    static constexpr bool kSplitRing = SplitRing<In>::value;
    __device__ __forceinline__ bool inside(int i, int j) const { return i >= i0 && i <= i1 && j >= j0 && j <= j1; }
    __device__ __forceinline__ double operator()(int b, int i, int j) const {
        if constexpr (kSplitRing)
            return inside(i, j) ? in(b, i, j) : in.ring(0.0, b, i, j);
        else
            return inside(i, j) ? in(b, i, j) : 0.0;
    }
    __device__ __forceinline__ double plain(int b, int i, int j) const { return inside(i, j) ? in.plain(b, i, j) : 0.0; }
    __device__ __forceinline__ bool ring_row(int j) const { return in.ring_row(j); }
    __device__ __forceinline__ double ring(double v, int b, int i, int j) const { return in.ring(v, b, i, j); }
};

// Prologue rot!(Gamma, reg!(q, f)) (src/fluid.jl:101-111 after src/coupling.jl:72-85),
// evaluated from the regularised patch.
template <class T>
struct InRegRot {
    Patch<T> pt;
    __device__ __forceinline__ double operator()(int b, int I, int J) const {
        return (pt.get(b, 0, I + 1, J) - pt.get(b, 0, I + 1, J + 1)) + (pt.get(b, 1, I + 1, J + 1) - pt.get(b, 1, I, J + 1));
    }
};

// Prologue rot!(Gamma, reg!(q, f)) of the cases of a batched ensemble group:
// batch b reads case b's patch (zero outside its bounding box).
template <class T>
struct InRegRotTab {
    const CaseView *tab;
    __device__ __forceinline__ double operator()(int b, int I, int J) const {
        const CaseView &cv = tab[b];
        const Patch<T> pt{static_cast<const T *>(cv.patch), cv.P.bbox, 0};
        return (pt.get(0, 0, I + 1, J) - pt.get(0, 0, I + 1, J + 1)) + (pt.get(0, 1, I + 1, J + 1) - pt.get(0, 1, I, J + 1));
    }
};

// Epilogue: plain store
template <class T>
struct OutPlain {
    T *p;
    long long bs;
    int ld;
    __device__ __forceinline__ void operator()(int b, int i, int j, double v) const {
        p[b * bs + (long long)(i - 1) + (long long)ld * (j - 1)] = (T)v;
    }
};

// Epilogue of project_circ (src/coupling.jl:227): Gamma[:, 1] .-= x
template <class T>
struct OutSub {
    T *p;
    long long bs;
    int ld;
    __device__ __forceinline__ void operator()(int b, int i, int j, double v) const {
        T *q = p + b * bs + (long long)(i - 1) + (long long)ld * (j - 1);
        *q = (T)((double)*q - v);
    }
};

// 1/d: the hardware reciprocal approximation refined by two Newton-Raphson
// steps (e = 1 - d y, y += y e); within an ulp or two of the correctly rounded
// quotient, for the positive, normal d of the spectral multipliers.
__device__ __forceinline__ double recip(double d) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(d));
    double e = fma(-d, y, 1.0);
    y = fma(y, e, y);
    e = fma(-d, y, 1.0);
    return fma(y, e, y);
}

// Spectral multipliers scale / Lambda (src/fluid.jl:117-134)
enum { MULT_LAPINV = 0, MULT_AEXPL = 1, MULT_AIMPL = 2 };
struct Mult {
    int mode;
    const double *cx;   // cos(pi i / nx), i = 0..nx
    const double *cy;   // cos(pi j / ny), j = 0..ny
    double scale;       // 1 / (4 nx ny)
    double h, Re, dt;
    int lev0, levstep;  // level of batch b: lev0 + b * levstep
    const double *coef_tab;  // device, may be null: c of batch b (cases of an ensemble differ in Re)
    // c = dt / (2 Re hc^2) of the batch's level; the reference's (lam dt) / (2 Re hc^2)
    // becomes lam c (within one rounding), which leaves one division per element.
    __device__ __forceinline__ double coef(int b) const {
        if (coef_tab) return coef_tab[b];
        const int lev = lev0 + b * levstep;
        const double hc = ldexp(h, lev - 1);
        return dt / (2 * Re * (hc * hc));
    }
    __device__ __forceinline__ double eval(double c, double cxi, double cyj) const {
        const double lam = -2 * ((cxi + cyj) - 2);
        if (mode == MULT_LAPINV) return scale * recip(lam);
        if (mode == MULT_AEXPL) return scale * (1 - lam * c);  // scale / (1 / (1 - lam c))
        return scale * recip(1 + lam * c);
    }
    __device__ __forceinline__ double operator()(double c, int i, int j) const {
        return eval(c, __ldg(&cx[i]), __ldg(&cy[j]));
    }
};

// X pass: DST along x of rows (ja, jb) = (2p+1, 2p+2) of each batch field.
// D is the line transform (Pow2Dst<M> or GenericDst); NG line pairs per block.
// rows (device, may be null): the body's face window i0, i1, j0, j1 (batch b's
// at rows + b rows_stride).  A block
// none of whose rows lies in j0-1 .. j1 returns at once: with zero_outside = 0
// its output rows stay unwritten (the rows a curl of those faces reads lie
// inside), with zero_outside = 1 it writes them as zeros (the transform of the
// input's zero rows: rot of a patch inside the window is zero outside them).
template <class D, int NG, class In, class Out>
__global__ void __launch_bounds__(D::TPF *NG, D::OCC / (D::TPF * NG))
    xpass_kernel(In in, Out out, PlanT<typename D::Real> pl, int nrows, const int *__restrict__ rows = nullptr,
                 int zero_outside = 0, int rows_stride = 0) {
    if (rows != nullptr) {  // uniform over the block: before any barrier
        rows += (long long)rows_stride * blockIdx.y;
        const int r0 = 2 * NG * (int)blockIdx.x + 1, r1 = r0 + 2 * NG - 1;
        if (r1 < rows[2] - 1 || r0 > rows[3]) {
            if (zero_outside) {
                const int t = threadIdx.x % D::TPF, ja = r0 + 2 * (int)(threadIdx.x / D::TPF);
                for (int jj = ja; jj <= ja + 1 && jj <= nrows; ++jj)
                    for (int i = 1 + t; i < pl.M; i += D::TPF) out((int)blockIdx.y, i, jj, 0.0);
            }
            return;
        }
    }
    using T = typename D::Real;
    using C = typename D::C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *smem = reinterpret_cast<C *>(smem_raw);
    constexpr int TPF = D::TPF;
    const int M = pl.M;
    const int G = D::smem_len(M);
    const int g = threadIdx.x / TPF, t = threadIdx.x % TPF;
    C *buf = smem + g * G;
    double2 *wt = reinterpret_cast<double2 *>(smem_raw + scratch_offset<D>(M, NG)) + D::NWARP * g;
    const int b = blockIdx.y;
    const int pair = blockIdx.x * NG + g;
    const int ja = 2 * pair + 1, jb = 2 * pair + 2;
    const bool va = ja <= nrows, vb = jb <= nrows;
    if constexpr (D::MC > 0) {
        // compile-time trip count: every global load of the thread is in flight
        // before the first shared-memory store
        constexpr int NIT = (D::MC + 1 + TPF - 1) / TPF;
        T za[NIT], zb[NIT];
        if constexpr (SplitRing<In>::value) {
#pragma unroll
            for (int k = 0; k < NIT; ++k) {
                const int i = t + k * TPF;
                const bool in_line = i >= 1 && i < D::MC;
                za[k] = (in_line && va) ? (T)in.plain(b, i, ja) : (T)0;
                zb[k] = (in_line && vb) ? (T)in.plain(b, i, jb) : (T)0;
            }
            // boundary values on the ring: whole rows 1 and ny-1, the ends of the others
            const bool ra = va && in.ring_row(ja), rb = vb && in.ring_row(jb);
#pragma unroll
            for (int k = 0; k < NIT; ++k) {
                const int i = t + k * TPF;
                if (i < 1 || i >= D::MC) continue;
                const bool end = i == 1 || i == D::MC - 1;
                // za[k] holds the field value exactly ((T)(double)x == x), so no reload
                if (va && (ra || end)) za[k] = (T)in.ring((double)za[k], b, i, ja);
                if (vb && (rb || end)) zb[k] = (T)in.ring((double)zb[k], b, i, jb);
            }
        } else {
#pragma unroll
            for (int k = 0; k < NIT; ++k) {
                const int i = t + k * TPF;
                const bool in_line = i >= 1 && i < D::MC;
                za[k] = (in_line && va) ? (T)in(b, i, ja) : (T)0;
                zb[k] = (in_line && vb) ? (T)in(b, i, jb) : (T)0;
            }
        }
#pragma unroll
        for (int k = 0; k < NIT; ++k) {
            const int i = t + k * TPF;
            if (i <= D::MC) buf[D::idx(i)] = Cx<T>::make(za[k], zb[k]);
        }
    } else {
        for (int i = t; i <= M; i += TPF) {
            C z = Cx<T>::make(0, 0);
            if (i >= 1 && i < M) {
                if (va) z.x = (T)in(b, i, ja);
                if (vb) z.y = (T)in(b, i, jb);
            }
            buf[D::idx(i)] = z;
        }
    }
    __syncthreads();
    D::dst(buf, pl, t, wt);
    for (int i = 1 + t; i < M; i += TPF) {
        const C y = buf[D::idx(i)];
        if (va) out(b, i, ja, y.x);
        if (vb) out(b, i, jb, y.y);
    }
}

// Y pass: for each column i, x[i, :] = DST_y(mult(i, :) * DST_y(in[i, :])).
// A block owns 2*NG adjacent columns; loads and stores are row-coalesced.
template <class D, int NG>
__global__ void __launch_bounds__(D::TPF *NG, D::OCC / (D::TPF * NG))
    ypass_kernel(const typename D::Real *__restrict__ in, typename D::Real *__restrict__ out, long long bs, int ncols,
                 PlanT<typename D::Real> pl, Mult mult) {
    using T = typename D::Real;
    using C = typename D::C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *smem = reinterpret_cast<C *>(smem_raw);
    constexpr int TPF = D::TPF;
    const int M = pl.M;
    const int G = D::smem_len(M);
    const int g = threadIdx.x / TPF, t = threadIdx.x % TPF;
    C *buf = smem + g * G;
    double2 *wt = reinterpret_cast<double2 *>(smem_raw + scratch_offset<D>(M, NG)) + D::NWARP * g;
    const int b = blockIdx.y;
    const int c0 = blockIdx.x * 2 * NG;  // 0-based first column of the block
    const T *src = in + b * bs;
    T *dst = out + b * bs;
    constexpr int W = 2 * NG;
    if constexpr (D::MC > 0) {
        // compile-time trip count, loads issued in chunks of CH before their stores
        constexpr int NT = NG * TPF;
        constexpr int NIT = (W * (D::MC + 1) + NT - 1) / NT;
        constexpr int CH = 12;
#pragma unroll
        for (int k0 = 0; k0 < NIT; k0 += CH) {
            T v[CH];
#pragma unroll
            for (int k = 0; k < CH; ++k) {
                const int e = threadIdx.x + (k0 + k) * NT;
                const int c = e % W, jj = e / W;
                const int col = c0 + c;
                v[k] = (k0 + k < NIT && jj >= 1 && jj < D::MC && col < ncols) ? src[col + (long long)ncols * (jj - 1)]
                                                                               : (T)0;
            }
#pragma unroll
            for (int k = 0; k < CH; ++k) {
                const int e = threadIdx.x + (k0 + k) * NT;
                const int c = e % W, jj = e / W;
                if (k0 + k < NIT && jj <= D::MC) *(reinterpret_cast<T *>(smem + (c >> 1) * G + D::idx(jj)) + (c & 1)) = v[k];
            }
        }
    } else {
        for (int e = threadIdx.x; e < W * (M + 1); e += blockDim.x) {
            const int c = e % W, jj = e / W;
            const int col = c0 + c;
            T v = 0;
            if (jj >= 1 && jj < M && col < ncols) v = src[col + (long long)ncols * (jj - 1)];
            T *slot = reinterpret_cast<T *>(smem + (c >> 1) * G + D::idx(jj)) + (c & 1);
            *slot = v;
        }
    }
    __syncthreads();
    // DST, spectral multiply, DST; one loop body so the transform is emitted once
#pragma unroll 1
    for (int pass = 0; pass < 2; ++pass) {
        D::dst(buf, pl, t, wt);
        if (pass == 1) break;
        const int ia = c0 + 2 * g + 1, ib = c0 + 2 * g + 2;  // 1-based columns
        const double cb = mult.coef(b);
        if constexpr (D::MC > 0) {
            constexpr int NIT = (D::MC - 1 + TPF - 1) / TPF;
            const double cxa = ia <= ncols ? __ldg(&mult.cx[ia]) : 0.0, cxb = ib <= ncols ? __ldg(&mult.cx[ib]) : 0.0;
            double cyv[NIT];
#pragma unroll
            for (int k = 0; k < NIT; ++k) {
                const int jj = 1 + t + k * TPF;
                cyv[k] = jj < D::MC ? __ldg(&mult.cy[jj]) : 0.0;
            }
#pragma unroll
            for (int k = 0; k < NIT; ++k) {
                const int jj = 1 + t + k * TPF;
                if (jj >= D::MC) break;
                C y = buf[D::idx(jj)];
                y.x = (T)(y.x * ((ia <= ncols) ? mult.eval(cb, cxa, cyv[k]) : 0.0));
                y.y = (T)(y.y * ((ib <= ncols) ? mult.eval(cb, cxb, cyv[k]) : 0.0));
                buf[D::idx(jj)] = y;
            }
        } else {
            for (int jj = 1 + t; jj < M; jj += TPF) {
                C y = buf[D::idx(jj)];
                y.x = (T)(y.x * ((ia <= ncols) ? mult(cb, ia, jj) : 0.0));
                y.y = (T)(y.y * ((ib <= ncols) ? mult(cb, ib, jj) : 0.0));
                buf[D::idx(jj)] = y;
            }
        }
        __syncthreads();
    }
    for (int e = threadIdx.x; e < W * (M + 1); e += blockDim.x) {
        const int c = e % W, jj = e / W;
        const int col = c0 + c;
        if (jj >= 1 && jj < M && col < ncols) {
            const T *slot = reinterpret_cast<const T *>(smem + (c >> 1) * G + D::idx(jj)) + (c & 1);
            dst[col + (long long)ncols * (jj - 1)] = *slot;
        }
    }
}

// ---------------------------------------------------------------------------
// Merged trial solve of get_trial_state (src/fluid.jl:485-496):
//   Gamma_s = Ainv (A Gamma + rest),  rest = dt (1.5 N1 - 0.5 N2) + rhsbc.
// With S the 2D DST-I and S S = 1/scale:  S(A Gamma) = S(Gamma) / Lambda_e, so
//   Gamma_s = S( scale / Lambda_i * ( S(Gamma) / Lambda_e + S(rest) ) ),
// three passes instead of the reference's four transforms in six passes.
// ---------------------------------------------------------------------------

// X pass: row j of level b as one complex line z = Gamma + i rest.
template <class D, int NG>
__global__ void __launch_bounds__(D::TPF *NG, D::OCC / (D::TPF * NG))
    xpass_trial_kernel(const typename D::Real *__restrict__ gam, const typename D::Real *__restrict__ rest,
                       typename D::Real *__restrict__ t1, typename D::Real *__restrict__ t2, long long bs, int ld,
                       PlanT<typename D::Real> pl, int nrows) {
    using T = typename D::Real;
    using C = typename D::C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *smem = reinterpret_cast<C *>(smem_raw);
    constexpr int TPF = D::TPF;
    const int M = pl.M;
    const int G = D::smem_len(M);
    const int g = threadIdx.x / TPF, t = threadIdx.x % TPF;
    C *buf = smem + g * G;
    double2 *wt = reinterpret_cast<double2 *>(smem_raw + scratch_offset<D>(M, NG)) + D::NWARP * g;
    const int b = blockIdx.y;
    const int j = blockIdx.x * NG + g + 1;
    const bool valid = j <= nrows;
    const long long row = b * bs + (long long)ld * (j - 1);
    if constexpr (D::MC > 0) {
        constexpr int NIT = (D::MC + 1 + TPF - 1) / TPF;
        T za[NIT], zb[NIT];
#pragma unroll
        for (int k = 0; k < NIT; ++k) {
            const int i = t + k * TPF;
            const bool ok = valid && i >= 1 && i < D::MC;
            za[k] = ok ? gam[row + i - 1] : (T)0;
            zb[k] = ok ? rest[row + i - 1] : (T)0;
        }
#pragma unroll
        for (int k = 0; k < NIT; ++k) {
            const int i = t + k * TPF;
            if (i <= D::MC) buf[D::idx(i)] = Cx<T>::make(za[k], zb[k]);
        }
    } else {
        for (int i = t; i <= M; i += TPF) {
            C z = Cx<T>::make(0, 0);
            if (valid && i >= 1 && i < M) z = Cx<T>::make(gam[row + i - 1], rest[row + i - 1]);
            buf[D::idx(i)] = z;
        }
    }
    __syncthreads();
    D::dst(buf, pl, t, wt);
    if (valid)
        for (int i = 1 + t; i < M; i += TPF) {
            const C y = buf[D::idx(i)];
            t1[row + i - 1] = y.x;
            t2[row + i - 1] = y.y;
        }
}

// Y pass: a block owns 2NG adjacent columns.  Phase 1 transforms each column's
// (S_x Gamma, S_x rest) pair as one complex line and combines
//   v = scale / Lambda_i * (S Gamma / Lambda_e + S rest)
//     = (S Gamma (1 - lam c) + S rest) * scale / (1 + lam c),   c = dt / (2 Re hc^2);
// phase 2 transforms the real v of two columns packed as one complex line.
// Resident threads per SM the kernel is compiled for: 512 for FP32 lines of up to
// 512 points (at most 128 registers a thread), 256 otherwise.
template <class D>
constexpr int trial_occ() {
    return (sizeof(typename D::Real) == 4 && D::MC > 0 && D::MC <= 512) ? 512 : 256;
}
template <class D, int NG>
__global__ void __launch_bounds__(D::TPF *NG, trial_occ<D>() / (D::TPF * NG))
    ypass_trial_kernel(const typename D::Real *__restrict__ t1, const typename D::Real *__restrict__ t2,
                       typename D::Real *__restrict__ out, long long bs, int ncols, PlanT<typename D::Real> pl,
                       Mult mult) {
    using T = typename D::Real;
    using C = typename D::C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *smem = reinterpret_cast<C *>(smem_raw);
    constexpr int TPF = D::TPF;
    constexpr int W = 2 * NG;
    const int M = pl.M;
    const int G = D::smem_len(M);
    const int g = threadIdx.x / TPF, t = threadIdx.x % TPF;
    double2 *wt = reinterpret_cast<double2 *>(smem_raw + scratch_offset<D>(M, W)) + D::NWARP * g;
    const int b = blockIdx.y;
    const int c0 = blockIdx.x * W;  // 0-based first column
    const T *s1 = t1 + b * bs, *s2 = t2 + b * bs;
    T *dst = out + b * bs;
    if constexpr (D::MC > 0) {
        constexpr int NT = NG * TPF;
        constexpr int NIT = (W * (D::MC + 1) + NT - 1) / NT;
        constexpr int CH = 8;
#pragma unroll
        for (int k0 = 0; k0 < NIT; k0 += CH) {
            T va[CH], vb[CH];
#pragma unroll
            for (int k = 0; k < CH; ++k) {
                const int e = threadIdx.x + (k0 + k) * NT;
                const int c = e % W, jj = e / W;
                const int col = c0 + c;
                const bool ok = k0 + k < NIT && jj >= 1 && jj < D::MC && col < ncols;
                const long long o = col + (long long)ncols * (jj - 1);
                va[k] = ok ? s1[o] : (T)0;
                vb[k] = ok ? s2[o] : (T)0;
            }
#pragma unroll
            for (int k = 0; k < CH; ++k) {
                const int e = threadIdx.x + (k0 + k) * NT;
                const int c = e % W, jj = e / W;
                if (k0 + k < NIT && jj <= D::MC) smem[c * G + D::idx(jj)] = Cx<T>::make(va[k], vb[k]);
            }
        }
    } else
    for (int e = threadIdx.x; e < W * (M + 1); e += blockDim.x) {
        const int c = e % W, jj = e / W;
        const int col = c0 + c;
        C z = Cx<T>::make(0, 0);
        if (jj >= 1 && jj < M && col < ncols) {
            const long long o = col + (long long)ncols * (jj - 1);
            z = Cx<T>::make(s1[o], s2[o]);
        }
        smem[c * G + D::idx(jj)] = z;
    }
    __syncthreads();
    const double cb = mult.coef(b);
    const double scale = mult.scale;
#pragma unroll 1
    for (int r = 0; r < 2; ++r) {
        const int c = r * NG + g;
        C *buf = smem + c * G;
        D::dst(buf, pl, t, wt);
        const int col1 = c0 + c + 1;  // 1-based column
        const bool ok = col1 <= ncols;
        const double cxv = ok ? __ldg(&mult.cx[col1]) : 0.0;
        auto combine = [&](int jj, double cyj) {
            const C y = buf[D::idx(jj)];
            double v = 0.0;
            if (ok) {
                const double lam = -2 * ((cxv + cyj) - 2);
                v = ((double)y.x * (1 - lam * cb) + (double)y.y) * (scale * recip(1 + lam * cb));
            }
            buf[D::idx(jj)] = Cx<T>::make((T)v, 0);
        };
        if constexpr (D::MC > 0) {
            constexpr int NIT = (D::MC - 1 + TPF - 1) / TPF;
            double cyv[NIT];
#pragma unroll
            for (int k = 0; k < NIT; ++k) {
                const int jj = 1 + t + k * TPF;
                cyv[k] = jj < D::MC ? __ldg(&mult.cy[jj]) : 0.0;
            }
#pragma unroll
            for (int k = 0; k < NIT; ++k) {
                const int jj = 1 + t + k * TPF;
                if (jj < D::MC) combine(jj, cyv[k]);
            }
        } else {
            for (int jj = 1 + t; jj < M; jj += TPF) combine(jj, __ldg(&mult.cy[jj]));
        }
        __syncthreads();
    }
    // phase 2: pack columns (2g, 2g+1) into buffer 2g
    {
        C *ba = smem + (2 * g) * G;
        const C *bb = smem + (2 * g + 1) * G;
        for (int jj = 1 + t; jj < M; jj += TPF) ba[D::idx(jj)].y = bb[D::idx(jj)].x;
        __syncthreads();
        D::dst(ba, pl, t, wt);
    }
    for (int e = threadIdx.x; e < W * (M + 1); e += blockDim.x) {
        const int c = e % W, jj = e / W;
        const int col = c0 + c;
        if (jj >= 1 && jj < M && col < ncols) {
            const C y = smem[(c & ~1) * G + D::idx(jj)];
            dst[col + (long long)ncols * (jj - 1)] = (c & 1) ? y.y : y.x;
        }
    }
}

// ---------------------------------------------------------------------------
// Stencil kernels
// ---------------------------------------------------------------------------

// nonlinear (src/fluid.jl:441-455) = rot(direct_product(avg_flux(q + q0), Gamma, Gamma_bc)) / hc^2,
// with Gamma_bc = 0.25 get_bc(Gamma[:, lev+1]) (src/fluid.jl:473-483).  Batch b = level - 1.
template <class T, class TC = T>
struct NonlinArgs {
    const T *q;           // nq x L
    const T *gam;         // ng x L
    T *out;               // ng x L (state.nonlin[1])
    const T *n2;          // ng x L (state.nonlin[2]); with rest != nullptr
    T *rest;              // ng x L: dt (1.5 N1 - 0.5 N2) + rhsbc, or nullptr
    const StepDev *prm;
    Grid g;
    // Ensembles of cases of one shape, stacked case-major (batch b = case L + level - 1):
    // per-case Reynolds numbers (null: g.Re) and callback values (prm[case] when set)
    const double *re_tab = nullptr;
    int prm_per_case = 0;
    // Fields that start at level lev0 (batch b is level lev0 + b % (L - lev0 + 1));
    // coarse (element type TC), when set, is the Gamma of level lev0 + 1 (a field
    // of another precision); otherwise a field's coarser level is the next batch.
    int lev0 = 1;
    const TC *coarse = nullptr;
};

// Tile of the nonlinear kernel: kNlTX x kNlTY circulation points per block of
// kNlTX x kNlBY threads (two rows of outputs per thread).
constexpr int kNlTX = 32, kNlTY = 16, kNlBY = 8;

// nonlinear (src/fluid.jl:340-455) fused with the rhs assembly of
// get_trial_state (src/fluid.jl:487-493), all levels (blockIdx.z) at once.
// The tile's faces, Gamma (with a one-point halo) and N2 are copied to shared
// memory with cp.async, all in flight at once; every face average Q = (q + q0)
// pair sum / 2 (avg_flux!) is then formed once per tile, and each flux product
// (direct_product_loops!) and the rot! difference from there, with the
// reference's expressions, so each value rounds exactly as in a direct
// evaluation.
// EXT: the ensemble / mixed-precision features of NonlinArgs (levels from lev0,
// per-case tables, a coarse field of another type); without them the kernel
// keeps the single-case code (fewer live registers, more resident blocks).
template <class T, class TC = T, bool EXT = false>
__global__ void __launch_bounds__(kNlTX *kNlBY, EXT ? 4 : 5) nonlinear_kernel(NonlinArgs<T, TC> a) {
    const Grid &g = a.g;
    const int nx = g.nx, ny = g.ny;
    const int b = blockIdx.z;
    int lev = b + 1, cs = 0;
    if constexpr (EXT) {
        const int nlev = g.L - a.lev0 + 1;
        lev = a.lev0 + b % nlev;
        cs = b / nlev;
    }
    // per-case values, formed where they are used (no register held across the kernel)
    auto prm_of = [&]() -> const StepDev * { return EXT ? a.prm + (a.prm_per_case ? cs : 0) : a.prm; };
    auto re_of = [&]() -> double { return (EXT && a.re_tab) ? a.re_tab[cs] : g.Re; };
    const int I0 = blockIdx.x * kNlTX, J0 = blockIdx.y * kNlTY;  // outputs I0+1..I0+TX, J0+1..J0+TY
    const long long nq = (long long)(nx + 1) * ny + (long long)nx * (ny + 1), ng = (long long)(nx - 1) * (ny - 1);
    const long long nu = (long long)(nx + 1) * ny;
    const T *q = a.q + b * nq;
    const T *Gt = a.gam + b * ng;
    const TC *C = nullptr;
    if (lev < g.L) {
        if (EXT && a.coarse != nullptr)
            C = a.coarse + cs * ng;
        else if constexpr (std::is_same<T, TC>::value)
            C = a.gam + (b + 1) * ng;
    }
    __shared__ double aqy[kNlTY + 2][kNlTX];      // avg_qy(i, j), i = I0+2+x, j = J0+1+y
    __shared__ double aqx[kNlTY][kNlTX + 2];      // avg_qx(i, j), i = I0+1+x, j = J0+2+y
    __shared__ T gm[kNlTY + 2][kNlTX + 2];        // Gamma(i, j),  i = I0+x,   j = J0+y
    __shared__ T ru[kNlTY + 1][kNlTX + 2];        // q_u(i, j),    i = I0+1+x, j = J0+1+y
    __shared__ T rv[kNlTY + 2][kNlTX + 1];        // q_v(i, j),    i = I0+1+x, j = J0+1+y
    __shared__ T rn[kNlTY][kNlTX];                // N2(i, j),     i = I0+1+x, j = J0+1+y
    const int tid = threadIdx.y * kNlTX + threadIdx.x;
    constexpr int NT = kNlTX * kNlBY;
    const double hc = gridstep(g, lev);
    // base_flux! of a static grid is U hc on every face (fluid.jl:22-32)
    const double sbx = prm_of()->fs[0] * hc, sby = prm_of()->fs[1] * hc;
    const bool moving = g.grid_moving;
    // the tile's raw faces, Gamma and N2, all in flight at once (zeros outside the grid)
#pragma unroll
    for (int e = tid; e < (kNlTY + 1) * (kNlTX + 2); e += NT) {
        const int x = e % (kNlTX + 2), y = e / (kNlTX + 2);
        const int i = I0 + 1 + x, j = J0 + 1 + y;
        if (i <= nx + 1 && j <= ny)
            cp_async_elem(&ru[y][x], q + UI(i, j));
        else
            ru[y][x] = T(0);
    }
#pragma unroll
    for (int e = tid; e < (kNlTY + 2) * (kNlTX + 1); e += NT) {
        const int x = e % (kNlTX + 1), y = e / (kNlTX + 1);
        const int i = I0 + 1 + x, j = J0 + 1 + y;
        if (i <= nx && j <= ny + 1)
            cp_async_elem(&rv[y][x], q + VI(i, j));
        else
            rv[y][x] = T(0);
    }
#pragma unroll
    for (int e = tid; e < (kNlTY + 2) * (kNlTX + 2); e += NT) {
        const int x = e % (kNlTX + 2), y = e / (kNlTX + 2);
        const int i = I0 + x, j = J0 + y;
        if (i >= 1 && i <= nx - 1 && j >= 1 && j <= ny - 1)
            cp_async_elem(&gm[y][x], Gt + GI(i, j));
        else
            gm[y][x] = T(0);
    }
    if (a.rest) {
#pragma unroll
        for (int e = tid; e < kNlTY * kNlTX; e += NT) {
            const int x = e % kNlTX, y = e / kNlTX;
            const int i = I0 + 1 + x, j = J0 + 1 + y;
            if (i <= nx - 1 && j <= ny - 1)
                cp_async_elem(&rn[y][x], a.n2 + b * ng + GI(i, j));
            else
                rn[y][x] = T(0);
        }
    }
    cp_async_wait_all();
    __syncthreads();
    // face averages Q = (q + q0) pair sums / 2 (avg_flux!), each formed once per tile
#pragma unroll
    for (int e = tid; e < (kNlTY + 2) * kNlTX; e += NT) {
        const int x = e % kNlTX, y = e / kNlTX;
        const int i = I0 + 2 + x, j = J0 + 1 + y;
        double v = 0.0;
        if (i <= nx && j <= ny + 1) {
            // q_v(i, j) = rv[y][x + 1], q_v(i - 1, j) = rv[y][x]
            if (moving)
                v = ((double)rv[y][x + 1] + (double)rv[y][x] + base_flux_y(g, prm_of(), lev, i, j) +
                     base_flux_y(g, prm_of(), lev, i - 1, j)) / 2;
            else
                v = ((double)rv[y][x + 1] + (double)rv[y][x] + sby + sby) / 2;
        }
        aqy[y][x] = v;
    }
#pragma unroll
    for (int e = tid; e < kNlTY * (kNlTX + 2); e += NT) {
        const int x = e % (kNlTX + 2), y = e / (kNlTX + 2);
        const int i = I0 + 1 + x, j = J0 + 2 + y;
        double v = 0.0;
        if (i <= nx + 1 && j <= ny) {
            // q_u(i, j) = ru[y + 1][x], q_u(i, j - 1) = ru[y][x]
            if (moving)
                v = ((double)ru[y + 1][x] + (double)ru[y][x] + base_flux_x(g, prm_of(), lev, i, j) +
                     base_flux_x(g, prm_of(), lev, i, j - 1)) / 2;
            else
                v = ((double)ru[y + 1][x] + (double)ru[y][x] + sbx + sbx) / 2;
        }
        aqx[y][x] = v;
    }
    __syncthreads();
    const int x = threadIdx.x, I = I0 + 1 + x;
    if (I > nx - 1) return;
    // x-flux product at (I+1, j) (direct_product_loops!, fluid.jl:396-415)
    auto fqx = [&](int j) -> double {
        const int i = I + 1, yj = j - J0;
        if (j == 1) return (aqy[yj][x] * gm[yj][x + 1] + aqy[yj - 1][x] * (getbc(C, g, SIDE_B, i) * 0.25)) / 2;
        if (j == ny) return (aqy[yj - 1][x] * gm[yj - 1][x + 1] + aqy[yj][x] * (getbc(C, g, SIDE_T, i) * 0.25)) / 2;
        return (aqy[yj][x] * gm[yj][x + 1] + aqy[yj - 1][x] * gm[yj - 1][x + 1]) / 2;
    };
    // y-flux product at (i, J+1), i in {I, I+1} (fluid.jl:417-436)
    auto fqy = [&](int i, int y) -> double {
        const int xi = i - I0;  // aqx column of avg_qx(i, .) is xi - 1, gm column of Gamma(i, .) is xi
        if (i == 1) return -(aqx[y][xi] * gm[y + 1][xi] + aqx[y][xi - 1] * (getbc(C, g, SIDE_L, J0 + 2 + y) * 0.25)) / 2;
        if (i == nx)
            return -(aqx[y][xi - 1] * gm[y + 1][xi - 1] + aqx[y][xi] * (getbc(C, g, SIDE_R, J0 + 2 + y) * 0.25)) / 2;
        return -(aqx[y][xi] * gm[y + 1][xi] + aqx[y][xi - 1] * gm[y + 1][xi - 1]) / 2;
    };
#pragma unroll
    for (int k = 0; k < kNlTY / kNlBY; ++k) {
        const int y = threadIdx.y + k * kNlBY, J = J0 + 1 + y;
        if (J > ny - 1) break;
        // rot! at Gamma(I, J) with i = I+1, j = J+1 (fluid.jl:106-108)
        const double r = (fqx(J) - fqx(J + 1)) + (fqy(I + 1, y) - fqy(I, y));
        const double n1 = r * (1 / (hc * hc));
        a.out[b * ng + GI(I, J)] = (T)n1;
        if (a.rest) {
            // rest = dt b1 N1 + dt b2 N2 + rhsbc (fluid.jl:487-493), rhsbc = apply_bc!(0, get_bc(..); fac)
            double v = (g.dt * 1.5) * n1 + (g.dt * -0.5) * (double)rn[y][x];
            if (lev < g.L && on_ring(g, I, J)) {
                const double fac = 0.25 * g.dt / (re_of() * (hc * hc));
                v = v + apply_bc_at(0.0, C, g, I, J, fac);
            }
            a.rest[b * ng + GI(I, J)] = (T)v;
        }
    }
}

// 4-argument curl! (src/fluid.jl:230-276) with psi_bc = get_bc(psi_coarse) (zero if null).
// One thread per (i, j) writes both faces there: the x face u(i, j) (i <= nx+1,
// j <= ny) and the y face v(i, j) (i <= nx, j <= ny+1); inside the ring they share
// psi(i-1, j-1).  Batch b (blockIdx.z) uses psi + b*bs, q + b*qbs, coarse + b*cbs.
// win (device, may be null): only the faces in i0..i1 x j0..j1 are written, by a
// grid of any size sweeping the window.
template <class T, class TP, class TC>
__global__ void curl_kernel(T *__restrict__ qout, long long qbs, const TP *__restrict__ psi, long long bs,
                            const TC *__restrict__ coarse, long long cbs, Grid g, const int *__restrict__ win = nullptr) {
    const int nx = g.nx, ny = g.ny;
    const long long nu = (long long)(nx + 1) * ny;
    const int b = blockIdx.z;
    const TP *Pt = psi + b * bs;
    const TC *C = coarse ? coarse + b * cbs : nullptr;
    T *q = qout + b * qbs;
    auto P = [&](long long k) -> double { return (double)Pt[k]; };
    auto face = [&](int i, int j) {
        if (i >= 2 && i <= nx - 1 && j >= 2 && j <= ny - 1) {
            const double pc = P(GI(i - 1, j - 1));
            q[UI(i, j)] = (T)(P(GI(i - 1, j)) - pc);
            q[VI(i, j)] = (T)(pc - P(GI(i, j - 1)));
            return;
        }
        if (j <= ny) {
            double v;
            if (i == 1)
                v = getbc(C, g, SIDE_L, j + 1) - getbc(C, g, SIDE_L, j);
            else if (i == nx + 1)
                v = getbc(C, g, SIDE_R, j + 1) - getbc(C, g, SIDE_R, j);
            else if (j == 1)
                v = P(GI(i - 1, 1)) - getbc(C, g, SIDE_B, i);
            else if (j == ny)
                v = getbc(C, g, SIDE_T, i) - P(GI(i - 1, ny - 1));
            else
                v = P(GI(i - 1, j)) - P(GI(i - 1, j - 1));
            q[UI(i, j)] = (T)v;
        }
        if (i <= nx) {
            double v;
            if (j == 1)
                v = getbc(C, g, SIDE_B, i) - getbc(C, g, SIDE_B, i + 1);
            else if (j == ny + 1)
                v = getbc(C, g, SIDE_T, i) - getbc(C, g, SIDE_T, i + 1);
            else if (i == 1)
                v = getbc(C, g, SIDE_L, j) - P(GI(1, j - 1));
            else if (i == nx)
                v = P(GI(nx - 1, j - 1)) - getbc(C, g, SIDE_R, j);
            else
                v = P(GI(i - 1, j - 1)) - P(GI(i, j - 1));
            q[VI(i, j)] = (T)v;
        }
    };
    const int ti = blockIdx.x * blockDim.x + threadIdx.x, tj = blockIdx.y * blockDim.y + threadIdx.y;
    if (win == nullptr) {
        if (ti + 1 <= nx + 1 && tj + 1 <= ny + 1) face(ti + 1, tj + 1);
        return;
    }
    // the window (known on the device only) in grid-strided sweeps of a smaller grid
    const int i1 = min(win[1], nx + 1), j1 = min(win[3], ny + 1);
    for (int j = max(win[2], 1) + tj; j <= j1; j += gridDim.y * blockDim.y)
        for (int i = max(win[0], 1) + ti; i <= i1; i += gridDim.x * blockDim.x) face(i, j);
}

// coarsify! (src/fluid.jl:208-228): fine level -> central block of the next coarser level
// (the fine level may be of another element type TF).
// fine_central: the fine level is zero outside its own central block (faces
// nx/4+1 .. 3nx/4-1 by ny/4+1 .. 3ny/4-1); stencils wholly outside it give zero
// without a load.
template <class T, class TF = T>
__global__ void coarsify_kernel(T *__restrict__ coarse, const TF *__restrict__ fine, long long bs, Grid g,
                                int fine_central = 0) {
    const int nx = g.nx, ny = g.ny;
    const int ni = (nx / 2 - 2 - (-nx / 2 + 2)) / 2 + 1, nic = (nx / 4 - 1) - (-nx / 4 + 1) + 1;
    const int nj = (ny / 2 - 2 - (-ny / 2 + 2)) / 2 + 1, njc = (ny / 4 - 1) - (-ny / 4 + 1) + 1;
    const int ci = ni < nic ? ni : nic, cj = nj < njc ? nj : njc;
    const int a = blockIdx.x * blockDim.x + threadIdx.x, bb = blockIdx.y * blockDim.y + threadIdx.y;
    if (a >= ci || bb >= cj) return;
    const TF *Gf = fine + blockIdx.z * bs;
    T *Gc = coarse + blockIdx.z * bs;
    auto G = [&](long long k) -> double { return (double)Gf[k]; };
    const int i = nx / 2 + (-nx / 2 + 2) + 2 * a, ic = nx / 2 + (-nx / 4 + 1) + a;
    const int j = ny / 2 + (-ny / 2 + 2) + 2 * bb, jc = ny / 2 + (-ny / 4 + 1) + bb;
    if (fine_central && (i + 1 < nx / 4 + 1 || i - 1 > 3 * nx / 4 - 1 || j + 1 < ny / 4 + 1 || j - 1 > 3 * ny / 4 - 1)) {
        Gc[GI(ic, jc)] = (T)0.0;
        return;
    }
    Gc[GI(ic, jc)] = (T)(G(GI(i, j)) + 0.5 * (G(GI(i + 1, j)) + G(GI(i, j + 1)) + G(GI(i - 1, j)) + G(GI(i, j - 1))) +
                         0.25 * (G(GI(i + 1, j + 1)) + G(GI(i + 1, j - 1)) + G(GI(i - 1, j - 1)) + G(GI(i - 1, j + 1))));
}

// x = Binv z for the precomputed B^-1 (src/coupling.jl:187-192), column-major n x n.
// Grid (ceil(n/64), ceil(n/64)); partial sums part[chunk * n + row], summed in
// chunk order by binv_reduce_kernel (deterministic).
static __global__ void __launch_bounds__(256) binv_gemv_kernel(const double *__restrict__ A, const double *__restrict__ z,
                                                        double *__restrict__ part, int n) {
    __shared__ double red[4][64];
    const int r = threadIdx.x % 64, s = threadIdx.x / 64;
    const int row = blockIdx.x * 64 + r;
    const int cbeg = blockIdx.y * 64;
    double acc = 0.0;
    if (row < n) {
        if (cbeg + 64 <= n) {
#pragma unroll
            for (int c = cbeg + s; c < cbeg + 64; c += 4) acc += A[row + (long long)n * c] * __ldg(&z[c]);
        } else {
            for (int c = cbeg + s; c < n; c += 4) acc += A[row + (long long)n * c] * __ldg(&z[c]);
        }
    }
    red[s][r] = acc;
    __syncthreads();
    if (s == 0 && row < n) part[(long long)blockIdx.y * n + row] = ((red[0][r] + red[1][r]) + red[2][r]) + red[3][r];
}

// binv_gemv_kernel for the cases of a batched ensemble group (case = blockIdx.z,
// grid sized for the largest case): x = Binv Ftmp of each case into its partials.
static __global__ void __launch_bounds__(256) binv_gemv_multi_kernel(const CaseView *__restrict__ tab) {
    __shared__ double red[4][64];
    const CaseView &cv = tab[blockIdx.z];
    const int n = 2 * cv.P.np;
    const int nchunk = (n + 63) / 64;
    if ((int)blockIdx.x >= nchunk || (int)blockIdx.y >= nchunk) return;  // uniform over the block
    const double *__restrict__ A = cv.Binv;
    const double *__restrict__ z = cv.Ftmp;
    const int r = threadIdx.x % 64, s = threadIdx.x / 64;
    const int row = blockIdx.x * 64 + r;
    const int cbeg = blockIdx.y * 64;
    double acc = 0.0;
    if (row < n) {
        if (cbeg + 64 <= n) {
#pragma unroll
            for (int c = cbeg + s; c < cbeg + 64; c += 4) acc += A[row + (long long)n * c] * __ldg(&z[c]);
        } else {
            for (int c = cbeg + s; c < n; c += 4) acc += A[row + (long long)n * c] * __ldg(&z[c]);
        }
    }
    red[s][r] = acc;
    __syncthreads();
    if (s == 0 && row < n) cv.part[(long long)blockIdx.y * n + row] = ((red[0][r] + red[1][r]) + red[2][r]) + red[3][r];
}

// F~b = sum of the chunk partials; update_vars! fb = F~b h / dt (problem.jl:676-685);
// total force sum over panels (problem.jl:853-856).  One block.
static __global__ void binv_reduce_kernel(const double *__restrict__ part, int nchunk, int n, double *__restrict__ fbt,
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

// binv_reduce_kernel for the cases of a batched ensemble group: one block per case.
static __global__ void binv_reduce_multi_kernel(const CaseView *__restrict__ tab, double h, double dt) {
    __shared__ double sx[32], sy[32];
    const CaseView &cv = tab[blockIdx.x];
    const int n = 2 * cv.P.np, np = n / 2, nchunk = (n + 63) / 64;
    double tx = 0.0, ty = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        double v = 0.0;
        for (int c = 0; c < nchunk; ++c) v += cv.part[(long long)c * n + k];
        cv.Fbt[k] = v;
        const double f = v * h / dt;
        cv.fb[k] = f;
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
        cv.total[0] = ax;
        cv.total[1] = ay;
    }
}

// Gauss-Jordan inversion without pivoting of a positive definite matrix (stands
// in for LinearAlgebra.inv at src/coupling.jl:190).  Element (a, b) after step k
// of S: the pivot row scaled by 1/p, the pivot column by -1/p, the pivot by 1/p,
// every other element S[a,b] - S[a,k] (S[k,b] / p).
__device__ __forceinline__ double gj_elem(const double *__restrict__ S, int n, int k, int a, int b) {
    const double p = S[k + (long long)n * k];
    if (a == k && b == k) return 1.0 / p;
    if (a == k) return S[k + (long long)n * b] / p;
    if (b == k) return -S[a + (long long)n * k] / p;
    return S[a + (long long)n * b] - S[a + (long long)n * k] * (S[k + (long long)n * b] / p);
}
// Steps k and k+1 in one launch, from S into D (ping-pong buffers, so no element
// is read after another thread overwrote it): the step-(k+1) expression applied
// to the step-k elements gj_elem forms, the same values bit for bit as two
// one-step launches.  A pivot <= 0 sets *err to its step + 1.
static __global__ void gj_step2_kernel(const double *__restrict__ S, double *__restrict__ D, int n, int k, int *err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= n) return;
    const int k1 = k + 1;
    const double q = gj_elem(S, n, k, k1, k1);
    if (i == 0 && j == 0) {
        if (!(S[k + (long long)n * k] > 0.0))
            atomicCAS(err, 0, k + 1);
        else if (!(q > 0.0))
            atomicCAS(err, 0, k1 + 1);
    }
    const double rk = gj_elem(S, n, k, k1, j) / q;
    const double ck = gj_elem(S, n, k, i, k1);
    double v;
    if (i == k1 && j == k1)
        v = 1.0 / q;
    else if (i == k1)
        v = rk;
    else if (j == k1)
        v = -ck / q;
    else
        v = gj_elem(S, n, k, i, j) - ck * rk;
    D[i + (long long)n * j] = v;
}

// Steps k .. k + b - 1 (b <= kGJB) of the same elimination in one launch, as one
// block pivot: with K = {k .. k + b - 1}, P = S_KK^-1 (formed here by b
// unpivoted steps on the b x b block),
//   D_KK = P, D_KR = P S_KR, D_RK = -S_RK P, D_RR = S_RR - S_RK P S_KR,
// which equals the b single steps in exact arithmetic (not bit for bit).  One
// block per column j, threads over rows i (n <= blockDim.x * gridDim.x).  A
// pivot <= 0 sets *err to its step + 1.
constexpr int kGJB = 16;  // steps per block-pivot launch (blockDim >= kGJB^2)
static __global__ void gj_block_kernel(const double *__restrict__ S, double *__restrict__ D, int n, int k, int b,
                                       int *err) {
    __shared__ double Pm[kGJB][kGJB];
    __shared__ double T[kGJB];  // P S_Kj for this block's column j
    const int j = blockIdx.y, t = threadIdx.x;
    constexpr int kE = kGJB * kGJB;
    if (t < kE) {
        const int a = t / kGJB, c = t % kGJB;
        Pm[a][c] = (a < b && c < b) ? S[(k + a) + (long long)n * (k + c)] : 0.0;
    }
    __syncthreads();
    // in-place unpivoted Gauss-Jordan of the b x b block, thread t < kGJB^2 owning (t / kGJB, t % kGJB)
    const int a = t / kGJB, c = t % kGJB;
    for (int q = 0; q < b; ++q) {
        double p = 0.0, aq = 0.0, qc = 0.0, ac = 0.0;
        if (t < kE) {
            p = Pm[q][q];
            aq = Pm[a][q];
            qc = Pm[q][c];
            ac = Pm[a][c];
        }
        __syncthreads();
        if (t == 0 && blockIdx.x == 0 && j == 0 && !(p > 0.0)) atomicCAS(err, 0, k + q + 1);
        if (t < kE && a < b && c < b) {
            const double ip = 1.0 / p;
            if (a == q && c == q)
                Pm[a][c] = ip;
            else if (a == q)
                Pm[a][c] = qc * ip;
            else if (c == q)
                Pm[a][c] = -aq * ip;
            else
                Pm[a][c] = ac - aq * (qc * ip);
        }
        __syncthreads();
    }
    const bool jk = j >= k && j < k + b;
    if (t < b) {
        double v = 0.0;
        if (!jk)
            for (int e = 0; e < b; ++e) v += Pm[t][e] * S[(k + e) + (long long)n * j];
        T[t] = v;
    }
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + t;
    if (i >= n) return;
    const bool ik = i >= k && i < k + b;
    double v;
    if (ik && jk) {
        v = Pm[i - k][j - k];
    } else if (ik) {
        v = T[i - k];
    } else if (jk) {
        v = 0.0;
        for (int e = 0; e < b; ++e) v -= S[i + (long long)n * (k + e)] * Pm[e][j - k];
    } else {
        v = S[i + (long long)n * j];
        for (int e = 0; e < b; ++e) v -= S[i + (long long)n * (k + e)] * T[e];
    }
    D[i + (long long)n * j] = v;
}

// M <- (M + M^T) / 2 in place (n x n, column-major): thread (i, j) with i < j
// owns both entries of its pair.
static __global__ void symmetrize_kernel(double *__restrict__ M, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (i >= j || j >= n) return;
    const double a = M[i + (long long)n * j], b = M[j + (long long)n * i];
    const double v = 0.5 * (a + b);
    M[i + (long long)n * j] = v;
    M[j + (long long)n * i] = v;
}

// Identity columns [c0, c0+nb) of a 2np-length basis, one per batch.
static __global__ void unit_columns_kernel(double *__restrict__ f, int n, int c0, int nb) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * nb) return;
    const int b = t / n, k = t % n;
    f[t] = (k == c0 + b) ? 1.0 : 0.0;
}

}  // namespace ibpm
