// fft_dst.cuh -- shared-memory DST-I line transforms for the Poisson / CN solves.
//
// The reference applies x = S(S(b) * scale / Lambda) with S the unnormalised 2D
// DST-I (FFTW RODFT00 over both dims, src/fluid.jl:113-115 and 145-166).  Here
// a 2D solve is three passes over the (nx-1) x (ny-1) field:
//   X pass   : DST along x of every row            (rows are contiguous)
//   Y pass   : DST along y, multiply, DST along y  (coalesced column blocks)
//   X pass   : DST along x, with a fused epilogue
// Each length-(M-1) DST-I is one complex M-point FFT of two packed real lines
// z = a + i b, pre-twiddled with v_j = sin(pi j/M)(z_j + z_{M-j}) + (z_j - z_{M-j})/2.
// With V = FFT(v):  y_1 = V_0,  y_{2k} = i (V_k - V_{M-k}),
//                   y_{2k+1} = y_{2k-1} + V_k + V_{M-k}  (a prefix scan),
// and DST(a) = Re y, DST(b) = Im y.  This file holds the runtime mixed-radix
// (4, 2, 3, 5) Stockham transform for any even M = 2^a 3^b 5^c <= 1024; each
// stage keeps its butterflies in registers between one read phase and one write
// phase, so a line needs a single (M+1)-entry buffer.  fft_pow2.cuh holds the
// compile-time power-of-two transforms behind the same interface.
//
// Element type T is double or float; the prefix scan always accumulates in
// double (its partial sums are larger than its outputs).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace ibpm {

constexpr int kTPF = 64;        // threads per FFT group (two warps)
constexpr int kMaxV = 20;       // complex values a thread holds in one stage
constexpr int kMaxE = 8;        // scan values per thread (M/2/kTPF, M <= 1024)
constexpr int kMaxStages = 12;
constexpr int kMaxM = 1024;     // largest transform length (nx or ny)

template <class T>
struct PlanT {
    using C = typename Cx<T>::type;
    int M;                      // transform length (nx or ny); DST length M-1
    int nst;                    // number of FFT stages
    int radix[kMaxStages];
    const C *tw;                // tw[k] = exp(-2 pi i k / M), k < M
    const T *sn;                // sn[j] = sin(pi j / M), j <= M
};

__host__ __device__ __forceinline__ double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 operator*(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
__host__ __device__ __forceinline__ float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 operator*(float s, float2 a) { return make_float2(s * a.x, s * a.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// multiply by -i
__device__ __forceinline__ double2 mul_mi(double2 a) { return make_double2(a.y, -a.x); }
__device__ __forceinline__ float2 mul_mi(float2 a) { return make_float2(a.y, -a.x); }
__device__ __forceinline__ double2 to_d2(double2 a) { return a; }
__device__ __forceinline__ double2 to_d2(float2 a) { return make_double2(a.x, a.y); }
template <class C>
__device__ __forceinline__ C from_d2(double2 a);
template <>
__device__ __forceinline__ double2 from_d2<double2>(double2 a) { return a; }
template <>
__device__ __forceinline__ float2 from_d2<float2>(double2 a) { return make_float2((float)a.x, (float)a.y); }

template <int R, class C>
struct Dft;

template <class C>
struct Dft<2, C> {
    static __device__ __forceinline__ void run(C *v) {
        const C a = v[0], b = v[1];
        v[0] = a + b;
        v[1] = a - b;
    }
};

template <class C>
struct Dft<4, C> {
    static __device__ __forceinline__ void run(C *v) {
        const C t0 = v[0] + v[2], t1 = v[0] - v[2];
        const C t2 = v[1] + v[3], t3 = mul_mi(v[1] - v[3]);
        v[0] = t0 + t2;
        v[2] = t0 - t2;
        v[1] = t1 + t3;
        v[3] = t1 - t3;
    }
};

template <class C>
struct Dft<3, C> {
    static __device__ __forceinline__ void run(C *v) {
        using R = decltype(C().x);
        const R s3 = (R)0.86602540378443864676;  // sin(2 pi / 3)
        const C a1 = v[1] + v[2], d1 = v[1] - v[2];
        const C x0 = v[0] + a1;
        const C t = v[0] - (R)0.5 * a1;
        const C u = mul_mi(s3 * d1);
        v[0] = x0;
        v[1] = t + u;
        v[2] = t - u;
    }
};

template <class C>
struct Dft<5, C> {
    static __device__ __forceinline__ void run(C *v) {
        using R = decltype(C().x);
        const R c1 = (R)0.30901699437494742410, c2 = (R)-0.80901699437494742410;  // cos(2pi/5), cos(4pi/5)
        const R s1 = (R)0.95105651629515357212, s2 = (R)0.58778525229247312917;   // sin(2pi/5), sin(4pi/5)
        const C b1 = v[1] + v[4], b2 = v[2] + v[3];
        const C d1 = v[1] - v[4], d2 = v[2] - v[3];
        const C x0 = v[0] + b1 + b2;
        const C e1 = v[0] + c1 * b1 + c2 * b2;
        const C e2 = v[0] + c2 * b1 + c1 * b2;
        const C f1 = mul_mi(s1 * d1 + s2 * d2);
        const C f2 = mul_mi(s2 * d1 - s1 * d2);
        v[0] = x0;
        v[1] = e1 + f1;
        v[4] = e1 - f1;
        v[2] = e2 + f2;
        v[3] = e2 - f2;
    }
};

// One Stockham stage of radix R over buf[0..M).  Every thread of the block
// must call it (it contains block barriers).
template <int R, class C>
__device__ __forceinline__ void fft_stage(C *buf, int M, int Ns, const C *__restrict__ tw, int t) {
    constexpr int KMAX = kMaxV / R;
    const int nb = M / R;
    const int twstep = M / (Ns * R);
    C v[KMAX][R];
    int dst[KMAX];
#pragma unroll
    for (int kb = 0; kb < KMAX; ++kb) {
        const int j = t + kb * kTPF;
        dst[kb] = -1;
        if (j < nb) {
            const int k = j % Ns;
            v[kb][0] = buf[j];
#pragma unroll
            for (int r = 1; r < R; ++r) v[kb][r] = cmul(buf[j + r * nb], __ldg(&tw[r * k * twstep]));
            Dft<R, C>::run(v[kb]);
            dst[kb] = (j / Ns) * Ns * R + k;
        }
    }
    __syncthreads();
#pragma unroll
    for (int kb = 0; kb < KMAX; ++kb) {
        if (dst[kb] >= 0) {
#pragma unroll
            for (int r = 0; r < R; ++r) buf[dst[kb] + r * Ns] = v[kb][r];
        }
    }
    __syncthreads();
}

// Forward complex FFT of buf[0..M) in place (natural order in and out).
template <class T>
__device__ __forceinline__ void fft(typename Cx<T>::type *buf, const PlanT<T> &pl, int t) {
    using C = typename Cx<T>::type;
    int Ns = 1;
    for (int s = 0; s < pl.nst; ++s) {
        const int R = pl.radix[s];
        if (R == 4)
            fft_stage<4, C>(buf, pl.M, Ns, pl.tw, t);
        else if (R == 2)
            fft_stage<2, C>(buf, pl.M, Ns, pl.tw, t);
        else if (R == 3)
            fft_stage<3, C>(buf, pl.M, Ns, pl.tw, t);
        else
            fft_stage<5, C>(buf, pl.M, Ns, pl.tw, t);
        Ns *= R;
    }
}

// DST pre-twiddle in place: buf[1..M-1] holds z, buf[0] and buf[M] are read as 0.
template <class T>
__device__ __forceinline__ void dst_pre(typename Cx<T>::type *buf, const PlanT<T> &pl, int t) {
    using C = typename Cx<T>::type;
    const int M = pl.M, H = M >> 1;
    for (int j = t; j <= H; j += kTPF) {
        if (j == 0) {
            buf[0] = Cx<T>::make(0, 0);
        } else if (j == H) {
            const C z = buf[H];
            const T s = __ldg(&pl.sn[H]);
            buf[H] = s * (z + z);
        } else {
            const C a = buf[j], b = buf[M - j];
            const T s = __ldg(&pl.sn[j]);
            buf[j] = s * (a + b) + (T)0.5 * (a - b);
            buf[M - j] = s * (a + b) + (T)0.5 * (b - a);
        }
    }
    __syncthreads();
}

// DST post-processing: buf[0..M) holds V; on return buf[1..M-1] holds y and
// buf[0] = buf[M] = 0.  wt: two double2 scratch slots for this group.
template <class T>
__device__ __forceinline__ void dst_post(typename Cx<T>::type *buf, const PlanT<T> &pl, int t, double2 *wt) {
    using C = typename Cx<T>::type;
    const int M = pl.M, H = M >> 1;
    const int E = (H + kTPF - 1) / kTPF;
    const int k0 = t * E;
    double2 c[kMaxE];
    C ev[kMaxE];
    double2 run = make_double2(0.0, 0.0);
#pragma unroll
    for (int e = 0; e < kMaxE; ++e) {
        const int k = k0 + e;
        c[e] = make_double2(0.0, 0.0);
        ev[e] = Cx<T>::make(0, 0);
        if (e < E && k < H) {
            const C Vk = buf[k];
            if (k == 0) {
                run = to_d2(Vk);
            } else {
                const C Vm = buf[M - k];
                run = run + to_d2(Vk + Vm);
                const C d = Vk - Vm;
                ev[e] = Cx<T>::make(-d.y, d.x);  // i (V_k - V_{M-k})
            }
            c[e] = run;
        }
    }
    // exclusive scan of the thread totals across the 64-thread group
    const int lane = t & 31, w = t >> 5;
    double2 incl = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double ux = __shfl_up_sync(0xffffffffu, incl.x, o);
        const double uy = __shfl_up_sync(0xffffffffu, incl.y, o);
        if (lane >= o) incl = incl + make_double2(ux, uy);
    }
    double2 excl;
    excl.x = __shfl_up_sync(0xffffffffu, incl.x, 1);
    excl.y = __shfl_up_sync(0xffffffffu, incl.y, 1);
    if (lane == 0) excl = make_double2(0.0, 0.0);
    if (lane == 31) wt[w] = incl;
    __syncthreads();  // all reads of buf done, warp totals visible
    if (w == 1) excl = excl + wt[0];
#pragma unroll
    for (int e = 0; e < kMaxE; ++e) {
        const int k = k0 + e;
        if (e < E && k < H) {
            buf[2 * k + 1] = from_d2<C>(c[e] + excl);
            if (k > 0) buf[2 * k] = ev[e];
        }
    }
    if (t == 0) {
        buf[0] = Cx<T>::make(0, 0);
        buf[M] = Cx<T>::make(0, 0);
    }
    __syncthreads();
}

// Full DST-I of the packed lines in buf[1..M-1] (in place).
template <class T>
__device__ __forceinline__ void dst_inplace(typename Cx<T>::type *buf, const PlanT<T> &pl, int t, double2 *wt) {
    dst_pre<T>(buf, pl, t);
    fft<T>(buf, pl, t);
    dst_post<T>(buf, pl, t, wt);
}

}  // namespace ibpm
