// fft_pow2.cuh -- DST-I line transform for power-of-two lengths M = 64..1024.
//
// Same algorithm as fft_dst.cuh (complex M-point FFT of two packed lines with
// the sin pre-twiddle and the prefix-scan post-processing), specialised at
// compile time: the Stockham stages use radix 16 / 8 / 4 butterflies held in
// registers (three shared-memory round trips for M = 1024 instead of five), the
// pre-twiddle is formed in registers from the first stage's reads, all strides
// and index splits are constants, the shared buffer is padded by one complex per
// 16 to keep the strided Stockham writes free of bank conflicts, and the
// post-processing scan runs on warp shuffles with one block barrier.
// T (double or float) is the element type; the scan accumulates in double.
#pragma once
#include "fft_dst.cuh"

namespace ibpm {

// Barrier policies of the transforms: the whole block (every group of the block
// steps through the transform together), or only the TPF threads of the
// calling thread's group, with hardware barrier 1 + group index (named
// barriers; groups of one block then run out of step with each other).
struct CtaSync {
    static __device__ __forceinline__ void sync() { __syncthreads(); }
};
template <int TPF>
struct GroupSync {
    static __device__ __forceinline__ void sync() {
        asm volatile("bar.sync %0, %1;" ::"r"((int)(threadIdx.x / TPF) + 1), "r"(TPF) : "memory");
    }
};

// Padded shared-memory index: one spare double2 per 16.
__device__ __forceinline__ int pad16(int i) { return i + (i >> 4); }
__host__ __device__ constexpr int padded_len(int M) { return (M + 1) + ((M + 1) >> 4) + 1; }

// ---- small DFTs (forward, e^{-2 pi i / R}) with constant twiddles ----

constexpr double kR2 = 0.70710678118654752440;   // sqrt(2)/2
constexpr double kC16 = 0.92387953251128675613;  // cos(pi/8)
constexpr double kS16 = 0.38268343236508977173;  // sin(pi/8)

// multiply by W16^m for the exponents the radix-16 butterfly needs
template <int m, class C>
struct W16;
template <class C>
struct W16<0, C> {
    static __device__ __forceinline__ C mul(C a) { return a; }
};
template <class C>
struct W16<1, C> {
    static __device__ __forceinline__ C mul(C a) {
        using R = decltype(C().x);
        return C{a.x * (R)kC16 + a.y * (R)kS16, a.y * (R)kC16 - a.x * (R)kS16};
    }
};
template <class C>
struct W16<2, C> {
    static __device__ __forceinline__ C mul(C a) {
        using R = decltype(C().x);
        return C{(R)kR2 * (a.x + a.y), (R)kR2 * (a.y - a.x)};
    }
};
template <class C>
struct W16<3, C> {
    static __device__ __forceinline__ C mul(C a) {
        using R = decltype(C().x);
        return C{a.x * (R)kS16 + a.y * (R)kC16, a.y * (R)kS16 - a.x * (R)kC16};
    }
};
template <class C>
struct W16<4, C> {
    static __device__ __forceinline__ C mul(C a) { return mul_mi(a); }
};
template <class C>
struct W16<6, C> {
    static __device__ __forceinline__ C mul(C a) {
        using R = decltype(C().x);
        return C{(R)kR2 * (a.y - a.x), -(R)kR2 * (a.x + a.y)};
    }
};
template <class C>
struct W16<9, C> {
    static __device__ __forceinline__ C mul(C a) {
        using R = decltype(C().x);
        return C{-a.x * (R)kC16 - a.y * (R)kS16, a.x * (R)kS16 - a.y * (R)kC16};
    }
};
template <int m, class C>
__device__ __forceinline__ C w16(C a) {
    return W16<m, C>::mul(a);
}

template <class C>
__device__ __forceinline__ void dft4(C &a0, C &a1, C &a2, C &a3) {
    const C t0 = a0 + a2, t1 = a0 - a2, t2 = a1 + a3, t3 = mul_mi(a1 - a3);
    a0 = t0 + t2;
    a2 = t0 - t2;
    a1 = t1 + t3;
    a3 = t1 - t3;
}

template <int R, class C>
struct DftC;

template <class C>
struct DftC<4, C> {
    static __device__ __forceinline__ void run(C *v) { dft4(v[0], v[1], v[2], v[3]); }
};

template <class C>
struct DftC<2, C> {
    static __device__ __forceinline__ void run(C *v) {
        const C a = v[0], b = v[1];
        v[0] = a + b;
        v[1] = a - b;
    }
};

// 8 = 4 x 2: n = 2 n1 + n2, k = k1 + 4 k2
template <class C>
struct DftC<8, C> {
    static __device__ __forceinline__ void run(C *v) {
        C a0 = v[0], a1 = v[2], a2 = v[4], a3 = v[6];  // n2 = 0
        C b0 = v[1], b1 = v[3], b2 = v[5], b3 = v[7];  // n2 = 1
        dft4(a0, a1, a2, a3);
        dft4(b0, b1, b2, b3);
        b1 = w16<2>(b1);  // W8^1
        b2 = mul_mi(b2);  // W8^2
        b3 = w16<6>(b3);  // W8^3
        v[0] = a0 + b0;
        v[4] = a0 - b0;
        v[1] = a1 + b1;
        v[5] = a1 - b1;
        v[2] = a2 + b2;
        v[6] = a2 - b2;
        v[3] = a3 + b3;
        v[7] = a3 - b3;
    }
};

// 16 = 4 x 4: n = 4 n1 + n2, k = k1 + 4 k2
template <class C>
struct DftC<16, C> {
    static __device__ __forceinline__ void run(C *v) {
        C a[4][4];  // a[n2][k1]
#pragma unroll
        for (int n2 = 0; n2 < 4; ++n2) {
            a[n2][0] = v[n2];
            a[n2][1] = v[4 + n2];
            a[n2][2] = v[8 + n2];
            a[n2][3] = v[12 + n2];
            dft4(a[n2][0], a[n2][1], a[n2][2], a[n2][3]);
        }
        a[1][1] = w16<1>(a[1][1]);
        a[1][2] = w16<2>(a[1][2]);
        a[1][3] = w16<3>(a[1][3]);
        a[2][1] = w16<2>(a[2][1]);
        a[2][2] = w16<4>(a[2][2]);
        a[2][3] = w16<6>(a[2][3]);
        a[3][1] = w16<3>(a[3][1]);
        a[3][2] = w16<6>(a[3][2]);
        a[3][3] = w16<9>(a[3][3]);
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) {
            C b0 = a[0][k1], b1 = a[1][k1], b2 = a[2][k1], b3 = a[3][k1];
            dft4(b0, b1, b2, b3);
            v[k1] = b0;
            v[k1 + 4] = b1;
            v[k1 + 8] = b2;
            v[k1 + 12] = b3;
        }
    }
};

template <class C>
struct DftC<3, C> {
    static __device__ __forceinline__ void run(C *v) { Dft<3, C>::run(v); }
};

// ---- compile-time plans ----
// Every stage has NB = M/R butterflies with NB % 16 == 0 and a stride NS that
// is 1 or a multiple of 16, so all padded shared-memory offsets of a stage are
// compile-time constants added to one per-thread base.
// A plan lists the radices R0..R4 (1 = unused); TPF threads per line pair;
// OCC the resident threads per SM the kernels are compiled for (it caps the
// registers per thread at 65536 / OCC).
template <int TPF_, int R0_, int R1_, int R2_, int R3_ = 1, int R4_ = 1, int OCC_ = 512>
struct PlanCT {
    static constexpr int TPF = TPF_;
    static constexpr int OCC = OCC_;
    static constexpr int R0 = R0_, R1 = R1_, R2 = R2_, R3 = R3_, R4 = R4_;
};
template <int M>
struct Pow2Plan;
template <>
struct Pow2Plan<1024> : PlanCT<64, 16, 16, 4> {};
template <>
struct Pow2Plan<512> : PlanCT<64, 16, 8, 4> {};
template <>
struct Pow2Plan<256> : PlanCT<32, 16, 4, 4> {};

// padded offset of (base + c) given that base % 16 == b16 is known to leave room
template <int NS, int R, int r>
struct WriteOff {
    // NS == 1: targets R j + r with (R j) % 16 + r < 16 -> base + r
    // NS % 16 == 0: targets d + r NS -> pad(d) + r NS 17/16
    static constexpr int value = NS == 1 ? r : r * NS * 17 / 16;
};

// Padded offset of the r-th output of a butterfly relative to its first output
// d = (j / NS) NS R + (j % NS): a constant when NS is a multiple of 16 (then
// d + r NS crosses r NS / 16 pads) or when NS R divides 16 (then the R outputs
// stay inside one 16-entry row).
template <int R, int NS>
__host__ __device__ constexpr int write_off(int r) {
    return NS % 16 == 0 ? r * NS * 17 / 16 : r * NS;
}

// One Stockham stage with compile-time sizes on a padded buffer.
template <int M, int R, int NS, int TPF, class C, class S = CtaSync>
__device__ __forceinline__ void stage_ct(C *buf, const C *__restrict__ tw, int t) {
    constexpr int NB = M / R;
    constexpr int K = NB >= TPF ? NB / TPF : 1;  // butterflies per thread
    constexpr bool ALL = NB >= TPF;              // every thread has a butterfly
    constexpr int TWS = M / (NS * R);
    static_assert((NB % TPF == 0 || TPF % NB == 0) && NB % 16 == 0, "stage layout");
    static_assert(NS % 16 == 0 || 16 % (NS * R) == 0, "stage stride");
    constexpr int RSTEP = NB * 17 / 16;  // padded distance between the R inputs
    C v[K][R];
#pragma unroll
    for (int kb = 0; kb < K; ++kb) {
        const int j = t + kb * TPF;
        if (!ALL && j >= NB) break;
        const int k = j % NS;
        C w[R];
        if (NS > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) w[r] = __ldg(&tw[r * k * TWS]);
        }
        const C *src = buf + pad16(j);
#pragma unroll
        for (int r = 0; r < R; ++r) v[kb][r] = src[r * RSTEP];
        if (NS > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) v[kb][r] = cmul(v[kb][r], w[r]);
        }
        DftC<R, C>::run(v[kb]);
    }
    S::sync();
#pragma unroll
    for (int kb = 0; kb < K; ++kb) {
        const int j = t + kb * TPF;
        if (!ALL && j >= NB) break;
        const int k = j % NS;
        C *dst = buf + pad16((j / NS) * NS * R + k);
#pragma unroll
        for (int r = 0; r < R; ++r) dst[write_off<R, NS>(r)] = v[kb][r];
    }
    S::sync();
}

// The first Stockham stage (stride 1) with the DST pre-twiddle folded into its
// reads: input n is v_n = s (z_n + z_{M-n}) + (z_n - z_{M-n}) / 2 with
// s = sin(pi min(n, M-n) / M), v_0 = 0 -- the values the separate pre-twiddle
// pass writes, formed in registers from z_n and its mirror.  buf[0..M] hold z
// (z_0 = z_M = 0).
template <int M, int R, int TPF, class C, class T, class S = CtaSync>
__device__ __forceinline__ void stage_first_pre(C *buf, const T *__restrict__ sn, int t) {
    constexpr int NB = M / R;
    constexpr int K = NB >= TPF ? NB / TPF : 1;
    constexpr bool ALL = NB >= TPF;
    constexpr int H = M / 2;
    static_assert((NB % TPF == 0 || TPF % NB == 0) && NB % 16 == 0, "stage layout");
    constexpr int RSTEP = NB * 17 / 16;
    T s[K][R];
#pragma unroll
    for (int kb = 0; kb < K; ++kb) {  // table loads first
        const int j = t + kb * TPF;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int n = j + r * NB;
            s[kb][r] = (ALL || j < NB) ? __ldg(&sn[n <= H ? n : M - n]) : (T)0;
        }
    }
    C v[K][R];
#pragma unroll
    for (int kb = 0; kb < K; ++kb) {
        const int j = t + kb * TPF;
        if (!ALL && j >= NB) break;
        const C *src = buf + pad16(j);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int n = j + r * NB;
            const C a = src[r * RSTEP], b = buf[pad16(M - n)];
            v[kb][r] = n == 0 ? Cx<T>::make(0, 0) : s[kb][r] * (a + b) + (T)0.5 * (a - b);
        }
        DftC<R, C>::run(v[kb]);
    }
    S::sync();
#pragma unroll
    for (int kb = 0; kb < K; ++kb) {
        const int j = t + kb * TPF;
        if (!ALL && j >= NB) break;
        C *dst = buf + pad16(j * R);
#pragma unroll
        for (int r = 0; r < R; ++r) dst[write_off<R, 1>(r)] = v[kb][r];
    }
    S::sync();
}

// A Stockham stage with compile-time sizes for any radix and stride: the same
// butterflies as stage_ct, with the padded shared-memory index computed for
// every element (strides with a factor 3 do not keep the pads at constant
// offsets).  Butterfly j < M/R takes inputs j + r M/R and writes outputs
// (j / NS) NS R + j % NS + r NS.
template <int M, int R, int NS, int TPF, class C, class S = CtaSync>
__device__ __forceinline__ void stage_gen(C *buf, const C *__restrict__ tw, int t) {
    constexpr int NB = M / R;
    constexpr int K = (NB + TPF - 1) / TPF;
    constexpr int TWS = M / (NS * R);
    C v[K][R];
#pragma unroll
    for (int kb = 0; kb < K; ++kb) {
        const int j = t + kb * TPF;
        if (j >= NB) break;
        const int k = j % NS;
        C w[R];
        if (NS > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) w[r] = __ldg(&tw[r * k * TWS]);
        }
#pragma unroll
        for (int r = 0; r < R; ++r) v[kb][r] = buf[pad16(j + r * NB)];
        if (NS > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) v[kb][r] = cmul(v[kb][r], w[r]);
        }
        DftC<R, C>::run(v[kb]);
    }
    S::sync();
#pragma unroll
    for (int kb = 0; kb < K; ++kb) {
        const int j = t + kb * TPF;
        if (j >= NB) break;
        const int base = (j / NS) * NS * R + j % NS;
#pragma unroll
        for (int r = 0; r < R; ++r) buf[pad16(base + r * NS)] = v[kb][r];
    }
    S::sync();
}

// stage_gen's first stage (NS = 1) with the DST pre-twiddle folded into its reads,
// as stage_first_pre.
template <int M, int R, int TPF, class C, class T, class S = CtaSync>
__device__ __forceinline__ void stage_gen_first_pre(C *buf, const T *__restrict__ sn, int t) {
    constexpr int NB = M / R;
    constexpr int K = (NB + TPF - 1) / TPF;
    constexpr int H = M / 2;
    T s[K][R];
#pragma unroll
    for (int kb = 0; kb < K; ++kb) {
        const int j = t + kb * TPF;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int n = j + r * NB;
            s[kb][r] = j < NB ? __ldg(&sn[n <= H ? n : M - n]) : (T)0;
        }
    }
    C v[K][R];
#pragma unroll
    for (int kb = 0; kb < K; ++kb) {
        const int j = t + kb * TPF;
        if (j >= NB) break;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int n = j + r * NB;
            const C a = buf[pad16(n)], b = buf[pad16(M - n)];
            v[kb][r] = n == 0 ? Cx<T>::make(0, 0) : s[kb][r] * (a + b) + (T)0.5 * (a - b);
        }
        DftC<R, C>::run(v[kb]);
    }
    S::sync();
#pragma unroll
    for (int kb = 0; kb < K; ++kb) {
        const int j = t + kb * TPF;
        if (j >= NB) break;
#pragma unroll
        for (int r = 0; r < R; ++r) buf[pad16(j * R + r)] = v[kb][r];
    }
    S::sync();
}

template <int M, class T, class PL = Pow2Plan<M>>
struct Pow2Dst {
    using P = PL;
    // FP32 lines of up to 256 points are compiled for twice the plan's resident
    // threads (64 registers; the Y pass spills 32-52 bytes) -- measured faster
    static constexpr int OCC = (sizeof(T) == 4 && M <= 256) ? 2 * P::OCC : P::OCC;
    static constexpr int MC = M;  // compile-time transform length
    using Real = T;
    using C = typename Cx<T>::type;
    static constexpr int TPF = P::TPF;
    static constexpr int NWARP = TPF / 32;
    static __host__ __device__ constexpr int smem_len(int) { return padded_len(M); }

    static __device__ __forceinline__ int idx(int i) { return pad16(i); }

    // post-processing: V in buf[0..M) -> y in buf[1..M-1]; buf[0] = buf[M] = 0.
    // Thread t owns the E = H/TPF consecutive k in [t E, t E + E): a sequential
    // scan of its segment, one warp shuffle scan of the segment totals, and one
    // block barrier for the warp totals.
    template <class S = CtaSync>
    static __device__ __forceinline__ void post(C *buf, int t, double2 *wt) {
        constexpr int H = M / 2;
        constexpr int E = H / TPF;
        static_assert(E >= 1 && H % TPF == 0, "scan layout");
        const int lane = t & 31, w = t >> 5;
        const int k0 = t * E;
        double2 odd[E];
        C even[E];
        double2 run = make_double2(0.0, 0.0);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int k = k0 + e;
            const C Vk = buf[pad16(k)];
            const C Vm = buf[pad16(M - k)];  // k == 0 reads buf[M] = V_M, unused
            if (k == 0) {
                run = to_d2(Vk);
                even[e] = Cx<T>::make(0, 0);
            } else {
                run = run + to_d2(Vk + Vm);
                const C d = Vk - Vm;
                even[e] = Cx<T>::make(-d.y, d.x);
            }
            odd[e] = run;
        }
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
        if (NWARP > 1 && lane == 31) wt[w] = incl;
        S::sync();  // all reads of V done; warp totals visible
#pragma unroll
        for (int q = 0; q < NWARP - 1; ++q)
            if (q < w) excl = excl + wt[q];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int k = k0 + e;
            buf[pad16(2 * k + 1)] = from_d2<C>(odd[e] + excl);
            if (k > 0) buf[pad16(2 * k)] = even[e];
        }
        if (t == 0) {
            buf[0] = Cx<T>::make(0, 0);
            buf[pad16(M)] = Cx<T>::make(0, 0);
        }
        S::sync();
    }

    // the FFT of the pre-twiddled packed lines, the pre-twiddle folded into stage 1
    template <class S = CtaSync>
    static __device__ __forceinline__ void fft_pre(C *buf, const C *__restrict__ tw, const T *__restrict__ sn, int t) {
        constexpr int N1 = P::R0, N2 = N1 * P::R1, N3 = N2 * P::R2, N4 = N3 * P::R3;
        static_assert(N4 * P::R4 == M, "plan must factor M");
        stage_first_pre<M, P::R0, TPF, C, T, S>(buf, sn, t);
        stage_ct<M, P::R1, N1, TPF, C, S>(buf, tw, t);
        stage_ct<M, P::R2, N2, TPF, C, S>(buf, tw, t);
        if constexpr (P::R3 > 1) stage_ct<M, P::R3, N3, TPF, C, S>(buf, tw, t);
        if constexpr (P::R4 > 1) stage_ct<M, P::R4, N4, TPF, C, S>(buf, tw, t);
    }

    template <class S = CtaSync>
    static __device__ __forceinline__ void dst(C *buf, const PlanT<T> &pl, int t, double2 *wt) {
        fft_pre<S>(buf, pl.tw, pl.sn, t);
        post<S>(buf, t, wt);
    }
};

// Compile-time transforms for lengths with a factor 3 (M = 384 = 3 x 8 x 16):
// the general stages above, Pow2Dst's scan post-processing.
template <int M>
struct MixPlan;
template <>
struct MixPlan<384> : PlanCT<64, 3, 8, 16> {};

template <int M, class T, class PL = MixPlan<M>>
struct MixDst : Pow2Dst<M, T, PL> {
    using Base = Pow2Dst<M, T, PL>;
    using C = typename Base::C;
    using P = PL;
    static constexpr int TPF = P::TPF;
    template <class S = CtaSync>
    static __device__ __forceinline__ void fft_pre(C *buf, const C *__restrict__ tw, const T *__restrict__ sn, int t) {
        constexpr int N1 = P::R0, N2 = N1 * P::R1, N3 = N2 * P::R2, N4 = N3 * P::R3;
        static_assert(N4 * P::R4 == M, "plan must factor M");
        stage_gen_first_pre<M, P::R0, TPF, C, T, S>(buf, sn, t);
        stage_gen<M, P::R1, N1, TPF, C, S>(buf, tw, t);
        stage_gen<M, P::R2, N2, TPF, C, S>(buf, tw, t);
        if constexpr (P::R3 > 1) stage_gen<M, P::R3, N3, TPF, C, S>(buf, tw, t);
        if constexpr (P::R4 > 1) stage_gen<M, P::R4, N4, TPF, C, S>(buf, tw, t);
    }
    template <class S = CtaSync>
    static __device__ __forceinline__ void dst(C *buf, const PlanT<T> &pl, int t, double2 *wt) {
        fft_pre<S>(buf, pl.tw, pl.sn, t);
        Base::template post<S>(buf, t, wt);
    }
};

// The runtime mixed-radix transform behind the same interface (any even M <= 1024
// of the form 2^a 3^b 5^c), unpadded.
template <class T>
struct GenericDst {
    static constexpr int OCC = 512;
    static constexpr int MC = 0;  // transform length known only at run time
    using Real = T;
    using C = typename Cx<T>::type;
    static constexpr int TPF = kTPF;
    static constexpr int NWARP = kTPF / 32;
    static __host__ __device__ constexpr int smem_len(int m) { return m + 1; }
    static __device__ __forceinline__ int idx(int i) { return i; }
    static __device__ __forceinline__ void dst(C *buf, const PlanT<T> &pl, int t, double2 *wt) {
        dst_inplace<T>(buf, pl, t, wt);
    }
};

}  // namespace ibpm
