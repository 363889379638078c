// Batched 2D DST-I solves on the tensor cores (tcgen05, BF16 operands, FP32
// accumulation in tensor memory), for the B assembly of the preconditioned
// moving-body modes, where B^-1 serves as a preconditioner and need not be exact.
//
// A solve x = S(m ⊙ S(b)) of one P x P field (P = nx = ny, the (P-1)^2 interior)
// is four passes of one dense product per line, y_k = sum_j S[k][j] x_j with
// S[k][j] = 2 sin(pi k j / P) (FFTW's RODFT00, the reference's transform at
// src/fluid.jl:113-115).  Since S[k][P-j] = (-1)^(k+1) S[k][j], odd k need only
// u_j = x_j + x_(P-j) and even k only v_j = x_j - x_(P-j) (j < P/2; u_(P/2) =
// x_(P/2)): two products of half the length, half the work of the full one.
//
// Storage.  A line is held in "uv form": P BF16 values, u in slots [0, P/2) and
// v in [P/2, P); slot s (s' = s mod P/2) holds the pair (j, P - j) with j =
// tc_uvj(s').  Lines are held in "block order": storage index l is physical
// index tc_blk(l) (odd indices first, then the even ones arranged so that l and
// P/2 - 1 - l, or P - 1 - (l - P/2) in the second half, are mirror pairs j,
// P - j; one padding slot).  Pass p transforms the lines of its input along
// their positions: output row r (frequency tc_blk(r)) of the lines of one field
// becomes line r of pass p + 1, whose positions are pass p's lines:
//   (y, x) -> (kx, y) -> (ky, kx) [x m] -> (x, ky) -> (y, x) in FP64.
// Operands are BF16: one product S_hi X_hi, or the split form S_hi X_hi +
// S_hi X_lo + S_lo X_hi with v = hi + lo, lo = bf16(v - hi) (about 16
// significant bits per operand).
#pragma once
#include <cstdint>
#include <type_traits>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

struct TcDstPlan;

// Physical index (1 .. P-1; 0 for the padding slot) of storage index i in block order.
__host__ __device__ __forceinline__ int tc_blk(int i, int P) {
    if (i < P / 2) return 2 * i + 1;
    const int c = i - P / 2;
    if (c < P / 4) return 2 * (c + 1);
    if (c == P / 4) return 0;
    return 2 * c;
}
// Physical index j (1 .. P/2) of the pair (j, P - j) held in uv slot s' (0 .. P/2 - 1).
__host__ __device__ __forceinline__ int tc_uvj(int s, int P) {
    return s < P / 4 ? 2 * s + 1 : 2 * (s - P / 4 + 1);
}

// P in {256, 512}; fmax fields per call; nprod 1 (BF16) or 3 (split BF16).
// Allocates the transform matrices, two line buffers (hi and lo parts) and the
// TMA descriptors on the current device.  Returns nullptr (and sets *why) when
// the device or sizes are unsupported.
TcDstPlan *tc_create(int P, int fmax, int nprod, const char **why);
void tc_destroy(TcDstPlan *p);
int tc_P(const TcDstPlan *p);
int tc_nprod(const TcDstPlan *p);
int tc_fmax(const TcDstPlan *p);
// the buffer the first pass reads: lines y (block order) of positions x (uv form)
__nv_bfloat16 *tc_in_hi(TcDstPlan *p);
__nv_bfloat16 *tc_in_lo(TcDstPlan *p);
// Which elements of the result a solve stores: all; those a windowed curl
// reads (win: device [i0, i1, j0, j1], 1-based face indices; the psi entries
// (i - 1 .. i, j - 1 .. j) of every face in it); or the four lines a finer
// level's boundary values read (lines: 0-based rows y0, y1 and columns x0, x1).
enum { TC_KEEP_ALL = 0, TC_KEEP_WINDOW = 1, TC_KEEP_LINES = 2 };
struct TcKeep {
    int mode;
    const int *win;
    int lines[4];
};

// Runs the four passes over nf fields whose lines the caller wrote to
// tc_in_hi / tc_in_lo; mult (device, P x P floats, [kx storage][ky storage],
// both in block order: read coalesced by the rows ky of a tile) is applied
// after the second pass; the result goes to out[f * bs + x + ld * y] for the x,
// y < P - 1 that `keep` selects.  *err (device) is set to 1 if a wait inside a
// pass gave up (after one second; never in normal use).  Returns the number of
// kernels launched.
int tc_solve_tail(TcDstPlan *p, int nf, const float *mult, double *out, long long bs, int ld, TcKeep keep,
                  int *err, cudaStream_t st);

// Splits v into hi = bf16(v), lo = bf16(v - hi).
__device__ __forceinline__ void tc_split(float v, __nv_bfloat16 &hi, __nv_bfloat16 &lo) {
    hi = __float2bfloat16_rn(v);
    lo = __float2bfloat16_rn(v - __bfloat162float(hi));
}

// The first pass's lines from a solve prologue `in` (in(f, i, j): the value at
// 1-based (i, j) of field f, 1 <= i, j <= P - 1): line l of field f is physical
// row y = tc_blk(l) in uv form (zero for the padding line).  The row is read
// once, coalesced, into shared memory (P doubles); thread t then forms slots t,
// t + P/8, ... (neighbouring threads read neighbouring pairs).  Block: P / 8
// threads; grid (1, P, nf); P * 8 bytes of shared memory.
// A prologue with kSplitRing = true offers plain(f, i, j), the field alone, and
// ring(v, f, i, j), v plus its boundary values on the outer ring (in the same
// order as its operator()); the row is then loaded plainly first and the few
// ring elements completed after, so no load of the row waits behind the
// boundary reads.
template <class In, class = void>
struct TcSplitRing {
    static constexpr bool value = false;
};
template <class In>
struct TcSplitRing<In, std::void_t<decltype(In::kSplitRing)>> {
    static constexpr bool value = In::kSplitRing;
};

template <class In>
__global__ void tc_lines_kernel(In in, int P, __nv_bfloat16 *hi, __nv_bfloat16 *lo) {
    extern __shared__ double tc_row[];
    const int f = blockIdx.z, l = blockIdx.y, t = threadIdx.x, nt = blockDim.x;
    const int y = tc_blk(l, P);
    if constexpr (TcSplitRing<In>::value) {
        for (int x = t + 1; x < P; x += nt) tc_row[x] = y != 0 ? in.plain(f, x, y) : 0.0;
        __syncthreads();
        if (y != 0) {
            if (in.ring_row(y)) {
                for (int x = t + 1; x < P; x += nt) tc_row[x] = in.ring(tc_row[x], f, x, y);
            } else if (t < 2) {
                const int x = t == 0 ? 1 : P - 1;
                tc_row[x] = in.ring(tc_row[x], f, x, y);
            }
        }
    } else {
        for (int x = t + 1; x < P; x += nt) tc_row[x] = y != 0 ? in(f, x, y) : 0.0;
    }
    __syncthreads();
    const size_t off = ((size_t)f * P + l) * P;
    for (int s = t; s < P; s += nt) {
        const int half = s >= P / 2;
        const int x = tc_uvj(half ? s - P / 2 : s, P);
        const double a = tc_row[x], b = x == P / 2 ? 0.0 : tc_row[P - x];
        const double v = half ? (x == P / 2 ? 0.0 : a - b) : a + b;
        const __nv_bfloat16 h = __double2bfloat16(v);
        hi[off + s] = h;
        if (lo) lo[off + s] = __double2bfloat16(v - (double)__bfloat162float(h));
    }
}
