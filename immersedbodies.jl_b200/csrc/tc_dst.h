// Batched 2D DST-I solves on the tensor cores (tcgen05, BF16 operands, FP32
// accumulation in tensor memory), for the B assembly of the preconditioned
// moving-body modes, where B^-1 serves as a preconditioner and need not be exact.
//
// A solve x = S(m ⊙ S(b)) of one P x P field (P = nx = ny, the (P-1)^2 interior
// padded by a zero row and column) is four passes of the same dense product
//     D[f][k][l] = sum_p S[k][p] X[f][l][p]
// with S[k][p] = 2 sin(pi (k+1)(p+1) / P) (FFTW's RODFT00, the reference's
// transform at src/fluid.jl:113-115) as the A operand and the batch's lines as
// the B operand.  Each pass transforms along one axis and writes its result as
// the next pass's lines: (y, x) -> (kx, y) -> (ky, kx) with the spectral
// multiplier applied -> (x, ky) -> (y, x) in FP64.  Operands are BF16: one
// product S_hi X_hi, or the split form S_hi X_hi + S_hi X_lo + S_lo X_hi with
// v = hi + lo, lo = bf16(v - hi) (about 16 significant bits per operand).
#pragma once
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

struct TcDstPlan;

// P in {256, 512, 1024}; fmax fields per call; nprod 1 (BF16) or 3 (split BF16).
// Allocates the transform matrices, two line buffers (hi and lo parts) and the
// TMA descriptors on the current device.  Returns nullptr (and sets *why) when
// the device or sizes are unsupported.
TcDstPlan *tc_create(int P, int fmax, int nprod, const char **why);
void tc_destroy(TcDstPlan *p);
int tc_P(const TcDstPlan *p);
int tc_nprod(const TcDstPlan *p);
int tc_fmax(const TcDstPlan *p);
// the buffer the first pass reads: [f][line y][position x], P x P per field
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
// tc_in_hi / tc_in_lo; mult (device, P x P floats, [ky][kx]) is applied after
// the second pass; the result goes to out[f * bs + x + ld * y] for x, y < P - 1
// that `keep` selects.  *err (device) is set to 1 if a wait inside a pass gave
// up (after one second; never in normal use).  Returns the number of kernels
// launched.
int tc_solve_tail(TcDstPlan *p, int nf, const float *mult, double *out, long long bs, int ld, TcKeep keep,
                  int *err, cudaStream_t st);

// Splits v into hi = bf16(v), lo = bf16(v - hi).
__device__ __forceinline__ void tc_split(float v, __nv_bfloat16 &hi, __nv_bfloat16 &lo) {
    hi = __float2bfloat16_rn(v);
    lo = __float2bfloat16_rn(v - __bfloat162float(hi));
}

// The first pass's lines from a solve prologue `in` (in(f, i, j): the value at
// x = i - 1, y = j - 1 of field f, 1 <= i, j <= P - 1): line y of field f holds
// positions x = 0 .. P - 1, zero in the padding.  Block: P / 8 threads, 8
// positions each; grid (1, P, nf).
template <class In>
__global__ void tc_lines_kernel(In in, int P, __nv_bfloat16 *hi, __nv_bfloat16 *lo) {
    const int f = blockIdx.z, y = blockIdx.y, x0 = threadIdx.x * 8;
    __align__(16) __nv_bfloat16 h[8];
    __align__(16) __nv_bfloat16 l[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int x = x0 + j;
        const double v = (x < P - 1 && y < P - 1) ? in(f, x + 1, y + 1) : 0.0;
        h[j] = __double2bfloat16(v);
        l[j] = __double2bfloat16(v - (double)__bfloat162float(h[j]));
    }
    const size_t off = ((size_t)f * P + y) * P + x0;
    *reinterpret_cast<uint4 *>(hi + off) = *reinterpret_cast<const uint4 *>(h);
    if (lo) *reinterpret_cast<uint4 *>(lo + off) = *reinterpret_cast<const uint4 *>(l);
}
