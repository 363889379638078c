// noalloc.cu -- ibpm_lap_inv_noalloc: the Laplacian-inverse solve
// (Δinv_operator, src/fluid.jl:117-119 and 145-166) for callers that cannot
// allocate device memory.
//
// Some callers cannot call cudaMalloc at all: code running inside another
// framework's memory pool or a pre-sized arena, or a host loop that must not
// allocate between steps.  They pass device pointers for the right-hand side and
// the result; everything else this solve needs -- two scratch fields and the
// transform tables -- lives in the file-scope array `g_scratch` below, a fixed
// block of device memory that every GPU loading the library holds until the
// process exits.  No cudaMalloc, cudaFree or allocating library routine is
// called here.
//
// Limits and behaviour:
//  * (nx-1)(ny-1) <= kNoAllocMaxCells (2^18 = 262144 cells, e.g. 512 x 512) and
//    nx, ny even, <= 1024, of the form 2^a 3^b 5^c; larger sizes are rejected.
//  * The first call on a device (and any call whose nx/ny differ from that
//    device's previous call) writes the transform tables into g_scratch; make
//    that first call before any stream capture.  Such a call made while the
//    stream is capturing is rejected (IBPM_ERR_INVALID): its table kernels would
//    only enter the graph, and later eager calls would read unwritten tables.
//  * b and x may be the same buffer: the first pass reads b into scratch and
//    only the last pass writes x, in stream order.
//  * Errors are read from each launch's own return code (cudaLaunchKernelEx), so
//    an error left pending by an unrelated earlier launch is not reported as
//    this call's failure.
//  * Every call shares g_scratch, which keeps the last call's contents: calls
//    that overlap on the GPU (different streams, or other host threads) race.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "../../include/ibpm_b200.h"
#include "kernels.cuh"

using namespace ibpm;

namespace {

constexpr long long kNoAllocMaxCells = 1LL << 18;
constexpr int kNoAllocMaxM = 1024;
// field scratch (2 fields) + twiddles and sine/cosine tables for x and y
constexpr size_t kScratchDoubles = 2 * kNoAllocMaxCells + 2 * (2 * kNoAllocMaxM) + 4 * (kNoAllocMaxM + 1);

static __device__ __align__(256) double g_scratch[kScratchDoubles];

struct DeviceSlot {
    double *base = nullptr;  // device address of g_scratch on this device
    int nx = 0, ny = 0;      // sizes the tables were written for
};
constexpr int kMaxDevices = 64;
DeviceSlot g_slots[kMaxDevices];
std::mutex g_mu;
thread_local char g_err[256];

int fail(int code, const char *msg) {
    strncpy(g_err, msg, sizeof g_err - 1);
    g_err[sizeof g_err - 1] = 0;
    return code;
}

__global__ void noalloc_tables_kernel(double2 *tw, double *sn, double *cs, int M) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k <= M; k += gridDim.x * blockDim.x) {
        if (k < M) {
            double s, c;
            sincospi(-2.0 * k / M, &s, &c);
            tw[k] = make_double2(c, s);
        }
        sn[k] = sinpi((double)k / M);
        cs[k] = cospi((double)k / M);
    }
}

bool plan_ok(int M, PlanT<double> &pl) {
    if (M < 8 || M > kNoAllocMaxM || (M & 1)) return false;
    pl.M = M;
    pl.nst = 0;
    int m = M;
    const int rs[4] = {4, 2, 3, 5};
    for (int r : rs)
        while (m % r == 0) {
            if (pl.nst >= kMaxStages) return false;
            pl.radix[pl.nst++] = r;
            m /= r;
        }
    if (m != 1) return false;
    for (int s = 0; s < pl.nst; ++s) {
        const int K = (M / pl.radix[s] + kTPF - 1) / kTPF;
        if (K * pl.radix[s] > kMaxV) return false;
    }
    return (M / 2 + kTPF - 1) / kTPF <= kMaxE;
}

// Launches return their own error code (cudaLaunchKernelEx, whose template
// form checks the arguments against the kernel's parameters).
inline cudaLaunchConfig_t launch_cfg(dim3 grid, dim3 block, size_t smem, cudaStream_t st) {
    cudaLaunchConfig_t c{};
    c.gridDim = grid;
    c.blockDim = block;
    c.dynamicSmemBytes = smem;
    c.stream = st;
    c.attrs = nullptr;
    c.numAttrs = 0;
    return c;
}

template <class D, class In, class Out>
cudaError_t xpass_na(const PlanT<double> &pl, In in, Out out, int nrows, cudaStream_t st) {
    constexpr int NG = 2;
    const cudaLaunchConfig_t c =
        launch_cfg(dim3(((nrows + 1) / 2 + NG - 1) / NG, 1), dim3(NG * D::TPF), pass_smem<D>(pl.M, NG, NG), st);
    return cudaLaunchKernelEx(&c, xpass_kernel<D, NG, In, Out>, in, out, pl, nrows, (const int *)nullptr, 0, 0);
}

template <class D>
cudaError_t ypass_na(const PlanT<double> &pl, const double *in, double *out, int ncols, Mult m, cudaStream_t st) {
    constexpr int NG = 2;
    const cudaLaunchConfig_t c =
        launch_cfg(dim3((ncols + 2 * NG - 1) / (2 * NG), 1), dim3(NG * D::TPF), pass_smem<D>(pl.M, NG, NG), st);
    return cudaLaunchKernelEx(&c, ypass_kernel<D, NG>, in, out, 0LL, ncols, pl, m);
}

cudaError_t tables_na(double2 *tw, double *sn, double *cs, int M, cudaStream_t st) {
    const cudaLaunchConfig_t c = launch_cfg(dim3(8), dim3(128), 0, st);
    return cudaLaunchKernelEx(&c, noalloc_tables_kernel, tw, sn, cs, M);
}

}  // namespace

extern "C" {

/* Declared in include/ibpm_b200.h. */
int ibpm_lap_inv_noalloc(int nx, int ny, const double *b, double *x, void *stream) {
    if (!b || !x) return fail(IBPM_ERR_INVALID, "null field pointer");
    PlanT<double> plx{}, ply{};
    if (!plan_ok(nx, plx) || !plan_ok(ny, ply))
        return fail(IBPM_ERR_INVALID, "nx and ny must be even, 8..1024, of the form 2^a 3^b 5^c");
    const long long ng = (long long)(nx - 1) * (ny - 1);
    if (ng > kNoAllocMaxCells) return fail(IBPM_ERR_INVALID, "(nx-1)(ny-1) exceeds the no-alloc limit of 262144 cells");
    cudaStream_t st = (cudaStream_t)stream;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return fail(IBPM_ERR_CUDA, "no CUDA device");
    double *base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        DeviceSlot &slot = g_slots[dev];
        if (!slot.base) {
            void *p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
            if (e != cudaSuccess) return fail(IBPM_ERR_CUDA, cudaGetErrorString(e));
            slot.base = static_cast<double *>(p);
        }
        base = slot.base;
        double *tab = base + 2 * kNoAllocMaxCells;
        double2 *twx = reinterpret_cast<double2 *>(tab), *twy = reinterpret_cast<double2 *>(tab + 2 * kNoAllocMaxM);
        double *snx = tab + 4 * kNoAllocMaxM, *sny = snx + (kNoAllocMaxM + 1);
        double *csx = sny + (kNoAllocMaxM + 1), *csy = csx + (kNoAllocMaxM + 1);
        if (slot.nx != nx || slot.ny != ny) {
            cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
            cudaError_t e = cudaStreamIsCapturing(st, &cs);
            if (e != cudaSuccess) return fail(IBPM_ERR_CUDA, cudaGetErrorString(e));
            if (cs != cudaStreamCaptureStatusNone)
                return fail(IBPM_ERR_INVALID,
                            "the transform tables for this size are not written yet: make the first call for these "
                            "nx, ny on this device outside stream capture");
            e = tables_na(twx, snx, csx, nx, st);
            if (e == cudaSuccess) e = tables_na(twy, sny, csy, ny, st);
            if (e != cudaSuccess) return fail(IBPM_ERR_CUDA, cudaGetErrorString(e));
            slot.nx = nx;
            slot.ny = ny;
        }
    }
    double *t1 = base, *t2 = base + kNoAllocMaxCells;
    double *tab = base + 2 * kNoAllocMaxCells;
    plx.tw = reinterpret_cast<const double2 *>(tab);
    ply.tw = reinterpret_cast<const double2 *>(tab + 2 * kNoAllocMaxM);
    plx.sn = tab + 4 * kNoAllocMaxM;
    ply.sn = plx.sn + (kNoAllocMaxM + 1);
    Mult m{};
    m.mode = MULT_LAPINV;
    m.cx = ply.sn + (kNoAllocMaxM + 1);
    m.cy = m.cx + (kNoAllocMaxM + 1);
    m.scale = 1.0 / (double)(4 * (long long)nx * (long long)ny);
    m.h = 1.0;
    m.Re = 1.0;
    m.dt = 0.0;
    m.lev0 = 1;
    m.levstep = 0;
    using D = GenericDst<double>;
    cudaError_t e = xpass_na<D>(plx, InPlain<double>{b, 0, nx - 1}, OutPlain<double>{t1, 0, nx - 1}, ny - 1, st);
    if (e == cudaSuccess) e = ypass_na<D>(ply, t1, t2, nx - 1, m, st);
    if (e == cudaSuccess)
        e = xpass_na<D>(plx, InPlain<double>{t2, 0, nx - 1}, OutPlain<double>{x, 0, nx - 1}, ny - 1, st);
    if (e != cudaSuccess) return fail(IBPM_ERR_CUDA, cudaGetErrorString(e));
    return IBPM_OK;
}

const char *ibpm_noalloc_last_error(void) { return g_err; }

}  // extern "C"
