// ibpm.cu -- libibpm_b200: the FP64 CNAB/IBPM time step on one B200, behind
// the C ABI of include/ibpm_b200.h.
//
// Device state per handle (column-major, the reference's State layout):
//   q (nq x L), psi (ng x L), Gamma[2] (ng x L, ping-pong: state.Γ and the
//   trial Γs of the running step), nonlin[2] (ng x L, swapped per step like
//   _cycle!), panels, F~b, fb.  q0 is never stored on the hot path: every
//   consumer evaluates base_flux! per face; it is materialised only for
//   ibpm_get_state.
// One step (advance!, src/solver.jl:155-190) is ~60 kernels on one stream;
// each 2D DST solve is three line passes (see fft_dst.cuh).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ibpm_b200.h"
#include "coupling.h"
#include "kernels.cuh"

using namespace ibpm;

namespace {

constexpr int kNG = 2;  // FFT groups (line pairs) per block

thread_local std::string g_create_error;

struct CudaError {
    cudaError_t e;
    const char *where;
};

#define CK(call)                                                   \
    do {                                                           \
        cudaError_t _e = (call);                                   \
        if (_e != cudaSuccess) throw CudaError{_e, #call};         \
    } while (0)

struct ApiError {
    int code;
    std::string msg;
};

bool make_plan(int M, Plan &pl) {
    if (M < 4 || M > kMaxM || (M & 1)) return false;
    pl.M = M;
    pl.nst = 0;
    int m = M;
    auto push = [&](int r) {
        if (pl.nst >= kMaxStages) return false;
        pl.radix[pl.nst++] = r;
        return true;
    };
    while (m % 4 == 0) {
        if (!push(4)) return false;
        m /= 4;
    }
    while (m % 2 == 0) {
        if (!push(2)) return false;
        m /= 2;
    }
    while (m % 3 == 0) {
        if (!push(3)) return false;
        m /= 3;
    }
    while (m % 5 == 0) {
        if (!push(5)) return false;
        m /= 5;
    }
    if (m != 1) return false;
    for (int s = 0; s < pl.nst; ++s) {
        const int R = pl.radix[s];
        const int nb = M / R;
        const int K = (nb + kTPF - 1) / kTPF;
        if (K * R > kMaxV) return false;
    }
    return (M / 2 + kTPF - 1) / kTPF <= kMaxE;
}

}  // namespace

struct ibpm_handle {
    // problem
    Grid g{};
    int nx = 0, ny = 0, L = 0, np = 0, nbody = 0;
    long long nq = 0, ng = 0, nu = 0, nbc = 0;
    std::vector<int> body_kind, body_start;
    std::vector<double> ref_xb, ref_ds;
    bool static_bodies = true;
    ibpm_options opt{};
    int device = 0;
    cudaStream_t st = nullptr;
    // transforms
    Plan plx{}, ply{};
    double2 *twx = nullptr, *twy = nullptr;
    double *snx = nullptr, *sny = nullptr, *cx = nullptr, *cy = nullptr;
    // state
    int64_t index = 0;
    double t0 = 0.0;
    double *q = nullptr, *psi = nullptr, *G[2] = {nullptr, nullptr}, *nl[2] = {nullptr, nullptr};
    int gc = 0;  // state.Γ = G[gc]
    int nc = 0;  // state.nonlin[1] = nl[nc], state.nonlin[2] = nl[1 - nc]
    double *q0mat = nullptr;
    bool q0_from_user = false;
    bool q0_zero = true;  // State(prob) starts with q0 = 0 until the first step
    Panels P{};
    double *ref_xb_d = nullptr, *ds = nullptr;
    double *Fbt = nullptr, *fb = nullptr, *total = nullptr;
    StepDev *prm = nullptr, *prm_h = nullptr;
    double *motion = nullptr, *motion_h = nullptr;
    double fs_last[2] = {0, 0}, gm_last[6] = {0, 0, 0, 0, 0, 0};
    // work
    int kbatch = 1;  // columns per batch in the B setup
    double *t1 = nullptr, *t2 = nullptr, *rhs = nullptr, *rest = nullptr, *qs1 = nullptr, *Ftmp = nullptr;
    double *part = nullptr;
    double *patch = nullptr;
    long long patch_stride = 0;
    double *Gw = nullptr, *psiw = nullptr, *qw = nullptr, *fcol = nullptr;  // batch work (K columns)
    double *Binv = nullptr, *rowk = nullptr, *colk = nullptr;
    double *cg_u = nullptr, *cg_r = nullptr, *cg_c = nullptr, *cg_s = nullptr, *cg_s_h = nullptr;
    int *err = nullptr, *err_h = nullptr;
    int last_cg_iters = 0;
    double last_cg_res = 0.0;
    long long launches = 0;
    long long dev_bytes = 0;
    // kernel timing (ibpm_profile)
    bool prof = false;
    struct ProfRec {
        int cls;
        int ev;
        double bytes;
    };
    std::vector<ProfRec> prof_recs;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_next = 0;
    int prof_begin() {
        if (!prof) return -1;
        if (ev_next + 2 > ev_pool.size()) {
            for (int k = 0; k < 64; ++k) {
                cudaEvent_t e;
                CK(cudaEventCreate(&e));
                ev_pool.push_back(e);
            }
        }
        const int i = (int)ev_next;
        ev_next += 2;
        CK(cudaEventRecord(ev_pool[i], st));
        return i;
    }
    void prof_end(int i, int cls, double bytes) {
        if (i < 0) return;
        CK(cudaEventRecord(ev_pool[i + 1], st));
        prof_recs.push_back(ProfRec{cls, i, bytes});
    }
    std::vector<void *> allocs;
    std::string last_error;

    template <class T>
    T *dalloc(size_t n) {
        void *p = nullptr;
        if (n == 0) n = 1;
        cudaError_t e = cudaMalloc(&p, n * sizeof(T));
        if (e != cudaSuccess) throw ApiError{IBPM_ERR_NOMEM, "cudaMalloc of " + std::to_string(n * sizeof(T)) + " bytes failed"};
        allocs.push_back(p);
        dev_bytes += (long long)(n * sizeof(T));
        CK(cudaMemsetAsync(p, 0, n * sizeof(T), st));
        return static_cast<T *>(p);
    }
    ~ibpm_handle() {
        if (st) cudaStreamSynchronize(st);
        for (int p = 0; p < 2; ++p) {
            if (graph_exec[p]) cudaGraphExecDestroy(graph_exec[p]);
            if (graph[p]) cudaGraphDestroy(graph[p]);
        }
        for (cudaEvent_t e : ev_pool) cudaEventDestroy(e);
        for (void *p : allocs) cudaFree(p);
        if (prm_h) cudaFreeHost(prm_h);
        if (motion_h) cudaFreeHost(motion_h);
        if (cg_s_h) cudaFreeHost(cg_s_h);
        if (err_h) cudaFreeHost(err_h);
        if (st) cudaStreamDestroy(st);
    }

    void check_launch() {
        ++launches;
        CK(cudaGetLastError());
    }

    // ---- line passes ----
    // Dispatch on the transform length: compile-time power-of-two transforms
    // for M in {128, 256, 512, 1024}, the runtime mixed-radix one otherwise.
    template <class D, class In, class Out>
    void xpass_t(In in, Out out, int nbatch) {
        const int pairs = (ny - 1 + 1) / 2;
        const dim3 grid((pairs + kNG - 1) / kNG, nbatch);
        const size_t sm = (size_t)(kNG * D::smem_len(plx.M) + D::NWARP * kNG) * sizeof(double2);
        xpass_kernel<D, kNG, In, Out><<<grid, kNG * D::TPF, sm, st>>>(in, out, plx, ny - 1);
    }
    template <class In, class Out>
    void xpass(In in, Out out, int nbatch) {
        const int pe = prof_begin();
        switch (plx.M) {
            case 1024: xpass_t<Pow2Dst<1024>>(in, out, nbatch); break;
            case 512: xpass_t<Pow2Dst<512>>(in, out, nbatch); break;
            case 256: xpass_t<Pow2Dst<256>>(in, out, nbatch); break;
            default: xpass_t<GenericDst>(in, out, nbatch); break;
        }
        check_launch();
        prof_end(pe, IBPM_KCLASS_XPASS, 16.0 * (double)ng * nbatch);
    }
    template <class D>
    void ypass_t(const double *in, double *out, long long bs, int nbatch, Mult m) {
        const dim3 grid((nx - 1 + 2 * kNG - 1) / (2 * kNG), nbatch);
        const size_t sm = (size_t)(kNG * D::smem_len(ply.M) + D::NWARP * kNG) * sizeof(double2);
        ypass_kernel<D, kNG><<<grid, kNG * D::TPF, sm, st>>>(in, out, bs, nx - 1, ply, m);
    }
    void ypass(const double *in, double *out, long long bs, int nbatch, Mult m) {
        const int pe = prof_begin();
        switch (ply.M) {
            case 1024: ypass_t<Pow2Dst<1024>>(in, out, bs, nbatch, m); break;
            case 512: ypass_t<Pow2Dst<512>>(in, out, bs, nbatch, m); break;
            case 256: ypass_t<Pow2Dst<256>>(in, out, bs, nbatch, m); break;
            default: ypass_t<GenericDst>(in, out, bs, nbatch, m); break;
        }
        check_launch();
        prof_end(pe, IBPM_KCLASS_YPASS, 16.0 * (double)ng * nbatch);
    }
    // Merged trial solve over all L levels: Gamma_new = Ainv(A Gamma + rest)
    template <class D>
    void trial_t(const double *Gold, const double *rest_, double *Gnew) {
        {
            const dim3 grid((ny - 1 + kNG - 1) / kNG, L);
            const size_t sm = (size_t)(kNG * D::smem_len(plx.M) + D::NWARP * kNG) * sizeof(double2);
            const int pe = prof_begin();
            xpass_trial_kernel<D, kNG><<<grid, kNG * D::TPF, sm, st>>>(Gold, rest_, t1, t2, ng, nx - 1, plx, ny - 1);
            check_launch();
            prof_end(pe, IBPM_KCLASS_XPASS, 32.0 * (double)ng * L);
        }
        {
            const dim3 grid((nx - 1 + 2 * kNG - 1) / (2 * kNG), L);
            const size_t sm = (size_t)(2 * kNG * D::smem_len(ply.M) + D::NWARP * kNG) * sizeof(double2);
            // the cap must cover the largest M this instantiation serves (kMaxM)
            static bool attr = false;
            if (!attr) {
                const int cap = (int)((2 * kNG * D::smem_len(kMaxM) + D::NWARP * kNG) * sizeof(double2));
                CK(cudaFuncSetAttribute(ypass_trial_kernel<D, kNG>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap));
                attr = true;
            }
            const int pe = prof_begin();
            ypass_trial_kernel<D, kNG><<<grid, kNG * D::TPF, sm, st>>>(t1, t2, rhs, ng, nx - 1, ply,
                                                                       mult(MULT_AIMPL, 1, 1));
            check_launch();
            prof_end(pe, IBPM_KCLASS_YPASS, 24.0 * (double)ng * L);
        }
        xpass(in_plain(rhs, ng), out_plain(Gnew, ng), L);
    }
    void trial(const double *Gold, const double *rest_, double *Gnew) {
        if (plx.M == 1024 && ply.M == 1024)
            trial_t<Pow2Dst<1024>>(Gold, rest_, Gnew);
        else if (plx.M == 512 && ply.M == 512)
            trial_t<Pow2Dst<512>>(Gold, rest_, Gnew);
        else if (plx.M == 256 && ply.M == 256)
            trial_t<Pow2Dst<256>>(Gold, rest_, Gnew);
        else
            trial_t<GenericDst>(Gold, rest_, Gnew);
    }

    Mult mult(int mode, int lev0, int levstep) const {
        Mult m;
        m.mode = mode;
        m.cx = cx;
        m.cy = cy;
        m.scale = 1.0 / (double)(4 * (long long)nx * (long long)ny);
        m.h = g.h;
        m.Re = g.Re;
        m.dt = g.dt;
        m.lev0 = lev0;
        m.levstep = levstep;
        return m;
    }
    InPlain in_plain(const double *p, long long bs) const { return InPlain{p, bs, nx - 1}; }
    OutPlain out_plain(double *p, long long bs) const { return OutPlain{p, bs, nx - 1}; }

    // vort2flux (src/fluid.jl:178-205) over nbatch independent fields.
    // G, psi: level 1 of batch 0, level stride ng, batch stride bs.
    // qout: level 1 of batch 0 (level stride nq, batch stride qbs); curl_all=false
    // computes q only at level 1 (the only level a caller reads).
    void vort2flux(double *psi_, double *qout, double *Gm, long long bs, long long qbs, int nbatch, bool curl_all) {
        for (int lev = 2; lev <= L; ++lev) {
            const int nx2 = nx / 2, ny2 = ny / 2;
            const dim3 blk(16, 16), grd((nx2 + 15) / 16, (ny2 + 15) / 16, nbatch);
            coarsify_kernel<<<grd, blk, 0, st>>>(Gm + (lev - 1) * ng, Gm + (lev - 2) * ng, bs, g);
            check_launch();
        }
        for (int lev = L; lev >= 1; --lev) {
            double *Gl = Gm + (lev - 1) * ng;
            double *Pl = psi_ + (lev - 1) * ng;
            if (lev == L)
                xpass(in_plain(Gl, bs), out_plain(t1, ng), nbatch);
            else
                xpass(InBC{Gl, psi_ + lev * ng, bs, bs, g}, out_plain(t1, ng), nbatch);
            ypass(t1, t2, ng, nbatch, mult(MULT_LAPINV, 1, 0));
            xpass(in_plain(t2, ng), out_plain(Pl, bs), nbatch);
            if (curl_all || lev == 1) {
                const dim3 blk(64, 4);
                const dim3 grd((nx + 1 + 63) / 64, (ny + 3) / 4 + (ny + 1 + 3) / 4, nbatch);
                const int pe = prof_begin();
                curl_kernel<<<grd, blk, 0, st>>>(qout + (lev - 1) * nq, qbs, Pl, bs, lev < L ? psi_ + lev * ng : nullptr,
                                                 bs, g);
                check_launch();
                prof_end(pe, IBPM_KCLASS_CURL, 8.0 * (double)(ng + nq) * nbatch);
            }
        }
    }

    // Regularisation patch of nbatch force vectors f (stride 2np).
    void reg_patch(const double *f, int nbatch) {
        launch_reg_patch(P, f, 2 * np, patch, patch_stride, nbatch, g, st);
        check_launch();
    }

    // B z (src/coupling.jl:163-176) for nbatch vectors z (stride 2np) into x (stride xs).
    void apply_B(const double *z, double *x, long long xs, int nbatch) {
        reg_patch(z, nbatch);
        InRegRot in{Patch{patch, P.bbox, patch_stride}};
        xpass(in, out_plain(t1, ng), nbatch);
        ypass(t1, t2, ng, nbatch, mult(MULT_AIMPL, 1, 0));
        xpass(in_plain(t2, ng), out_plain(Gw, ng * L), nbatch);
        if (L > 1)
            CK(cudaMemset2DAsync(Gw + ng, (size_t)(ng * L) * sizeof(double), 0, (size_t)(ng * (L - 1)) * sizeof(double),
                                 nbatch, st));
        vort2flux(psiw, qw, Gw, ng * L, nq, nbatch, false);
        launch_regT(P, qw, nq, x, xs, nbatch, 0, prm, g, st);
        check_launch();
    }

    void update_weights(int p0, int p1) {
        if (p1 <= p0) return;
        launch_reg_weights(P, p0, p1, g, st);
        check_launch();
    }

    void compute_bbox() {
        launch_bbox(P, g, st);
        check_launch();
    }

    // Reads and clears the device error flag; throws on a region error.
    void check_region_error() {
        CK(cudaMemcpyAsync(err_h, err, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        const int e = *err_h;
        if (e > 0) {
            CK(cudaMemsetAsync(err, 0, sizeof(int), st));
            std::vector<double> xb(2 * (size_t)np);
            CK(cudaMemcpyAsync(xb.data(), P.xb, sizeof(double) * 2 * np, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            const int p = e - 1;
            throw ApiError{IBPM_ERR_REGION, "Panel index=" + std::to_string(e) + " at (" + jl_float(xb[p]) + ", " +
                                                 jl_float(xb[np + p]) + ") outside allowed region"};
        }
    }

    static std::string jl_float(double v) {
        char buf[64];
        for (int prec = 1; prec <= 17; ++prec) {
            snprintf(buf, sizeof buf, "%.*g", prec, v);
            if (strtod(buf, nullptr) == v) break;
        }
        std::string s(buf);
        if (s.find_first_of(".eni") == std::string::npos) s += ".0";
        return s;
    }

    void setup();
    void build_Binv();
    int cg(double *x, const double *b);
    void step(const ibpm_step_params &prm_in);
    void step_body();
    // CUDA graphs of step_body (static bodies), one per buffer parity
    bool use_graphs = true;
    cudaGraph_t graph[2] = {nullptr, nullptr};
    cudaGraphExec_t graph_exec[2] = {nullptr, nullptr};
    long long graph_launches[2] = {0, 0};
    void materialise_q0();
};

void ibpm_handle::setup() {
    CK(cudaSetDevice(device));
    if (const char *e = getenv("IBPM_NO_GRAPHS")) use_graphs = e[0] == '0';
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    if (!make_plan(nx, plx) || !make_plan(ny, ply))
        throw ApiError{IBPM_ERR_INVALID, "nx and ny must be even, <= 1024 and of the form 2^a 3^b 5^c"};
    // transform tables
    auto tables = [&](int M, double2 *&tw, double *&sn, double *&cs, Plan &pl) {
        std::vector<double2> htw(M);
        std::vector<double> hsn(M + 1), hcs(M + 1);
        for (int k = 0; k < M; ++k) {
            const long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)k / (long double)M;
            htw[k] = make_double2((double)cosl(a), (double)sinl(a));
        }
        for (int j = 0; j <= M; ++j) {
            hsn[j] = (double)sinl(3.14159265358979323846264338327950288L * (long double)j / (long double)M);
            hcs[j] = cos(M_PI * j / M);  // _lap_eigs uses cos(pi * i / nx) in Float64
        }
        tw = dalloc<double2>(M);
        sn = dalloc<double>(M + 1);
        cs = dalloc<double>(M + 1);
        CK(cudaMemcpyAsync(tw, htw.data(), sizeof(double2) * M, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(sn, hsn.data(), sizeof(double) * (M + 1), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(cs, hcs.data(), sizeof(double) * (M + 1), cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
        pl.tw = tw;
        pl.sn = sn;
    };
    tables(nx, twx, snx, cx, plx);
    tables(ny, twy, sny, cy, ply);

    q = dalloc<double>(nq * L);
    psi = dalloc<double>(ng * L);
    G[0] = dalloc<double>(ng * L);
    G[1] = dalloc<double>(ng * L);
    nl[0] = dalloc<double>(ng * L);
    nl[1] = dalloc<double>(ng * L);
    P.np = np;
    P.xb = dalloc<double>(2 * np);
    P.ub = dalloc<double>(2 * np);
    P.pc = dalloc<int>(2 * np);
    P.w = dalloc<double>((size_t)np * 2 * 49);
    P.bbox = dalloc<int>(4);
    err = dalloc<int>(4);
    P.err = err;
    ref_xb_d = dalloc<double>(2 * np);
    ds = dalloc<double>(np);
    Fbt = dalloc<double>(2 * np);
    fb = dalloc<double>(2 * np);
    total = dalloc<double>(2);
    prm = dalloc<StepDev>(1);
    motion = dalloc<double>(6 * (size_t)std::max(nbody, 1));
    CK(cudaMallocHost(&prm_h, sizeof(StepDev)));
    CK(cudaMallocHost(&motion_h, sizeof(double) * 6 * std::max(nbody, 1)));
    CK(cudaMallocHost(&cg_s_h, sizeof(double) * 8));
    CK(cudaMallocHost(&err_h, sizeof(int) * 4));
    memset(prm_h, 0, sizeof(StepDev));
    CK(cudaMemcpyAsync(ref_xb_d, ref_xb.data(), sizeof(double) * 2 * np, cudaMemcpyHostToDevice, st));

    // batch width for the B^-1 setup: ~4 GB of column work
    const long long per_col = (2 * ng * L + nq) * 8 + 2 * ng * 8;
    kbatch = (int)std::max(1LL, std::min<long long>(64, (4LL << 30) / per_col));
    if (!static_bodies) kbatch = 1;
    kbatch = std::min(kbatch, 2 * np);
    const int kb = std::max(kbatch, L);
    t1 = dalloc<double>(ng * kb);
    t2 = dalloc<double>(ng * kb);
    rhs = dalloc<double>(ng * L);
    rest = dalloc<double>(ng * L);
    qs1 = dalloc<double>(nq);
    Ftmp = dalloc<double>(2 * np);
    const int nchunk = (2 * np + 63) / 64;
    part = dalloc<double>((size_t)nchunk * 2 * np);
    patch_stride = 2LL * (nx + 1) * (ny + 1);
    patch = dalloc<double>(patch_stride * kbatch);
    Gw = dalloc<double>(ng * L * kbatch);
    psiw = dalloc<double>(ng * L * kbatch);
    qw = dalloc<double>(nq * kbatch);
    fcol = dalloc<double>(2 * (size_t)np * kbatch);
    cg_u = dalloc<double>(2 * np);
    cg_r = dalloc<double>(2 * np);
    cg_c = dalloc<double>(2 * np);
    cg_s = dalloc<double>(8);

    // _init_body_motion! (src/bodies.jl:33-41): static bodies take their panels now.
    std::vector<double> hxb(2 * (size_t)np, 0.0), hds(np, 0.0);
    for (int b = 0; b < nbody; ++b)
        if (body_kind[b] == IBPM_BODY_STATIC)
            for (int p = body_start[b]; p < body_start[b + 1]; ++p) {
                hxb[p] = ref_xb[p];
                hxb[np + p] = ref_xb[np + p];
                hds[p] = ref_ds[p];
            }
    CK(cudaMemcpyAsync(P.xb, hxb.data(), sizeof(double) * 2 * np, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ds, hds.data(), sizeof(double) * np, cudaMemcpyHostToDevice, st));
    for (int b = 0; b < nbody; ++b)
        if (body_kind[b] == IBPM_BODY_STATIC) update_weights(body_start[b], body_start[b + 1]);
    check_region_error();
    if (static_bodies) {
        compute_bbox();
        build_Binv();
    }
    CK(cudaStreamSynchronize(st));
}

// _Binv_precomputed (src/coupling.jl:187-192): B column by column, then its inverse.
void ibpm_handle::build_Binv() {
    const int n = 2 * np;
    Binv = dalloc<double>((size_t)n * n);
    rowk = dalloc<double>(n);
    colk = dalloc<double>(n);
    for (int c0 = 0; c0 < n; c0 += kbatch) {
        const int nb = std::min(kbatch, n - c0);
        unit_columns_kernel<<<(n * nb + 255) / 256, 256, 0, st>>>(fcol, n, c0, nb);
        check_launch();
        apply_B(fcol, Binv + (size_t)c0 * n, n, nb);
    }
    for (int k = 0; k < n; ++k) {
        gj_save_kernel<<<(n + 255) / 256, 256, 0, st>>>(Binv, n, k, rowk, colk, err + 1);
        check_launch();
        gj_update_kernel<<<dim3((n + 255) / 256, n), 256, 0, st>>>(Binv, n, k, rowk, colk);
        check_launch();
    }
    CK(cudaMemcpyAsync(err_h, err, sizeof(int) * 2, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (err_h[1] != 0) throw ApiError{IBPM_ERR_INVALID, "B is not positive definite (pivot " + std::to_string(err_h[1]) + ")"};
}

namespace {
// Single-block CG vector kernels (2np is at most a few thousand).
// mode 0: r = b - c; s[0] = ||r||
// mode 1: beta = s0^2/s1^2; u = r + beta u
// mode 2: alpha = s0^2 / dot(u, c); x += alpha u; r -= alpha c; s1 = s0; s0 = ||r||
__global__ void cg_vec_kernel(int mode, int n, double *x, double *r, double *u, const double *c, const double *b,
                              double *s) {
    __shared__ double red[32];
    auto block_sum = [&](double v) -> double {
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        __syncthreads();
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
        __syncthreads();
        double t = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[k];
        return t;
    };
    if (mode == 0) {
        double a = 0.0;
        for (int k = threadIdx.x; k < n; k += blockDim.x) {
            const double v = b[k] - c[k];
            r[k] = v;
            u[k] = 0.0;
            a += v * v;
        }
        const double t = block_sum(a);
        if (threadIdx.x == 0) {
            s[0] = sqrt(t);
            s[1] = 1.0;
        }
    } else if (mode == 1) {
        const double beta = s[0] * s[0] / (s[1] * s[1]);
        for (int k = threadIdx.x; k < n; k += blockDim.x) u[k] = r[k] + beta * u[k];
    } else {
        double a = 0.0;
        for (int k = threadIdx.x; k < n; k += blockDim.x) a += u[k] * c[k];
        const double uc = block_sum(a);
        const double alpha = s[0] * s[0] / uc;
        double rr = 0.0;
        for (int k = threadIdx.x; k < n; k += blockDim.x) {
            x[k] += alpha * u[k];
            const double v = r[k] - alpha * c[k];
            r[k] = v;
            rr += v * v;
        }
        const double t = block_sum(rr);
        if (threadIdx.x == 0) {
            s[1] = s[0];
            s[0] = sqrt(t);
        }
    }
}
}  // namespace

// IterativeSolvers.jl cg! as called at src/coupling.jl:198-201: plain CG from
// the initial guess x; stops when ||r|| <= max(reltol ||r0||, abstol) or after
// maxiter iterations.  Returns the iteration count.
int ibpm_handle::cg(double *x, const double *b) {
    const int n = 2 * np;
    apply_B(x, cg_c, n, 1);
    cg_vec_kernel<<<1, 256, 0, st>>>(0, n, x, cg_r, cg_u, cg_c, b, cg_s);
    check_launch();
    CK(cudaMemcpyAsync(cg_s_h, cg_s, sizeof(double) * 2, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    double res = cg_s_h[0];
    if (!std::isfinite(res)) throw ApiError{IBPM_ERR_NONFINITE, "non-finite residual in CG"};
    const double tol = std::max(opt.cg_reltol * res, opt.cg_abstol);
    int it = 0;
    while (!(it >= opt.cg_maxiter || res <= tol)) {
        cg_vec_kernel<<<1, 256, 0, st>>>(1, n, x, cg_r, cg_u, cg_c, b, cg_s);
        check_launch();
        apply_B(cg_u, cg_c, n, 1);
        cg_vec_kernel<<<1, 256, 0, st>>>(2, n, x, cg_r, cg_u, cg_c, b, cg_s);
        check_launch();
        CK(cudaMemcpyAsync(cg_s_h, cg_s, sizeof(double) * 2, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        res = cg_s_h[0];
        if (!std::isfinite(res)) throw ApiError{IBPM_ERR_NONFINITE, "non-finite residual in CG"};
        ++it;
    }
    last_cg_res = res;
    return it;
}

// advance!(::CnabSolver) (src/solver.jl:155-190)
void ibpm_handle::step(const ibpm_step_params &sp) {
    // inc_time_index! and the host callbacks' values
    ++index;
    prm_h->fs[0] = sp.freestream[0];
    prm_h->fs[1] = sp.freestream[1];
    for (int k = 0; k < 6; ++k) prm_h->gm[k] = sp.grid_motion[k];
    fs_last[0] = sp.freestream[0];
    fs_last[1] = sp.freestream[1];
    for (int k = 0; k < 6; ++k) gm_last[k] = sp.grid_motion[k];
    CK(cudaMemcpyAsync(prm, prm_h, sizeof(StepDev), cudaMemcpyHostToDevice, st));
    // _update_body_motion! (src/bodies.jl:43-51)
    if (!static_bodies) {
        if (!sp.body_motion) throw ApiError{IBPM_ERR_INVALID, "body_motion is required for moving bodies"};
        memcpy(motion_h, sp.body_motion, sizeof(double) * 6 * nbody);
        CK(cudaMemcpyAsync(motion, motion_h, sizeof(double) * 6 * nbody, cudaMemcpyHostToDevice, st));
        for (int b = 0; b < nbody; ++b) {
            if (body_kind[b] != IBPM_BODY_MOVING_RIGID) continue;
            const int p0 = body_start[b], p1 = body_start[b + 1];
            launch_rigid_motion(P, ref_xb_d, motion + 6 * b, p0, p1, st);
            check_launch();
            update_weights(p0, p1);
        }
        compute_bbox();
        check_region_error();
    }
    q0_zero = false;
    q0_from_user = false;
    // Static bodies: the rest of the step is one CUDA graph per parity of the
    // ping-ponged Gamma / nonlin buffers (gc == nc always), captured on first use.
    if (static_bodies && use_graphs && !prof) {
        const int p = gc;
        if (!graph_exec[p]) {
            const int gc0 = gc, nc0 = nc;
            CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            try {
                step_body();
            } catch (...) {
                cudaGraph_t gdrop = nullptr;
                cudaStreamEndCapture(st, &gdrop);
                if (gdrop) cudaGraphDestroy(gdrop);
                (void)cudaGetLastError();
                gc = gc0;
                nc = nc0;
                throw;
            }
            CK(cudaStreamEndCapture(st, &graph[p]));
            CK(cudaGraphInstantiate(&graph_exec[p], graph[p], 0));
            gc = gc0;
            nc = nc0;
        }
        CK(cudaGraphLaunch(graph_exec[p], st));
        launches += graph_launches[p];
        gc = 1 - gc;
        nc = 1 - nc;
        last_cg_iters = 0;
        return;
    }
    step_body();
}

// The device work of one step after the per-step parameters are uploaded.
void ibpm_handle::step_body() {
    const long long launches0 = launches;
    double *Gold = G[gc], *Gnew = G[1 - gc];
    double *N1 = nl[nc], *N2 = nl[1 - nc];
    // get_trial_state (src/fluid.jl:467-506), all levels at once: the levels
    // only read the previous step's Gamma and q.
    {
        NonlinArgs a{q, Gold, N1, N2, rest, prm, g};
        const dim3 blk(32, 8), grd((nx - 1 + 31) / 32, (ny - 1 + 7) / 8, L);
        const int pe = prof_begin();
        nonlinear_kernel<<<grd, blk, 0, st>>>(a);
        check_launch();
        prof_end(pe, IBPM_KCLASS_NONLINEAR, 8.0 * (double)(nq + 4 * ng) * L);
    }
    trial(Gold, rest, Gnew);
    nc = 1 - nc;  // _cycle!(state.nonlin)
    vort2flux(psi, qs1, Gnew, 0, 0, 1, false);
    // couple_surface_rigid (src/coupling.jl:236-250)
    {
        launch_regT(P, qs1, 0, Ftmp, 0, 1, 1, prm, g, st);
        check_launch();
    }
    const int n = 2 * np;
    if (static_bodies) {
        const int nchunk = (n + 63) / 64;
        binv_gemv_kernel<<<dim3(nchunk, nchunk), 256, 0, st>>>(Binv, Ftmp, part, n);
        check_launch();
        binv_reduce_kernel<<<1, 1024, 0, st>>>(part, nchunk, n, Fbt, fb, total, g.h, g.dt, 1);
        check_launch();
        last_cg_iters = 0;
    } else {
        last_cg_iters = cg(Fbt, Ftmp);
        binv_reduce_kernel<<<1, 1024, 0, st>>>(nullptr, 0, n, Fbt, fb, total, g.h, g.dt, 0);
        check_launch();
    }
    // project_circ (src/coupling.jl:218-230): Gamma = Gamma_s; Gamma_1 -= Ainv_1 rot(E^T F~b)
    reg_patch(Fbt, 1);
    xpass(InRegRot{Patch{patch, P.bbox, patch_stride}}, out_plain(t1, ng), 1);
    ypass(t1, t2, ng, 1, mult(MULT_AIMPL, 1, 0));
    xpass(in_plain(t2, ng), OutSub{Gnew, ng, nx - 1}, 1);
    // vort2flux!(state.psi, state.q, state.Gamma)
    vort2flux(psi, q, Gnew, 0, 0, 1, true);
    gc = 1 - gc;
    graph_launches[1 - gc] = launches - launches0;
}

namespace {
// Evaluates an X-pass prologue functor on every (i, j) of one field (diagnostics).
template <class In>
__global__ void eval_prologue_kernel(In in, double *out, int nx, int ny) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (i > nx - 1 || j > ny - 1) return;
    out[(long long)(i - 1) + (long long)(nx - 1) * (j - 1)] = in(0, i, j);
}

__global__ void q0_fill_kernel(double *q0, const StepDev *prm, Grid g) {
    const long long nu = (long long)(g.nx + 1) * g.ny, nq = nu + (long long)g.nx * (g.ny + 1);
    const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int lev = blockIdx.y + 1;
    if (f >= nq) return;
    double v;
    if (f < nu)
        v = base_flux_x(g, prm, lev, (int)(f % (g.nx + 1)) + 1, (int)(f / (g.nx + 1)) + 1);
    else
        v = base_flux_y(g, prm, lev, (int)((f - nu) % g.nx) + 1, (int)((f - nu) / g.nx) + 1);
    q0[(long long)blockIdx.y * nq + f] = v;
}
}  // namespace

void ibpm_handle::materialise_q0() {
    if (!q0mat) q0mat = dalloc<double>(nq * L);
    if (q0_from_user) return;
    if (q0_zero) {
        CK(cudaMemsetAsync(q0mat, 0, sizeof(double) * nq * L, st));
        return;
    }
    prm_h->fs[0] = fs_last[0];
    prm_h->fs[1] = fs_last[1];
    for (int k = 0; k < 6; ++k) prm_h->gm[k] = gm_last[k];
    CK(cudaMemcpyAsync(prm, prm_h, sizeof(StepDev), cudaMemcpyHostToDevice, st));
    q0_fill_kernel<<<dim3((unsigned)((nq + 255) / 256), L), 256, 0, st>>>(q0mat, prm, g);
    check_launch();
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

template <class F>
static int guarded(ibpm_handle *h, F &&f) {
    try {
        f();
        return IBPM_OK;
    } catch (const ApiError &e) {
        if (h) h->last_error = e.msg;
        return e.code;
    } catch (const CudaError &e) {
        if (h) h->last_error = std::string("CUDA error ") + cudaGetErrorString(e.e) + " at " + e.where;
        return IBPM_ERR_CUDA;
    } catch (const std::exception &e) {
        if (h) h->last_error = e.what();
        return IBPM_ERR_INVALID;
    }
}

extern "C" {

void ibpm_default_options(ibpm_options *opt) {
    if (!opt) return;
    opt->precision = IBPM_FP64;
    opt->device = 0;
    opt->cg_maxiter = 5000;
    opt->cg_reltol = 1e-12;
    opt->cg_abstol = 0.0;
}

int ibpm_create(const ibpm_problem *p, const ibpm_options *opt_in, ibpm_handle **out) {
    if (out) *out = nullptr;
    if (!p || !out) {
        g_create_error = "null argument";
        return IBPM_ERR_INVALID;
    }
    ibpm_options opt;
    ibpm_default_options(&opt);
    if (opt_in) opt = *opt_in;
    if (opt.precision != IBPM_FP64) {
        g_create_error = "unsupported precision mode";
        return IBPM_ERR_INVALID;
    }
    if (p->nx < 8 || p->ny < 8 || p->nlevel < 1 || p->npanel < 1 || p->nbody < 1 || !p->body_kind || !p->body_start ||
        !p->body_xb || !p->body_ds || !(p->h > 0) || !(p->dt > 0) || !(p->Re > 0)) {
        g_create_error = "invalid problem description";
        return IBPM_ERR_INVALID;
    }
    if (p->body_start[0] != 0 || p->body_start[p->nbody] != p->npanel) {
        g_create_error = "body_start must run from 0 to npanel";
        return IBPM_ERR_INVALID;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= opt.device) {
        g_create_error = "no CUDA device available";
        return IBPM_ERR_CUDA;
    }
    ibpm_handle *h = new ibpm_handle();
    h->opt = opt;
    h->device = opt.device;
    h->nx = p->nx;
    h->ny = p->ny;
    h->L = p->nlevel;
    h->np = p->npanel;
    h->nbody = p->nbody;
    h->nu = (long long)(p->nx + 1) * p->ny;
    h->nq = h->nu + (long long)p->nx * (p->ny + 1);
    h->ng = (long long)(p->nx - 1) * (p->ny - 1);
    h->nbc = 2LL * (p->nx + 1) + 2LL * (p->ny + 1);
    h->g = Grid{p->nx, p->ny, p->nlevel, p->h, p->x0, p->y0, p->Re, p->dt, p->grid_moving ? 1 : 0};
    h->body_kind.assign(p->body_kind, p->body_kind + p->nbody);
    h->body_start.assign(p->body_start, p->body_start + p->nbody + 1);
    h->ref_xb.assign(p->body_xb, p->body_xb + 2 * (size_t)p->npanel);
    h->ref_ds.assign(p->body_ds, p->body_ds + p->npanel);
    for (int b = 0; b < p->nbody; ++b) {
        if (h->body_kind[b] != IBPM_BODY_STATIC && h->body_kind[b] != IBPM_BODY_MOVING_RIGID) {
            g_create_error = "unknown body kind";
            delete h;
            return IBPM_ERR_INVALID;
        }
        if (h->body_kind[b] != IBPM_BODY_STATIC) h->static_bodies = false;
    }
    // The reference rejects out-of-region static panels while building the
    // Regularization (coupling.jl:38-41), before any size restriction of ours.
    for (int b = 0; b < p->nbody; ++b) {
        if (h->body_kind[b] != IBPM_BODY_STATIC) continue;
        for (int k = h->body_start[b]; k < h->body_start[b + 1]; ++k) {
            const double xb = h->ref_xb[k], yb = h->ref_xb[p->npanel + k];
            const int ix = (int)nearbyint((xb - p->x0) / p->h + 1.0 - 0.25);
            const int iy = (int)nearbyint((yb - p->y0) / p->h + 1.0 - 0.25);
            if (!(3 < ix && ix <= p->nx - 3) || !(3 < iy && iy <= p->ny - 3)) {
                g_create_error = "Panel index=" + std::to_string(k + 1) + " at (" + ibpm_handle::jl_float(xb) + ", " +
                                 ibpm_handle::jl_float(yb) + ") outside allowed region";
                delete h;
                return IBPM_ERR_REGION;
            }
        }
    }
    const int rc = guarded(h, [&] { h->setup(); });
    if (rc != IBPM_OK) {
        g_create_error = h->last_error;
        delete h;
        return rc;
    }
    *out = h;
    return IBPM_OK;
}

void ibpm_destroy(ibpm_handle *h) { delete h; }

int ibpm_set_state(ibpm_handle *h, const ibpm_state_view *s) {
    if (!h || !s) return IBPM_ERR_INVALID;
    return guarded(h, [&] {
        CK(cudaSetDevice(h->device));
        const size_t ngL = sizeof(double) * h->ng * h->L, nqL = sizeof(double) * h->nq * h->L;
        const size_t np2 = sizeof(double) * 2 * h->np;
        h->index = s->index;
        h->t0 = s->t0;
        if (s->q) CK(cudaMemcpyAsync(h->q, s->q, nqL, cudaMemcpyHostToDevice, h->st));
        if (s->q0) {
            if (!h->q0mat) h->q0mat = h->dalloc<double>(h->nq * h->L);
            CK(cudaMemcpyAsync(h->q0mat, s->q0, nqL, cudaMemcpyHostToDevice, h->st));
            h->q0_from_user = true;
        }
        if (s->gamma) CK(cudaMemcpyAsync(h->G[h->gc], s->gamma, ngL, cudaMemcpyHostToDevice, h->st));
        if (s->psi) CK(cudaMemcpyAsync(h->psi, s->psi, ngL, cudaMemcpyHostToDevice, h->st));
        if (s->nonlin1) CK(cudaMemcpyAsync(h->nl[h->nc], s->nonlin1, ngL, cudaMemcpyHostToDevice, h->st));
        if (s->nonlin2) CK(cudaMemcpyAsync(h->nl[1 - h->nc], s->nonlin2, ngL, cudaMemcpyHostToDevice, h->st));
        if (s->xb) CK(cudaMemcpyAsync(h->P.xb, s->xb, np2, cudaMemcpyHostToDevice, h->st));
        if (s->ds) CK(cudaMemcpyAsync(h->ds, s->ds, np2 / 2, cudaMemcpyHostToDevice, h->st));
        if (s->ub) CK(cudaMemcpyAsync(h->P.ub, s->ub, np2, cudaMemcpyHostToDevice, h->st));
        if (s->fbt) CK(cudaMemcpyAsync(h->Fbt, s->fbt, np2, cudaMemcpyHostToDevice, h->st));
        h->fs_last[0] = s->freestream[0];
        h->fs_last[1] = s->freestream[1];
        // update_vars! (problem.jl:676-685)
        binv_reduce_kernel<<<1, 1024, 0, h->st>>>(nullptr, 0, 2 * h->np, h->Fbt, h->fb, h->total, h->g.h, h->g.dt, 0);
        h->check_launch();
        CK(cudaStreamSynchronize(h->st));
    });
}

int ibpm_get_state(ibpm_handle *h, ibpm_state_view *s) {
    if (!h || !s) return IBPM_ERR_INVALID;
    return guarded(h, [&] {
        CK(cudaSetDevice(h->device));
        const size_t ngL = sizeof(double) * h->ng * h->L, nqL = sizeof(double) * h->nq * h->L;
        const size_t np2 = sizeof(double) * 2 * h->np;
        s->index = h->index;
        s->t0 = h->t0;
        s->freestream[0] = h->fs_last[0];
        s->freestream[1] = h->fs_last[1];
        if (s->q) CK(cudaMemcpyAsync(s->q, h->q, nqL, cudaMemcpyDeviceToHost, h->st));
        if (s->q0) {
            h->materialise_q0();
            CK(cudaMemcpyAsync(s->q0, h->q0mat, nqL, cudaMemcpyDeviceToHost, h->st));
        }
        if (s->gamma) CK(cudaMemcpyAsync(s->gamma, h->G[h->gc], ngL, cudaMemcpyDeviceToHost, h->st));
        if (s->psi) CK(cudaMemcpyAsync(s->psi, h->psi, ngL, cudaMemcpyDeviceToHost, h->st));
        if (s->nonlin1) CK(cudaMemcpyAsync(s->nonlin1, h->nl[h->nc], ngL, cudaMemcpyDeviceToHost, h->st));
        if (s->nonlin2) CK(cudaMemcpyAsync(s->nonlin2, h->nl[1 - h->nc], ngL, cudaMemcpyDeviceToHost, h->st));
        if (s->xb) CK(cudaMemcpyAsync(s->xb, h->P.xb, np2, cudaMemcpyDeviceToHost, h->st));
        if (s->ds) CK(cudaMemcpyAsync(s->ds, h->ds, np2 / 2, cudaMemcpyDeviceToHost, h->st));
        if (s->ub) CK(cudaMemcpyAsync(s->ub, h->P.ub, np2, cudaMemcpyDeviceToHost, h->st));
        if (s->fbt) CK(cudaMemcpyAsync(s->fbt, h->Fbt, np2, cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
    });
}

int ibpm_advance(ibpm_handle *h, int64_t nsteps, const ibpm_step_params *params) {
    if (!h || nsteps < 0 || (nsteps > 0 && !params)) return IBPM_ERR_INVALID;
    bool maxiter = false;
    const int rc = guarded(h, [&] {
        CK(cudaSetDevice(h->device));
        for (int64_t k = 0; k < nsteps; ++k) {
            h->step(params[k]);
            if (!h->static_bodies && h->last_cg_iters >= h->opt.cg_maxiter) maxiter = true;
        }
        CK(cudaStreamSynchronize(h->st));
    });
    if (rc != IBPM_OK) return rc;
    if (maxiter) {
        h->last_error = "CG reached maxiter";
        return IBPM_WARN_CG_MAXITER;
    }
    return IBPM_OK;
}

int ibpm_get_forces(ibpm_handle *h, double *fb, double *total_force) {
    if (!h) return IBPM_ERR_INVALID;
    return guarded(h, [&] {
        CK(cudaSetDevice(h->device));
        if (fb) CK(cudaMemcpyAsync(fb, h->fb, sizeof(double) * 2 * h->np, cudaMemcpyDeviceToHost, h->st));
        if (total_force) CK(cudaMemcpyAsync(total_force, h->total, sizeof(double) * 2, cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
    });
}

int ibpm_get_time(ibpm_handle *h, int64_t *index, double *t) {
    if (!h) return IBPM_ERR_INVALID;
    if (index) *index = h->index;
    if (t) *t = h->t0 + h->g.dt * (double)(h->index - 1);
    return IBPM_OK;
}

int ibpm_get_info(ibpm_handle *h, ibpm_info *info) {
    if (!h || !info) return IBPM_ERR_INVALID;
    info->nq = h->nq;
    info->ng = h->ng;
    info->nbc = h->nbc;
    info->static_bodies = h->static_bodies ? 1 : 0;
    info->last_cg_iters = h->last_cg_iters;
    info->last_cg_residual = h->last_cg_res;
    info->device_bytes = h->dev_bytes;
    return IBPM_OK;
}

const char *ibpm_last_error(const ibpm_handle *h) { return h ? h->last_error.c_str() : g_create_error.c_str(); }

void *ibpm_stream(ibpm_handle *h) { return h ? (void *)h->st : nullptr; }

int64_t ibpm_kernel_launches(const ibpm_handle *h) { return h ? h->launches : 0; }

int ibpm_diag_solve(ibpm_handle *h, int op, int level, const double *b, double *x) {
    if (!h || !b || !x || op < 0 || op > 2 || level < 1 || level > h->L) return IBPM_ERR_INVALID;
    return guarded(h, [&] {
        CK(cudaSetDevice(h->device));
        const size_t bytes = sizeof(double) * h->ng;
        CK(cudaMemcpyAsync(h->rhs, b, bytes, cudaMemcpyHostToDevice, h->st));
        const int mode = op == 0 ? MULT_LAPINV : (op == 1 ? MULT_AEXPL : MULT_AIMPL);
        h->xpass(h->in_plain(h->rhs, h->ng), h->out_plain(h->t1, h->ng), 1);
        h->ypass(h->t1, h->t2, h->ng, 1, h->mult(mode, level, 0));
        h->xpass(h->in_plain(h->t2, h->ng), h->out_plain(h->rhs, h->ng), 1);
        CK(cudaMemcpyAsync(x, h->rhs, bytes, cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
    });
}

int ibpm_diag_apply_B(ibpm_handle *h, const double *z, double *x) {
    if (!h || !z || !x) return IBPM_ERR_INVALID;
    return guarded(h, [&] {
        CK(cudaSetDevice(h->device));
        const size_t bytes = sizeof(double) * 2 * h->np;
        CK(cudaMemcpyAsync(h->cg_u, z, bytes, cudaMemcpyHostToDevice, h->st));
        h->compute_bbox();
        h->apply_B(h->cg_u, h->cg_c, 2 * h->np, 1);
        CK(cudaMemcpyAsync(x, h->cg_c, bytes, cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
    });
}

int ibpm_diag_binv(ibpm_handle *h, double *out) {
    if (!h || !out) return IBPM_ERR_INVALID;
    if (!h->Binv) {
        h->last_error = "no precomputed B^-1 (moving bodies)";
        return IBPM_ERR_INVALID;
    }
    return guarded(h, [&] {
        const size_t n = 2 * (size_t)h->np;
        CK(cudaMemcpyAsync(out, h->Binv, sizeof(double) * n * n, cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
    });
}

int ibpm_diag_vort2flux(ibpm_handle *h, double *gamma, double *psi, double *q) {
    if (!h || !gamma || !psi || !q) return IBPM_ERR_INVALID;
    return guarded(h, [&] {
        CK(cudaSetDevice(h->device));
        const size_t ngL = sizeof(double) * h->ng * h->L;
        CK(cudaMemcpyAsync(h->Gw, gamma, ngL, cudaMemcpyHostToDevice, h->st));
        double *qd = h->dalloc<double>(h->nq * h->L);
        h->vort2flux(h->psiw, qd, h->Gw, 0, 0, 1, true);
        CK(cudaMemcpyAsync(gamma, h->Gw, ngL, cudaMemcpyDeviceToHost, h->st));
        CK(cudaMemcpyAsync(psi, h->psiw, ngL, cudaMemcpyDeviceToHost, h->st));
        CK(cudaMemcpyAsync(q, qd, sizeof(double) * h->nq * h->L, cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
    });
}

int ibpm_diag_reg(ibpm_handle *h, const double *f, double *gamma1, const double *q1, double *fout) {
    if (!h) return IBPM_ERR_INVALID;
    return guarded(h, [&] {
        CK(cudaSetDevice(h->device));
        const size_t nf = sizeof(double) * 2 * h->np;
        h->compute_bbox();
        if (f && gamma1) {
            CK(cudaMemcpyAsync(h->cg_u, f, nf, cudaMemcpyHostToDevice, h->st));
            h->reg_patch(h->cg_u, 1);
            // the X-pass prologue (InRegRot) evaluated on every Gamma point
            const dim3 blk(32, 8), grd((h->nx - 1 + 31) / 32, (h->ny - 1 + 7) / 8);
            eval_prologue_kernel<<<grd, blk, 0, h->st>>>(InRegRot{Patch{h->patch, h->P.bbox, h->patch_stride}}, h->t2,
                                                         h->nx, h->ny);
            h->check_launch();
            CK(cudaMemcpyAsync(gamma1, h->t2, sizeof(double) * h->ng, cudaMemcpyDeviceToHost, h->st));
        }
        if (q1 && fout) {
            CK(cudaMemcpyAsync(h->qw, q1, sizeof(double) * h->nq, cudaMemcpyHostToDevice, h->st));
            launch_regT(h->P, h->qw, 0, h->cg_c, 0, 1, 0, h->prm, h->g, h->st);
            h->check_launch();
            CK(cudaMemcpyAsync(fout, h->cg_c, nf, cudaMemcpyDeviceToHost, h->st));
        }
        CK(cudaStreamSynchronize(h->st));
    });
}

int ibpm_profile(ibpm_handle *h, int enable) {
    if (!h) return IBPM_ERR_INVALID;
    return guarded(h, [&] {
        CK(cudaStreamSynchronize(h->st));
        h->prof = enable != 0;
        h->prof_recs.clear();
        h->ev_next = 0;
    });
}

int ibpm_profile_read(ibpm_handle *h, int kclass, int64_t *launches, double *ms, double *bytes) {
    if (!h || kclass < 0 || kclass >= IBPM_KCLASS_COUNT) return IBPM_ERR_INVALID;
    return guarded(h, [&] {
        CK(cudaStreamSynchronize(h->st));
        int64_t n = 0;
        double t = 0.0, b = 0.0;
        for (const auto &r : h->prof_recs) {
            if (r.cls != kclass) continue;
            float e = 0.f;
            CK(cudaEventElapsedTime(&e, h->ev_pool[r.ev], h->ev_pool[r.ev + 1]));
            ++n;
            t += e;
            b += r.bytes;
        }
        if (launches) *launches = n;
        if (ms) *ms = t;
        if (bytes) *bytes = b;
    });
}

}  // extern "C"
