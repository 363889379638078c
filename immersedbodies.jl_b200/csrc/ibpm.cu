// ibpm.cu -- libibpm_b200: the CNAB/IBPM time step on one B200, behind the C
// ABI of include/ibpm_b200.h.  Engine<double> is the plain FP64 drop-in path;
// Engine<float> is the mixed-precision path (FP32 fields and transforms, FP64
// scans, boundary values, CG and force sums, and an FP64 B^-1).
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
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>
#include <fstream>
#include <initializer_list>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <vector>

#include "../../include/ibpm_b200.h"
#include "coupling.h"
#include "warmstart.h"
#include "kernels.cuh"
#include "tc_dst.h"

using namespace ibpm;

namespace {

constexpr int kNG = 2;  // FFT groups (line pairs) per block

// Spectral multipliers of one level for the tensor-core transforms, as FP32
// [kx][ky] with both frequencies in the transforms' block order (P x P, zero at
// the padding slots)
__global__ void tc_mult_kernel(Mult m, int P, float *tab) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
    if (r >= P) return;
    const int kx = tc_blk(c, P), ky = tc_blk(r, P);
    tab[(size_t)c * P + r] = (kx != 0 && ky != 0) ? (float)m(m.coef(0), kx, ky) : 0.0f;
}

constexpr int kNGWide = 4, kWideBatch = 16;  // Y-pass groups per block for launches over >= kWideBatch fields

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

// Julia's shortest round-trip printing of a Float64 (for the reference's error text).
std::string jl_float(double v) {
    char buf[64];
    for (int prec = 1; prec <= 17; ++prec) {
        snprintf(buf, sizeof buf, "%.*g", prec, v);
        if (strtod(buf, nullptr) == v) break;
    }
    std::string s(buf);
    if (s.find_first_of(".eni") == std::string::npos) s += ".0";
    return s;
}

template <class T>
bool make_plan(int M, PlanT<T> &pl) {
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

// ---- pass-shape autotuner ----
// The Y pass (DST along y, spectral multiply, DST along y) runs with NG line
// pairs (2 NG columns) per block, NG in {1, 2, 4, 8}.  Every NG evaluates the
// same per-line arithmetic, so the choice changes speed only, never results.
// The best NG depends on the transform length, the precision and how many
// fields one launch covers (one level, all levels, an ensemble group, a batch
// of B columns), so the table is keyed by (GPU name, transform length,
// precision, batch bucket).  With IBPM_TUNE=1 an engine times every NG on its
// own scratch fields for each key it will launch (before any graph capture) and
// keeps the fastest; IBPM_TUNE_CACHE names a text file the table is read from
// at first use and appended to after tuning, so later processes start tuned.
// Keys never tuned use the fixed rule (NG = 2, NG = 4 from 16 fields).
// IBPM_TUNE_FORCE_NG forces one NG everywhere (a test knob).
constexpr int kTuneNGs[4] = {1, 2, 4, 8};
inline int batch_bucket(int nb) { return nb <= 1 ? 0 : nb <= 4 ? 1 : nb <= 15 ? 2 : nb <= 63 ? 3 : 4; }

struct TuneTable {
    std::mutex mu;
    std::map<std::string, int> ng;  // key -> NG
    bool loaded = false;
    std::string path;
    // (re)reads the cache file named by IBPM_TUNE_CACHE when that name changes;
    // its entries replace the table's
    void load_locked() {
        const char *p = getenv("IBPM_TUNE_CACHE");
        const std::string want = p ? p : "";
        if (loaded && want == path) return;
        loaded = true;
        path = want;
        if (path.empty()) return;
        std::ifstream f(path);
        std::string line;
        while (std::getline(f, line)) {
            const size_t at = line.rfind(' ');
            if (at == std::string::npos) continue;
            const int v = atoi(line.c_str() + at + 1);
            if (v == 1 || v == 2 || v == 4 || v == 8) ng[line.substr(0, at)] = v;
        }
    }
    bool find(const std::string &key, int *out) {
        std::lock_guard<std::mutex> lk(mu);
        load_locked();
        auto it = ng.find(key);
        if (it == ng.end()) return false;
        *out = it->second;
        return true;
    }
    void put(const std::string &key, int v) {
        std::lock_guard<std::mutex> lk(mu);
        load_locked();
        ng[key] = v;
        if (!path.empty()) {
            std::ofstream f(path, std::ios::app);
            f << key << ' ' << v << '\n';
        }
    }
    std::string dump() {
        std::lock_guard<std::mutex> lk(mu);
        load_locked();
        std::ostringstream o;
        for (auto &kv : ng) o << kv.first << ' ' << kv.second << '\n';
        return o.str();
    }
};
TuneTable &tune_table() {
    static TuneTable t;
    return t;
}
bool tune_enabled() {
    const char *e = getenv("IBPM_TUNE");
    return e && e[0] == '1';
}
int tune_forced_ng() {
    const char *e = getenv("IBPM_TUNE_FORCE_NG");
    const int v = e ? atoi(e) : 0;
    return (v == 1 || v == 2 || v == 4 || v == 8) ? v : 0;
}

}  // namespace

// The C ABI's opaque handle: one engine of either precision.
struct ibpm_handle {
    std::string last_error;
    // the ensembles holding this case, told when it is destroyed, so that an
    // ensemble destroyed after its cases (any order of destruction) never
    // touches them
    std::vector<std::pair<ibpm_ensemble *, void (*)(ibpm_ensemble *, ibpm_handle *)>> holders;
    virtual ~ibpm_handle() {
        for (auto &w : holders) w.second(w.first, this);
    }
    virtual void set_state(const ibpm_state_view *s) = 0;
    virtual void get_state(ibpm_state_view *s) = 0;
    virtual void get_field(int field, int level, double *out) = 0;
    virtual bool advance(int64_t nsteps, const ibpm_step_params *params) = 0;  // true: CG hit maxiter
    // one step enqueued on the handle's stream without waiting for it (ensembles)
    virtual void enqueue_step(const ibpm_step_params &prm) = 0;
    // waits for the enqueued steps; true: a CG hit maxiter
    virtual bool finish_steps() = 0;
    virtual void get_forces(double *fb, double *total) = 0;
    virtual void get_time(int64_t *index, double *t) = 0;
    virtual void get_info(ibpm_info *info) = 0;
    virtual void *stream_ptr() = 0;
    virtual long long launch_count() const = 0;
    virtual void set_profile(int enable) = 0;
    virtual void read_profile(int kclass, int64_t *launches, double *ms, double *bytes) = 0;
    virtual void diag_solve(int op, int level, const double *b, double *x) = 0;
    virtual void diag_apply_B(const double *z, double *x) = 0;
    virtual void diag_binv(double *out) = 0;
    virtual void diag_vort2flux(double *gamma, double *psi, double *q) = 0;
    virtual void diag_reg(const double *f, double *gamma1, const double *q1, double *fout) = 0;
    virtual void set_warm_start(ibpm_net *net, int mode, int depth) = 0;
    virtual void set_rebuild_transform(int products) = 0;
    virtual void warm_start_sample(float *features, float *target, float *prediction) = 0;
};

template <class T>
struct Engine final : ibpm_handle {
    using C = typename Cx<T>::type;
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
    PlanT<T> plx{}, ply{};
    C *twx = nullptr, *twy = nullptr;
    T *snx = nullptr, *sny = nullptr;
    double *cx = nullptr, *cy = nullptr;
    // state
    int64_t index = 0;
    double t0 = 0.0;
    T *q = nullptr, *psi = nullptr, *G[2] = {nullptr, nullptr}, *nl[2] = {nullptr, nullptr};
    int gc = 0;  // state.Γ = G[gc]
    int nc = 0;  // state.nonlin[1] = nl[nc], state.nonlin[2] = nl[1 - nc]
    T *q0mat = nullptr;
    double *stage = nullptr;  // double staging buffer for FP32 state transfers
    size_t stage_len = 0;
    bool q0_from_user = false;
    bool q0_zero = true;  // State(prob) starts with q0 = 0 until the first step
    Panels P{};
    double *ref_xb_d = nullptr, *ds = nullptr;
    double *Fbt = nullptr, *fb = nullptr, *total = nullptr;
    StepDev *prm = nullptr, *prm_h = nullptr;
    double *motion = nullptr, *motion_h = nullptr;
    // Pinned staging of the per-step parameters: a ring of slots, each reused only
    // after the copies that read it have run (asynchronous copies read pinned
    // host memory when they execute, not when they are enqueued).
    static constexpr int kStage = 8;
    StepDev *stage_prm[kStage] = {};
    double *stage_motion[kStage] = {};
    cudaEvent_t stage_ev[kStage] = {};
    bool stage_used[kStage] = {};
    int stage_next = 0;
    // next free slot: prm_h / motion_h point into it
    void stage_acquire() {
        const int k = stage_next;
        stage_next = (stage_next + 1) % kStage;
        if (stage_used[k]) CK(cudaEventSynchronize(stage_ev[k]));
        prm_h = stage_prm[k];
        motion_h = stage_motion[k];
        stage_used[k] = true;
    }
    // marks the slot just used as busy until the stream reaches this point
    void stage_release() { CK(cudaEventRecord(stage_ev[(stage_next + kStage - 1) % kStage], st)); }
    // learned CG warm start (moving bodies): the installed network, the solution
    // of two steps back, the features and prediction of the current step
    ibpm_net *ws = nullptr;
    int ws_mode = IBPM_WS_PREVIOUS;
    int ws_depth = 0;                       // previous solutions kept for IBPM_WS_PROJECTED
    // IBPM_WS_DIRECT / IBPM_WS_PRECONDITIONED: B^-1 of the body position, rebuilt
    // every ws_refresh steps (ws_since counts the steps since the last rebuild) by
    // its own graph
    bool uses_binv_start() const {
        return ws_mode == IBPM_WS_DIRECT || ws_mode == IBPM_WS_PRECONDITIONED || ws_mode == IBPM_WS_PRECOND_EXTRAP;
    }
    bool preconditioned() const { return ws_mode == IBPM_WS_PRECONDITIONED || ws_mode == IBPM_WS_PRECOND_EXTRAP; }
    // IBPM_WS_PRECOND_EXTRAP: the last three stale errors e_k = F_k - Binv b_k (ring
    // of 3 x 2np), this step's Binv b, and how many errors are valid since the
    // last rebuild (device int)
    double *ws_stale = nullptr, *ws_x0 = nullptr;
    int *ws_nvalid = nullptr;
    // The preconditioned modes' B assembly on the tensor cores: tc_prod BF16
    // products per transform (0: the FP64 transforms); tc_on while an assembly
    // runs its solves there; multipliers of level 1: Laplacian inverse and
    // implicit diffusion (tc_mult[0], tc_mult[1]), any mode and level for
    // ibpm_diag_solve (tc_mult[2])
    int tc_prod = 0;
    bool tc_on = false;
    TcDstPlan *tc = nullptr;
    float *tc_mult[3] = {nullptr, nullptr, nullptr};
    int ws_refresh = 1;
    long long ws_since = 0;
    cudaGraph_t binv_graph = nullptr;
    cudaGraphExec_t binv_exec = nullptr;
    long long binv_graph_launches = 0;
    double *ws_hist = nullptr, *ws_bhist = nullptr, *ws_G = nullptr, *ws_h = nullptr;
    double *Fprev = nullptr, *ws_z = nullptr, *ws_bz = nullptr, *ws_x2 = nullptr, *ws_bx2 = nullptr;
    float *ws_feat = nullptr, *ws_y = nullptr, *ws_act = nullptr;
    size_t ws_act_cap = 0;
    int *pbody_d = nullptr;
    double fs_last[2] = {0, 0}, gm_last[6] = {0, 0, 0, 0, 0, 0};
    // work
    int kbatch = 1;  // columns per batch in the B setup
    T *t1 = nullptr, *t2 = nullptr, *rhs = nullptr, *rest = nullptr, *qs1 = nullptr;
    double *Ftmp = nullptr, *part = nullptr;
    T *patch = nullptr;
    long long patch_stride = 0;
    T *Gw = nullptr, *psiw = nullptr, *qw = nullptr;  // batch work (K columns)
    double *fcol = nullptr;
    double *Binv = nullptr, *Bwork = nullptr;  // B^-1 and the Gauss-Jordan ping-pong buffer
    double *cg_u = nullptr, *cg_r = nullptr, *cg_c = nullptr, *cg_z = nullptr, *cg_s = nullptr, *cg_s_h = nullptr;
    int *err = nullptr, *err_h = nullptr;
    int last_cg_iters = 0;
    double last_cg_res = 0.0, first_cg_res = 0.0, ws_coef[2] = {0.0, 0.0};
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
    std::vector<long long> alloc_bytes;  // size of each entry of allocs
    // frees one allocation of this handle
    void dfree(void *p) {
        if (!p) return;
        auto it = std::find(allocs.begin(), allocs.end(), p);
        if (it != allocs.end()) {
            const size_t i = (size_t)(it - allocs.begin());
            dev_bytes -= alloc_bytes[i];
            alloc_bytes.erase(alloc_bytes.begin() + (long)i);
            allocs.erase(it);
        }
        cudaFree(p);
    }
    // grows the column-batch buffers to kb columns (the projected warm start
    // applies B to all kept solutions in one batched pass)
    void grow_batch_buffers(int kb) {
        if (kb > kbatch) resize_batch_buffers(kb);
    }
    // After the B^-1 setup a static-body handle applies B to one vector at a time:
    // the setup's column-batch buffers shrink to one column.
    void shrink_batch_buffers() {
        if (kbatch > 1) resize_batch_buffers(1);
    }
    // Column-batch work buffers for kb columns.  The new buffers are allocated
    // before the old ones are freed, so a failed allocation leaves the handle as
    // it was; the captured graphs, which hold the old addresses, are dropped.
    void resize_batch_buffers(int kb) {
        CK(cudaStreamSynchronize(st));
        const int k2 = std::max(kb, L);
        const size_t sizes[7] = {sizeof(T) * (size_t)(ng * k2),        sizeof(T) * (size_t)(ng * k2),
                                 sizeof(T) * (size_t)(patch_stride * kb), sizeof(T) * (size_t)(ng * L * kb),
                                 sizeof(T) * (size_t)(ng * L * kb),     sizeof(T) * (size_t)(nq * kb),
                                 sizeof(double) * 2 * (size_t)np * kb};
        void *fresh[7] = {};
        try {
            for (int k = 0; k < 7; ++k) fresh[k] = dalloc<unsigned char>(sizes[k]);
        } catch (...) {
            for (void *p : fresh) dfree(p);
            throw;
        }
        drop_graphs();
        for (void *p : {(void *)t1, (void *)t2, (void *)patch, (void *)Gw, (void *)psiw, (void *)qw, (void *)fcol})
            dfree(p);
        t1 = static_cast<T *>(fresh[0]);
        t2 = static_cast<T *>(fresh[1]);
        patch = static_cast<T *>(fresh[2]);
        Gw = static_cast<T *>(fresh[3]);
        psiw = static_cast<T *>(fresh[4]);
        qw = static_cast<T *>(fresh[5]);
        fcol = static_cast<double *>(fresh[6]);
        kbatch = kb;
    }

    template <class U>
    U *dalloc(size_t n) {
        void *p = nullptr;
        if (n == 0) n = 1;
        cudaError_t e = cudaMalloc(&p, n * sizeof(U));
        if (e != cudaSuccess) {
            (void)cudaGetLastError();  // not sticky: clear it so later launch checks do not report it
            throw ApiError{IBPM_ERR_NOMEM, "cudaMalloc of " + std::to_string(n * sizeof(U)) + " bytes failed"};
        }
        allocs.push_back(p);
        alloc_bytes.push_back((long long)(n * sizeof(U)));
        dev_bytes += (long long)(n * sizeof(U));
        CK(cudaMemsetAsync(p, 0, n * sizeof(U), st));
        return static_cast<U *>(p);
    }
    // drops the captured step graphs (re-captured on the next step)
    void drop_graphs() {
        for (int p = 0; p < 2; ++p) {
            if (graph_exec[p]) cudaGraphExecDestroy(graph_exec[p]);
            if (graph[p]) cudaGraphDestroy(graph[p]);
            graph_exec[p] = nullptr;
            graph[p] = nullptr;
        }
        if (binv_exec) cudaGraphExecDestroy(binv_exec);
        if (binv_graph) cudaGraphDestroy(binv_graph);
        binv_exec = nullptr;
        binv_graph = nullptr;
    }
    ~Engine() override {
        if (st) cudaStreamSynchronize(st);
        drop_graphs();
        if (tc) tc_destroy(tc);
        for (cudaEvent_t e : ev_pool) cudaEventDestroy(e);
        for (void *p : allocs) cudaFree(p);
        for (int k = 0; k < kStage; ++k) {
            if (stage_prm[k]) cudaFreeHost(stage_prm[k]);
            if (stage_motion[k]) cudaFreeHost(stage_motion[k]);
            if (stage_ev[k]) cudaEventDestroy(stage_ev[k]);
        }
        if (cg_s_h) cudaFreeHost(cg_s_h);
        if (err_h) cudaFreeHost(err_h);
        if (st_side) cudaStreamDestroy(st_side);
        if (st) cudaStreamDestroy(st);
    }

    void check_launch() {
        ++launches;
        CK(cudaGetLastError());
    }
    // cudaFuncSetAttribute holds for the current device only: a kernel's launch
    // site records the devices it set an attribute on (devices >= 64 set it every time)
    unsigned long long device_bit() const { return device < 64 ? 1ull << device : 0ull; }
    bool need_attr(const std::atomic<unsigned long long> &done) const {
        const unsigned long long bit = device_bit();
        return bit == 0 || !(done.load() & bit);
    }

    // ---- line passes ----
    // Dispatch on the transform length: compile-time transforms for
    // M in {256, 384, 512, 1024}, the runtime mixed-radix one otherwise.
    template <class D, class In, class Out>
    void xpass_t(const PlanT<typename D::Real> &pl, In in, Out out, int nbatch, const int *rows, int zero_outside,
                 int rows_stride) {
        const int pairs = (ny - 1 + 1) / 2;
        const dim3 grid((pairs + kNG - 1) / kNG, nbatch);
        const size_t sm = pass_smem<D>(pl.M, kNG, kNG);
        xpass_kernel<D, kNG, In, Out><<<grid, kNG * D::TPF, sm, st>>>(in, out, pl, ny - 1, rows, zero_outside,
                                                                       rows_stride);
    }
    // X pass with transforms of element type R (the engine's T, or double for
    // the FP32 engine's FP64 level-1 solve); In/Out convert at the boundary.
    // rows, zero_outside, rows_stride: see xpass_kernel (rows null: every row).
    template <class R = T, class In, class Out>
    void xpass(In in, Out out, int nbatch, const int *rows = nullptr, int zero_outside = 0, int rows_stride = 0) {
        const PlanT<R> &pl = plan_x<R>();
        const int pe = prof_begin();
        switch (pl.M) {
            case 1024: xpass_t<Pow2Dst<1024, R>>(pl, in, out, nbatch, rows, zero_outside, rows_stride); break;
            case 512: xpass_t<Pow2Dst<512, R>>(pl, in, out, nbatch, rows, zero_outside, rows_stride); break;
            case 256: xpass_t<Pow2Dst<256, R>>(pl, in, out, nbatch, rows, zero_outside, rows_stride); break;
            case 384: xpass_t<MixDst<384, R>>(pl, in, out, nbatch, rows, zero_outside, rows_stride); break;
            default: xpass_t<GenericDst<R>>(pl, in, out, nbatch, rows, zero_outside, rows_stride); break;
        }
        check_launch();
        prof_end(pe, IBPM_KCLASS_XPASS, 2.0 * sizeof(R) * (double)ng * nbatch);
    }
    template <class D>
    void ypass_t(const PlanT<typename D::Real> &pl, const typename D::Real *in, typename D::Real *out, long long bs,
                 int nbatch, Mult m) {
        int ngy = ypass_ng<typename D::Real>(pl.M, nbatch, D::MC > 0);
        ypass_ng_launch<D>(ngy, pl, in, out, bs, nbatch, m);
    }
    template <class D>
    void ypass_ng_launch(int ngy, const PlanT<typename D::Real> &pl, const typename D::Real *in,
                         typename D::Real *out, long long bs, int nbatch, Mult m) {
        switch (ngy) {
            case 1: ypass_launch<D, 1>(pl, in, out, bs, nbatch, m); break;
            case 4: ypass_launch<D, 4>(pl, in, out, bs, nbatch, m); break;
            case 8: ypass_launch<D, 8>(pl, in, out, bs, nbatch, m); break;
            default: ypass_launch<D, 2>(pl, in, out, bs, nbatch, m); break;
        }
    }
    // the autotuner's key of a Y pass of length M over nbatch fields
    std::string devname;  // the GPU's name, read once at setup (a tuning key's first part)
    template <class R>
    std::string ypass_key(int M, int nbatch) const {
        return devname + " ypass M=" + std::to_string(M) + (sizeof(R) == 8 ? " fp64" : " fp32") +
               " batch=" + std::to_string(batch_bucket(nbatch));
    }
    // line pairs per block of a Y pass: forced, tuned, or the fixed rule
    template <class R>
    int ypass_ng(int M, int nbatch, bool compile_time) {
        if (const int f = tune_forced_ng()) return f;
        int v = 0;
        if (tune_table().find(ypass_key<R>(M, nbatch), &v)) return v;
        return compile_time && nbatch >= kWideBatch ? kNGWide : kNG;
    }
    // Times every NG of the Y pass over nbatch fields (scratch in -> out, at
    // least nbatch * ng elements each) and records the fastest; eager only.
    template <class R>
    void tune_ypass(const R *in, R *out, int nbatch) {
        if (!tune_enabled() || tune_forced_ng()) return;
        const PlanT<R> &pl = plan_y<R>();
        const std::string key = ypass_key<R>(pl.M, nbatch);
        int have = 0;
        if (tune_table().find(key, &have)) return;
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        CK(cudaStreamIsCapturing(st, &cs));
        if (cs != cudaStreamCaptureStatusNone) return;
        cudaEvent_t e0, e1;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        float best = 1e30f;
        int best_ng = kNG;
        for (int ngy : kTuneNGs) {
            auto run = [&] {
                switch (pl.M) {
                    case 1024: ypass_ng_launch<Pow2Dst<1024, R>>(ngy, pl, in, out, ng, nbatch, mult(MULT_LAPINV, 1, 0)); break;
                    case 512: ypass_ng_launch<Pow2Dst<512, R>>(ngy, pl, in, out, ng, nbatch, mult(MULT_LAPINV, 1, 0)); break;
                    case 256: ypass_ng_launch<Pow2Dst<256, R>>(ngy, pl, in, out, ng, nbatch, mult(MULT_LAPINV, 1, 0)); break;
                    case 384: ypass_ng_launch<MixDst<384, R>>(ngy, pl, in, out, ng, nbatch, mult(MULT_LAPINV, 1, 0)); break;
                    default: ypass_ng_launch<GenericDst<R>>(ngy, pl, in, out, ng, nbatch, mult(MULT_LAPINV, 1, 0)); break;
                }
                CK(cudaGetLastError());
            };
            // a block of NG line pairs must fit the shared memory a block may use
            const size_t need = (size_t)ngy * (size_t)(pl.M + 1 + (pl.M + 1) / 16 + 1) * 2 * sizeof(R) + 16 * 8 * ngy;
            if (need > 220 * 1024) continue;
            run();
            run();
            CK(cudaEventRecord(e0, st));
            for (int k = 0; k < 5; ++k) run();
            CK(cudaEventRecord(e1, st));
            CK(cudaEventSynchronize(e1));
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, e0, e1));
            if (ms < best) {
                best = ms;
                best_ng = ngy;
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        tune_table().put(key, best_ng);
    }
    // Y pass with NGY line pairs (2 NGY columns) per block.  Launches over many
    // fields (the B assembly) have waves to spare, and wider blocks read longer
    // segments of each row.
    template <class D, int NGY>
    void ypass_launch(const PlanT<typename D::Real> &pl, const typename D::Real *in, typename D::Real *out, long long bs,
                      int nbatch, Mult m) {
        const dim3 grid((nx - 1 + 2 * NGY - 1) / (2 * NGY), nbatch);
        const size_t sm = pass_smem<D>(pl.M, NGY, NGY);
        if (sm > 48 * 1024) {
            // one M per compile-time transform, so one size; the attribute is per device
            static std::atomic<unsigned long long> attr_devices{0};
            if (need_attr(attr_devices)) {
                CK(cudaFuncSetAttribute(ypass_kernel<D, NGY>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
                attr_devices.fetch_or(device_bit());
            }
        }
        ypass_kernel<D, NGY><<<grid, NGY * D::TPF, sm, st>>>(in, out, bs, nx - 1, pl, m);
    }
    template <class R = T>
    void ypass(const R *in, R *out, long long bs, int nbatch, Mult m) {
        const PlanT<R> &pl = plan_y<R>();
        const int pe = prof_begin();
        switch (pl.M) {
            case 1024: ypass_t<Pow2Dst<1024, R>>(pl, in, out, bs, nbatch, m); break;
            case 512: ypass_t<Pow2Dst<512, R>>(pl, in, out, bs, nbatch, m); break;
            case 256: ypass_t<Pow2Dst<256, R>>(pl, in, out, bs, nbatch, m); break;
            case 384: ypass_t<MixDst<384, R>>(pl, in, out, bs, nbatch, m); break;
            default: ypass_t<GenericDst<R>>(pl, in, out, bs, nbatch, m); break;
        }
        check_launch();
        prof_end(pe, IBPM_KCLASS_YPASS, 2.0 * sizeof(R) * (double)ng * nbatch);
    }
    // transform tables of element type R: the engine's own, or FP64 ones kept by
    // the FP32 engine for its level-1 solve
    PlanT<double> plx_d{}, ply_d{};
    template <class R>
    const PlanT<R> &plan_x() const {
        if constexpr (std::is_same<R, T>::value) return plx; else return plx_d;
    }
    template <class R>
    const PlanT<R> &plan_y() const {
        if constexpr (std::is_same<R, T>::value) return ply; else return ply_d;
    }
    double *psi1_hi = nullptr, *qs1_hi = nullptr, *t1_hi = nullptr, *t2_hi = nullptr;
    // Merged trial solve over all L levels: Gamma_new = Ainv(A Gamma + rest)
    // nb batches of ng (L for one case; cases x L for an ensemble group, whose
    // per-batch coefficients dt / (2 Re hc^2) come from ctab)
    // The merged trial solve on fields of element type R, with scratch t1_, t2_,
    // rhs_ (nb fields each) and the plans of R: the first X pass and the Y pass
    // each take the compile-time transform of their own length (nx and ny may
    // differ), then the plain X pass.
    template <class D, class R = typename D::Real>
    void trial_xpart(const R *Gold, const R *rest_, int nb, R *t1_, R *t2_, const PlanT<R> &px) {
        const dim3 grid((ny - 1 + kNG - 1) / kNG, nb);
        const size_t sm = pass_smem<D>(px.M, kNG, kNG);
        const int pe = prof_begin();
        xpass_trial_kernel<D, kNG><<<grid, kNG * D::TPF, sm, st>>>(Gold, rest_, t1_, t2_, ng, nx - 1, px, ny - 1);
        check_launch();
        prof_end(pe, IBPM_KCLASS_XTRIAL, 4.0 * sizeof(R) * (double)ng * nb);
    }
    template <class D, int NG = kNG, class R = typename D::Real>
    void trial_ypart(int nb, const double *ctab, R *t1_, R *t2_, R *rhs_, const PlanT<R> &py) {
        // many fields per launch (ensemble groups) take 2 NG columns per block
        if constexpr (NG == kNG) {
            if (nb >= 16 && py.M <= 512) {
                trial_ypart<D, 2 * kNG>(nb, ctab, t1_, t2_, rhs_, py);
                return;
            }
        }
        const dim3 grid((nx - 1 + 2 * NG - 1) / (2 * NG), nb);
        const size_t sm = pass_smem<D>(py.M, 2 * NG, NG);
        // the cap must cover the largest M this instantiation serves (kMaxM); the
        // attribute is per device
        static std::atomic<unsigned long long> attr_devices{0};
        if (need_attr(attr_devices)) {
            const int cap = (int)pass_smem<D>(kMaxM, 2 * NG, NG);
            CK(cudaFuncSetAttribute(ypass_trial_kernel<D, NG>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap));
            attr_devices.fetch_or(device_bit());
        }
        const int pe = prof_begin();
        Mult m = mult(MULT_AIMPL, 1, 1);
        m.coef_tab = ctab;
        ypass_trial_kernel<D, NG><<<grid, NG * D::TPF, sm, st>>>(t1_, t2_, rhs_, ng, nx - 1, py, m);
        check_launch();
        prof_end(pe, IBPM_KCLASS_YTRIAL, 3.0 * sizeof(R) * (double)ng * nb);
    }
    template <class R>
    void trial_core(const R *Gold, const R *rest_, R *Gnew, int nb, const double *ctab, R *t1_, R *t2_, R *rhs_,
                    const PlanT<R> &px, const PlanT<R> &py) {
        switch (px.M) {
            case 1024: trial_xpart<Pow2Dst<1024, R>>(Gold, rest_, nb, t1_, t2_, px); break;
            case 512: trial_xpart<Pow2Dst<512, R>>(Gold, rest_, nb, t1_, t2_, px); break;
            case 256: trial_xpart<Pow2Dst<256, R>>(Gold, rest_, nb, t1_, t2_, px); break;
            case 384: trial_xpart<MixDst<384, R>>(Gold, rest_, nb, t1_, t2_, px); break;
            default: trial_xpart<GenericDst<R>>(Gold, rest_, nb, t1_, t2_, px); break;
        }
        switch (py.M) {
            case 1024: trial_ypart<Pow2Dst<1024, R>>(nb, ctab, t1_, t2_, rhs_, py); break;
            case 512: trial_ypart<Pow2Dst<512, R>>(nb, ctab, t1_, t2_, rhs_, py); break;
            case 256: trial_ypart<Pow2Dst<256, R>>(nb, ctab, t1_, t2_, rhs_, py); break;
            case 384: trial_ypart<MixDst<384, R>>(nb, ctab, t1_, t2_, rhs_, py); break;
            default: trial_ypart<GenericDst<R>>(nb, ctab, t1_, t2_, rhs_, py); break;
        }
        xpass<R>(InPlain<R>{rhs_, ng, nx - 1}, OutPlain<R>{Gnew, ng, nx - 1}, nb);
    }
    // the merged trial solve of one FP64 level (IBPM_MIXED_L1's level 1)
    void trial_d(const double *Gold, const double *rest_, double *Gnew) {
        trial_core<double>(Gold, rest_, Gnew, 1, nullptr, t1d, t2d, rhsd, plan_x<double>(), plan_y<double>());
    }
    // Merged trial solve over all L levels: Gamma_new = Ainv(A Gamma + rest)
    // nb batches of ng (L for one case; cases x L for an ensemble group, whose
    // per-batch coefficients dt / (2 Re hc^2) come from ctab)
    void trial(const T *Gold, const T *rest_, T *Gnew, int nb = 0, const double *ctab = nullptr) {
        if (nb == 0) nb = L;
        trial_core<T>(Gold, rest_, Gnew, nb, ctab, t1, t2, rhs, plx, ply);
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
        m.coef_tab = nullptr;
        return m;
    }
    InPlain<T> in_plain(const T *p, long long bs) const { return InPlain<T>{p, bs, nx - 1}; }
    OutPlain<T> out_plain(T *p, long long bs) const { return OutPlain<T>{p, bs, nx - 1}; }

    // The tensor-core transforms for nf fields of nprod products: creates (or
    // re-creates) the plan and the level-1 multiplier tables outside any capture.
    // A new plan has new buffers, so the captured B rebuild is dropped.
    void tc_prepare(int nf, int nprod) {
        if (tc && tc_nprod(tc) == nprod && tc_fmax(tc) >= nf) return;
        CK(cudaStreamSynchronize(st));
        if (tc) {
            tc_destroy(tc);
            tc = nullptr;
        }
        if (binv_exec) cudaGraphExecDestroy(binv_exec);
        if (binv_graph) cudaGraphDestroy(binv_graph);
        binv_exec = nullptr;
        binv_graph = nullptr;
        const char *why = "tensor-core transforms unavailable";
        tc = tc_create(nx, nf, nprod, &why);
        if (!tc) {
            (void)cudaGetLastError();
            throw ApiError{IBPM_ERR_INVALID, why};
        }
        for (int k = 0; k < 2; ++k)
            if (!tc_mult[k]) {
                tc_mult[k] = dalloc<float>((size_t)nx * nx);
                tc_mult_table(k == 0 ? MULT_LAPINV : MULT_AIMPL, 1, tc_mult[k]);
            }
    }
    void tc_mult_table(int mode, int level, float *tab) {
        tc_mult_kernel<<<dim3((nx + 127) / 128, nx), 128, 0, st>>>(mult(mode, level, 0), nx, tab);
        check_launch();
    }
    // One batched solve x = S(m S(b)) on the tensor cores: b from the solve's
    // prologue `in` (the first X pass's input), x to out (batch stride bs), the
    // elements `keep` selects
    template <class In>
    void tc_solve(const In &in, int nf, const float *mtab, double *out, long long bs,
                  TcKeep keep = TcKeep{TC_KEEP_ALL, nullptr, {0, 0, 0, 0}}) {
        if (!tc || tc_fmax(tc) < nf) throw ApiError{IBPM_ERR_INVALID, "tensor-core transforms not prepared"};
        int pe = prof_begin();
        tc_lines_kernel<In><<<dim3(1, nx, nf), nx / 8, nx * sizeof(double), st>>>(in, nx, tc_in_hi(tc), tc_in_lo(tc));
        check_launch();
        const double P = nx, parts = tc_nprod(tc) == 3 ? 2 : 1;
        prof_end(pe, IBPM_KCLASS_TCLINES, (8.0 * ng + 2.0 * parts * P * P) * nf);
        pe = prof_begin();
        launches += tc_solve_tail(tc, nf, mtab, out, bs, nx - 1, keep, err + 4, st);
        CK(cudaGetLastError());
        // four passes of nprod half-length products: 4 nprod P^3 flops per field
        prof_end(pe, IBPM_KCLASS_TCDST, 4.0 * tc_nprod(tc) * P * P * P * nf);
    }

    // vort2flux (src/fluid.jl:178-205) over nbatch independent fields.
    // G, psi: level 1 of batch 0, level stride ng, batch stride bs.
    // qout: level 1 of batch 0 (level stride nq, batch stride qbs); curl_all=false
    // computes q only at level 1 (the only level a caller reads).  win (device,
    // with curl_all=false): the level-1 faces the caller reads (E's support, the
    // body's bbox); level 1's last X pass and curl then skip what lies outside,
    // leaving those rows of psi and faces of q unwritten.  central: the coarse
    // levels of Gm hold zeros outside the central block that coarsify! writes
    // (a B application's vorticity), so their prologues and coarsening skip the
    // loads there; the results are the same bits.
    void vort2flux(T *psi_, T *qout, T *Gm, long long bs, long long qbs, int nbatch, bool curl_all,
                   bool hi1 = false, const int *win = nullptr, bool central = false) {
        if (curl_all) win = nullptr;
        for (int lev = 2; lev <= L; ++lev) {
            const int nx2 = nx / 2, ny2 = ny / 2;
            const dim3 blk(16, 16), grd((nx2 + 15) / 16, (ny2 + 15) / 16, nbatch);
            coarsify_kernel<<<grd, blk, 0, st>>>(Gm + (lev - 1) * ng, Gm + (lev - 2) * ng, bs, g,
                                                 central && lev - 1 >= 2 ? 1 : 0);
            check_launch();
        }
        // the central block coarsify! writes (faces nx/4+1 .. 3nx/4-1 by ny/4+1 .. 3ny/4-1)
        auto centred = [&](const auto &in) {
            using In = std::decay_t<decltype(in)>;
            return InCentral<In>{in, nx / 4 + 1, 3 * nx / 4 - 1, ny / 4 + 1, 3 * ny / 4 - 1};
        };
        for (int lev = L; lev >= 1; --lev) {
            T *Gl = Gm + (lev - 1) * ng;
            T *Pl = psi_ + (lev - 1) * ng;
            if (lev == 1 && hi1) {
                // level 1 in FP64 from the FP32 coarser levels: psi1_hi and qs1_hi (x E),
                // batch strides ng and nq
                const T *coarse = L > 1 ? psi_ + ng : nullptr;
                if (coarse)
                    xpass<double>(InBC<T>{Gl, coarse, bs, bs, g}, OutPlain<double>{t1_hi, ng, nx - 1}, nbatch);
                else
                    xpass<double>(in_plain(Gl, bs), OutPlain<double>{t1_hi, ng, nx - 1}, nbatch);
                ypass<double>(t1_hi, t2_hi, ng, nbatch, mult(MULT_LAPINV, 1, 0));
                xpass<double>(InPlain<double>{t2_hi, ng, nx - 1}, OutPlain<double>{psi1_hi, ng, nx - 1}, nbatch);
                const dim3 blk(64, 4);
                const dim3 grd((nx + 1 + 63) / 64, (ny + 1 + 3) / 4, nbatch);
                curl_kernel<double, double, T><<<grd, blk, 0, st>>>(qs1_hi, nq, psi1_hi, ng, coarse, bs, g);
                check_launch();
                continue;
            }
            bool solved = false;
            if constexpr (std::is_same<T, double>::value) {
                if (tc_on) {
                    // coarse levels: only the lines the next finer level's boundary
                    // values read; level 1: the curl's window
                    TcKeep keep{TC_KEEP_LINES, nullptr, {ny / 4 - 1, 3 * ny / 4 - 1, nx / 4 - 1, 3 * nx / 4 - 1}};
                    if (lev == 1) keep = win ? TcKeep{TC_KEEP_WINDOW, win, {0, 0, 0, 0}} : TcKeep{TC_KEEP_ALL, nullptr, {0, 0, 0, 0}};
                    const bool cen = central && lev >= 2;
                    if (lev == L) {
                        if (cen)
                            tc_solve(centred(in_plain(Gl, bs)), nbatch, tc_mult[0], Pl, bs, keep);
                        else
                            tc_solve(in_plain(Gl, bs), nbatch, tc_mult[0], Pl, bs, keep);
                    } else {
                        const InBC<T> in{Gl, psi_ + lev * ng, bs, bs, g};
                        if (cen)
                            tc_solve(centred(in), nbatch, tc_mult[0], Pl, bs, keep);
                        else
                            tc_solve(in, nbatch, tc_mult[0], Pl, bs, keep);
                    }
                    solved = true;
                }
            }
            if (!solved) {
                bool cen = false;
                if constexpr (std::is_same<T, double>::value) cen = central && lev >= 2;
                if (lev == L) {
                    if constexpr (std::is_same<T, double>::value)
                        if (cen) xpass(centred(in_plain(Gl, bs)), out_plain(t1, ng), nbatch);
                    if (!cen) xpass(in_plain(Gl, bs), out_plain(t1, ng), nbatch);
                } else {
                    const InBC<T> in{Gl, psi_ + lev * ng, bs, bs, g};
                    if constexpr (std::is_same<T, double>::value)
                        if (cen) xpass(centred(in), out_plain(t1, ng), nbatch);
                    if (!cen) xpass(in, out_plain(t1, ng), nbatch);
                }
                ypass(t1, t2, ng, nbatch, mult(MULT_LAPINV, 1, 0));
                xpass(in_plain(t2, ng), out_plain(Pl, bs), nbatch, lev == 1 ? win : nullptr);
            }
            if (curl_all || lev == 1) {
                const dim3 blk(64, 4);
                // with a window and many fields the blocks sweep it (128 x 128 faces per
                // sweep); a few fields keep one thread per face of the whole grid
                const bool windowed = lev == 1 && win != nullptr && nbatch > 4;
                const dim3 grd(windowed ? std::min(2, (nx + 1 + 63) / 64) : (nx + 1 + 63) / 64,
                               windowed ? std::min(32, (ny + 1 + 3) / 4) : (ny + 1 + 3) / 4, nbatch);
                const int pe = prof_begin();
                curl_kernel<T, T, T><<<grd, blk, 0, st>>>(qout + (lev - 1) * nq, qbs, Pl, bs,
                                                          lev < L ? psi_ + lev * ng : nullptr, bs, g,
                                                          lev == 1 ? win : nullptr);
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
        InRegRot<T> in{Patch<T>{patch, P.bbox, patch_stride}};
        bool solved = false;
        if constexpr (std::is_same<T, double>::value) {
            if (tc_on) {
                tc_solve(in, nbatch, tc_mult[1], Gw, ng * L);
                solved = true;
            }
        }
        if (!solved) {
            xpass(in, out_plain(t1, ng), nbatch, P.bbox, 1);  // rot of the patch: zero outside its rows
            ypass(t1, t2, ng, nbatch, mult(MULT_AIMPL, 1, 0));
            // Gw's levels 2..L hold the level-1 vorticity coarsified and zeros elsewhere:
            // vort2flux's coarsify rewrites their central block, and nothing else ever
            // writes them, so the zeros of the allocation stay
            xpass(in_plain(t2, ng), out_plain(Gw, ng * L), nbatch);
        }
        // E reads the bbox only; Gw's coarse levels are zero outside coarsify!'s block
        vort2flux(psiw, qw, Gw, ng * L, nq, nbatch, false, false, P.bbox, true);
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
        cg_collect();
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


    // ---- FP32/FP64 conversions for state transfers ----
    double *staging(size_t n) {
        if (n > stage_len) {
            stage = dalloc<double>(n);
            stage_len = n;
        }
        return stage;
    }
    void upload(T *dst, const double *src, size_t n);
    void download(double *dst, const T *src, size_t n);

    void init(const ibpm_problem *p, const ibpm_options &o);
    bool hi_level1 = false;
    // IBPM_MIXED_L1: level 1 (the body's level) kept and solved in FP64 (G1, q1,
    // psi1, nl1 and FP64 scratch); the float arrays hold levels 2..L
    bool l1d = false;
    double *G1[2] = {nullptr, nullptr}, *nl1[2] = {nullptr, nullptr};
    double *q1 = nullptr, *psi1 = nullptr, *rest1 = nullptr, *t1d = nullptr, *t2d = nullptr, *rhsd = nullptr;
    double *patch_d = nullptr, *q0d = nullptr, *coef_coarse = nullptr;
    void step_body_l1d();
    void vort2flux_l1d(const double *G1v, T *Gm, T *qout, double *psi1_out, double *q1_out, bool curl_all);
    ibpm_problem problem_copy{};
    T *diag_q = nullptr, *diag_g = nullptr;  // diag_vort2flux buffers
    void set_state(const ibpm_state_view *s) override;
    void get_field(int field, int level, double *out) override;
    double *field_d = nullptr;  // one level of an output field
    void set_warm_start(ibpm_net *net, int mode, int depth) override;
    void set_rebuild_transform(int products) override;
    void warm_start_sample(float *features, float *target, float *prediction) override;
    void get_state(ibpm_state_view *s) override;
    bool advance(int64_t nsteps, const ibpm_step_params *params) override;
    void enqueue_step(const ibpm_step_params &prm) override {
        CK(cudaSetDevice(device));
        step(prm);
    }
    bool finish_steps() override {
        CK(cudaSetDevice(device));
        CK(cudaStreamSynchronize(st));
        cg_collect();
        const bool m = cg_hit_maxiter;
        cg_hit_maxiter = false;
        return m;
    }
    void get_forces(double *fb, double *total) override;
    void get_time(int64_t *index, double *t) override;
    void get_info(ibpm_info *info) override;
    void *stream_ptr() override { return (void *)st; }
    long long launch_count() const override { return launches; }
    void set_profile(int enable) override;
    void read_profile(int kclass, int64_t *launches, double *ms, double *bytes) override;
    void diag_solve(int op, int level, const double *b, double *x) override;
    void diag_apply_B(const double *z, double *x) override;
    void diag_binv(double *out) override;
    void diag_vort2flux(double *gamma, double *psi, double *q) override;
    void diag_reg(const double *f, double *gamma1, const double *q1, double *fout) override;
    void setup();
    void build_Binv();
    void assemble_invert_B();
    void direct_rebuild();
    int batch_width() const;
    void cg(double *x, const double *b, bool have_bx = false, bool precond = false, const double *rref = nullptr);
    void cg_collect();
    int *cg_it = nullptr;
    bool cg_pending = false, cg_hit_maxiter = false;
    cudaStream_t st_side = nullptr;
    void step(const ibpm_step_params &prm_in);
    void step_body();
    // CUDA graphs of step_body (static bodies), one per buffer parity
    bool use_graphs = true;
    cudaGraph_t graph[2] = {nullptr, nullptr};
    cudaGraphExec_t graph_exec[2] = {nullptr, nullptr};
    long long graph_launches[2] = {0, 0};
    void materialise_q0();
};

template <class T>
void Engine<T>::setup() {
    CK(cudaSetDevice(device));
    if (const char *e = getenv("IBPM_NO_GRAPHS")) use_graphs = e[0] == '0';
    {
        cudaDeviceProp pr{};
        CK(cudaGetDeviceProperties(&pr, device));
        devname = pr.name;
    }
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    if (!make_plan(nx, plx) || !make_plan(ny, ply))
        throw ApiError{IBPM_ERR_INVALID, "nx and ny must be even, <= 1024 and of the form 2^a 3^b 5^c"};
    // transform tables
    auto tables = [&](int M, C *&tw, T *&sn, double *&cs, PlanT<T> &pl) {
        std::vector<C> htw(M);
        std::vector<T> hsn(M + 1);
        std::vector<double> hcs(M + 1);
        for (int k = 0; k < M; ++k) {
            const long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)k / (long double)M;
            htw[k] = Cx<T>::make((T)cosl(a), (T)sinl(a));
        }
        for (int j = 0; j <= M; ++j) {
            hsn[j] = (T)sinl(3.14159265358979323846264338327950288L * (long double)j / (long double)M);
            hcs[j] = cos(M_PI * j / M);  // _lap_eigs uses cos(pi * i / nx) in Float64
        }
        tw = dalloc<C>(M);
        sn = dalloc<T>(M + 1);
        cs = dalloc<double>(M + 1);
        CK(cudaMemcpyAsync(tw, htw.data(), sizeof(C) * M, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(sn, hsn.data(), sizeof(T) * (M + 1), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(cs, hcs.data(), sizeof(double) * (M + 1), cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
        pl.tw = tw;
        pl.sn = sn;
    };
    tables(nx, twx, snx, cx, plx);
    tables(ny, twy, sny, cy, ply);
    if (!std::is_same<T, double>::value) {
        hi_level1 = true;
        if (const char *e = getenv("IBPM_FP32_LEVEL1")) hi_level1 = e[0] != '0';
        if (!make_plan(nx, plx_d) || !make_plan(ny, ply_d)) throw ApiError{IBPM_ERR_INVALID, "bad transform size"};
        auto dtables = [&](int M, PlanT<double> &pl) {
            std::vector<double2> htw(M);
            std::vector<double> hsn(M + 1);
            for (int k = 0; k < M; ++k) {
                const long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)k / (long double)M;
                htw[k] = make_double2((double)cosl(a), (double)sinl(a));
            }
            for (int j = 0; j <= M; ++j)
                hsn[j] = (double)sinl(3.14159265358979323846264338327950288L * (long double)j / (long double)M);
            double2 *tw = dalloc<double2>(M);
            double *sn = dalloc<double>(M + 1);
            CK(cudaMemcpyAsync(tw, htw.data(), sizeof(double2) * M, cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(sn, hsn.data(), sizeof(double) * (M + 1), cudaMemcpyHostToDevice, st));
            CK(cudaStreamSynchronize(st));
            pl.tw = tw;
            pl.sn = sn;
        };
        dtables(nx, plx_d);
        dtables(ny, ply_d);
        psi1_hi = dalloc<double>(ng);
        qs1_hi = dalloc<double>(nq);
        t1_hi = dalloc<double>(ng);
        t2_hi = dalloc<double>(ng);
        l1d = opt.precision == IBPM_MIXED_L1;
        if (l1d) {
            if (!static_bodies)
                throw ApiError{IBPM_ERR_INVALID, "the level-1-FP64 mixed precision needs static bodies"};
            for (int k = 0; k < 2; ++k) {
                G1[k] = dalloc<double>(ng);
                nl1[k] = dalloc<double>(ng);
            }
            q1 = dalloc<double>(nq);
            psi1 = dalloc<double>(ng);
            rest1 = dalloc<double>(ng);
            t1d = dalloc<double>(ng);
            t2d = dalloc<double>(ng);
            rhsd = dalloc<double>(ng);
            q0d = dalloc<double>(nq);
            patch_d = dalloc<double>(2LL * (nx + 1) * (ny + 1));
            // dt / (2 Re hc^2) of levels 2..L, as Mult::coef forms it on the device
            std::vector<double> cc(std::max(L - 1, 1), 0.0);
            for (int lev = 2; lev <= L; ++lev) {
                const double hc = ldexp(g.h, lev - 1);
                cc[lev - 2] = g.dt / (2 * g.Re * (hc * hc));
            }
            coef_coarse = dalloc<double>(cc.size());
            CK(cudaMemcpyAsync(coef_coarse, cc.data(), sizeof(double) * cc.size(), cudaMemcpyHostToDevice, st));
        }
    }

    q = dalloc<T>(nq * L);
    psi = dalloc<T>(ng * L);
    G[0] = dalloc<T>(ng * L);
    G[1] = dalloc<T>(ng * L);
    nl[0] = dalloc<T>(ng * L);
    nl[1] = dalloc<T>(ng * L);
    P.np = np;
    P.xb = dalloc<double>(2 * np);
    P.ub = dalloc<double>(2 * np);
    P.pc = dalloc<int>(2 * np);
    P.w = dalloc<double>((size_t)np * 2 * 49);
    P.bbox = dalloc<int>(4);
    err = dalloc<int>(8);
    P.err = err;
    ref_xb_d = dalloc<double>(2 * np);
    ds = dalloc<double>(np);
    Fbt = dalloc<double>(2 * np);
    fb = dalloc<double>(2 * np);
    total = dalloc<double>(2);
    prm = dalloc<StepDev>(1);
    motion = dalloc<double>(6 * (size_t)std::max(nbody, 1));
    for (int k = 0; k < kStage; ++k) {
        CK(cudaMallocHost(&stage_prm[k], sizeof(StepDev)));
        CK(cudaMallocHost(&stage_motion[k], sizeof(double) * 6 * std::max(nbody, 1)));
        CK(cudaEventCreateWithFlags(&stage_ev[k], cudaEventDisableTiming));
        memset(stage_prm[k], 0, sizeof(StepDev));
    }
    prm_h = stage_prm[0];
    motion_h = stage_motion[0];
    CK(cudaMallocHost(&cg_s_h, sizeof(double) * 8));
    CK(cudaMallocHost(&err_h, sizeof(int) * 8));
    memset(prm_h, 0, sizeof(StepDev));
    CK(cudaMemcpyAsync(ref_xb_d, ref_xb.data(), sizeof(double) * 2 * np, cudaMemcpyHostToDevice, st));

    kbatch = batch_width();
    if (!std::is_same<T, double>::value) kbatch = 1;  // FP32 builds B^-1 with an FP64 engine
    if (!static_bodies) kbatch = 2;  // the warm start applies B to two vectors at once
    kbatch = std::min(kbatch, 2 * np);
    const int kb = std::max(kbatch, L);
    t1 = dalloc<T>(ng * kb);
    t2 = dalloc<T>(ng * kb);
    rhs = dalloc<T>(ng * L);
    rest = dalloc<T>(ng * L);
    qs1 = dalloc<T>(nq);
    Ftmp = dalloc<double>(2 * np);
    if (!static_bodies) {
        Fprev = dalloc<double>(2 * np);
        ws_z = dalloc<double>(4 * (size_t)np);
        ws_bz = dalloc<double>(4 * (size_t)np);
        ws_x2 = dalloc<double>(4 * (size_t)np + 1);  // [x_e | p | |r|]
        ws_bx2 = dalloc<double>(4 * (size_t)np);
        ws_feat = dalloc<float>((size_t)kWsFeatures * np);
        ws_y = dalloc<float>((size_t)kWsOutputs * np);
        pbody_d = dalloc<int>(np);
        std::vector<int> pb(np, 0);
        for (int b = 0; b < nbody; ++b)
            for (int k = body_start[b]; k < body_start[b + 1]; ++k) pb[k] = b;
        CK(cudaMemcpyAsync(pbody_d, pb.data(), sizeof(int) * np, cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
    }
    const int nchunk = (2 * np + 63) / 64;
    part = dalloc<double>((size_t)nchunk * 2 * np);
    patch_stride = 2LL * (nx + 1) * (ny + 1);
    patch = dalloc<T>(patch_stride * kbatch);
    Gw = dalloc<T>(ng * L * kbatch);
    psiw = dalloc<T>(ng * L * kbatch);
    qw = dalloc<T>(nq * kbatch);
    fcol = dalloc<double>(2 * (size_t)np * kbatch);
    cg_u = dalloc<double>(2 * np);
    cg_z = dalloc<double>(2 * np);
    cg_r = dalloc<double>(2 * np);
    cg_c = dalloc<double>(2 * np);
    cg_s = dalloc<double>(16);
    cg_it = dalloc<int>(4);
    CK(cudaStreamCreateWithFlags(&st_side, cudaStreamNonBlocking));

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
    // pass shapes for one level and for all levels at once (scratch t1 -> t2)
    tune_ypass<T>(t1, t2, 1);
    if (L > 1) tune_ypass<T>(t1, t2, L);
    if (static_bodies) {
        compute_bbox();
        if (std::is_same<T, double>::value) {
            if (kbatch > L) tune_ypass<T>(Gw, psiw, kbatch);
            build_Binv();
            shrink_batch_buffers();
        } else {
            // B and B^-1 in FP64 with a temporary FP64 engine of the same problem;
            // only the (2np)^2 matrix is kept.
            Engine<double> e64;
            ibpm_options o64 = opt;
            o64.precision = IBPM_FP64;
            e64.init(&problem_copy, o64);
            e64.setup();
            const size_t n = 2 * (size_t)np;
            Binv = dalloc<double>(n * n);
            CK(cudaStreamSynchronize(st));
            CK(cudaMemcpy(Binv, e64.Binv, sizeof(double) * n * n, cudaMemcpyDeviceToDevice));
        }
    }
    CK(cudaStreamSynchronize(st));
}

// Columns of B applied at once when B is assembled: about 4 GB of column work.
template <class T>
int Engine<T>::batch_width() const {
    const long long per_col = (2 * ng * L + nq + 2 * ng) * (long long)sizeof(T);
    return (int)std::min<long long>(2 * np, std::max(1LL, std::min<long long>(64, (4LL << 30) / per_col)));
}

// _Binv_precomputed (src/coupling.jl:187-192): B column by column, then its inverse.
template <class T>
void Engine<T>::build_Binv() {
    const int n = 2 * np;
    Binv = dalloc<double>((size_t)n * n);
    Bwork = dalloc<double>((size_t)n * n);
    assemble_invert_B();
    CK(cudaMemcpyAsync(err_h, err, sizeof(int) * 2, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    dfree(Bwork);
    Bwork = nullptr;
    if (err_h[1] != 0) throw ApiError{IBPM_ERR_INVALID, "B is not positive definite (pivot " + std::to_string(err_h[1]) + ")"};
}

// B of the current body position into Binv, kbatch columns per batched
// application, then inverted by Gauss-Jordan elimination without pivoting
// between Binv and Bwork (the symmetric part of B is positive definite; with
// nested levels B itself is not exactly symmetric); a pivot <= 0 sets err[1].
template <class T>
void Engine<T>::assemble_invert_B() {
    const int n = 2 * np;
    const bool rebuilding = uses_binv_start();
    // the preconditioned modes may assemble with the tensor-core transforms
    tc_on = tc_prod > 0 && preconditioned() && tc != nullptr;
    const bool assembled_tc = tc_on;
    try {
        for (int c0 = 0; c0 < n; c0 += kbatch) {
            const int nb = std::min(kbatch, n - c0);
            unit_columns_kernel<<<(n * nb + 255) / 256, 256, 0, st>>>(fcol, n, c0, nb);
            check_launch();
            apply_B(fcol, Binv + (size_t)c0 * n, n, nb);
        }
    } catch (...) {
        tc_on = false;
        throw;
    }
    tc_on = false;
    // n = 2 np is even: n / 2 two-step launches, or for the moving-body rebuilds
    // (rebuilding) kGJB steps per launch as one block pivot; after an odd count
    // of launches the result is in Bwork
    int m = 0;
    const int step = rebuilding ? kGJB : 2;
    for (int k = 0; k < n; k += step, ++m) {
        const double *src = (m & 1) ? Bwork : Binv;
        double *dst = (m & 1) ? Binv : Bwork;
        if (rebuilding)
            gj_block_kernel<<<dim3((n + 255) / 256, n), 256, 0, st>>>(src, dst, n, k, std::min(step, n - k), err + 1);
        else
            gj_step2_kernel<<<dim3((n + 255) / 256, n), 256, 0, st>>>(src, dst, n, k, err + 1);
        check_launch();
    }
    if (m & 1) CK(cudaMemcpyAsync(Binv, Bwork, sizeof(double) * (size_t)n * n, cudaMemcpyDeviceToDevice, st));
    // a B assembled on the tensor cores is nonsymmetric at its rounding level
    // (1e-5 .. 1e-2); conjugate gradients wants a symmetric preconditioner, so
    // its inverse is replaced by the symmetric part (M + M^T) / 2
    if (assembled_tc) {
        symmetrize_kernel<<<dim3((n + 255) / 256, n), 256, 0, st>>>(Binv, n);
        check_launch();
    }
}

// IBPM_WS_DIRECT's rebuild of B^-1 for the body position of this step, as a graph
// captured on first use (its buffers stay fixed until drop_graphs).
template <class T>
void Engine<T>::direct_rebuild() {
    if (tc_prod > 0 && preconditioned()) tc_prepare(kbatch, tc_prod);
    if (!use_graphs || prof) {
        assemble_invert_B();
        return;
    }
    if (!binv_exec) {
        const long long l0 = launches;
        CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        try {
            assemble_invert_B();
        } catch (...) {
            cudaGraph_t gdrop = nullptr;
            cudaStreamEndCapture(st, &gdrop);
            if (gdrop) cudaGraphDestroy(gdrop);
            (void)cudaGetLastError();
            launches = l0;
            throw;
        }
        CK(cudaStreamEndCapture(st, &binv_graph));
        CK(cudaGraphInstantiate(&binv_exec, binv_graph, 0));
        binv_graph_launches = launches - l0;
        launches = l0;
    }
    CK(cudaGraphLaunch(binv_exec, st));
    launches += binv_graph_launches;
}

namespace {
// Device-resident CG state: s[0] = ||r||, s[1] = previous ||r||, s[2] = tol,
// s[3] = 1 while iterating; it[0] = iterations; err[2] = 1 on a non-finite residual.
// Preconditioned (pre = 1): s[8] = rho = r . z of the last direction, z = M r in z.
// rref (device, may be null): the residual norm the relative tolerance scales
// instead of ||r0|| (the reference start's, when CG starts elsewhere).
struct CgArgs {
    int n;
    double *x, *r, *u, *c;
    const double *b;
    double *s;
    int *it, *err;
    int maxiter;
    double reltol, abstol;
    int pre;
    double *z;
    const double *rref;
};

__device__ __forceinline__ double cg_block_sum(double v, double *red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[k];
    return t;
}

// r = b - c (c = B x0); u = 0; residual, tol = max(reltol ||r0||, abstol), and the
// loop condition of IterativeSolvers' done(): !(it >= maxiter || ||r|| <= tol).
__global__ void cg_init_kernel(CgArgs a, cudaGraphConditionalHandle h, int use_h) {
    __shared__ double red[32];
    double acc = 0.0;
    for (int k = threadIdx.x; k < a.n; k += blockDim.x) {
        const double v = a.b[k] - a.c[k];
        a.r[k] = v;
        a.u[k] = 0.0;
        acc += v * v;
    }
    const double t = cg_block_sum(acc, red);
    if (threadIdx.x == 0) {
        const double res = sqrt(t);
        const double tol = fmax(a.reltol * (a.rref ? *a.rref : res), a.abstol);
        int cont = !(0 >= a.maxiter || res <= tol);
        if (!isfinite(res)) {
            a.err[2] = 1;
            cont = 0;
        }
        a.s[0] = res;
        a.s[1] = 1.0;
        a.s[2] = tol;
        a.s[3] = cont;
        a.s[4] = res;  // initial residual, for reports
        a.s[8] = 1.0;  // rho before the first direction (u = 0 makes it immaterial)
        a.it[0] = 0;
        if (use_h) cudaGraphSetConditional(h, cont ? 1u : 0u);
    }
}

// IBPM_WS_PRECOND_EXTRAP's start: x0 = Binv b (in x) is kept, and x gets the
// stale error e = F - Binv b of this step extrapolated from the last ones,
// polynomially in time: e1, 2 e1 - e2 or 3 e1 - 3 e2 + e3 as 1, 2 or 3 are valid
// (none right after a rebuild).  stale = [e1 | e2 | e3].
__global__ void stale_start_kernel(double *__restrict__ x, double *__restrict__ x0,
                                   const double *__restrict__ stale, int n, const int *__restrict__ nvalid) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int v = *nvalid;
    const double b0 = x[k];
    x0[k] = b0;
    const double e1 = stale[k], e2 = stale[n + k], e3 = stale[2 * n + k];
    double e = 0.0;
    if (v >= 3)
        e = 3.0 * e1 - 3.0 * e2 + e3;
    else if (v == 2)
        e = 2.0 * e1 - e2;
    else if (v == 1)
        e = e1;
    x[k] = b0 + e;
}
// after CG: e_new = F - x0 enters the ring (e3 <- e2 <- e1 <- e_new), one block
__global__ void stale_update_kernel(const double *__restrict__ f, const double *__restrict__ x0,
                                    double *__restrict__ stale, int n, int *__restrict__ nvalid) {
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        stale[2 * n + k] = stale[n + k];
        stale[n + k] = stale[k];
        stale[k] = f[k] - x0[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) *nvalid = min(*nvalid + 1, 3);
}

// ||b - c|| into *out (one block, the reduction of cg_init_kernel)
__global__ void residual_norm_kernel(const double *__restrict__ b, const double *__restrict__ c, int n,
                                     double *__restrict__ out) {
    __shared__ double red[32];
    double acc = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const double v = b[k] - c[k];
        acc += v * v;
    }
    const double t = cg_block_sum(acc, red);
    if (threadIdx.x == 0) *out = sqrt(t);
}

// u = r + beta u, beta = ||r||^2 / ||r_prev||^2
__global__ void cg_dir_kernel(CgArgs a) {
    const double beta = a.s[0] * a.s[0] / (a.s[1] * a.s[1]);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < a.n; k += gridDim.x * blockDim.x)
        a.u[k] = a.r[k] + beta * a.u[k];
}

// Preconditioned direction (one block): z = M r from binv_gemv_kernel's chunk
// partials, rho = r . z, u = z + (rho / rho_prev) u -- IterativeSolvers' cg
// iteration with a left preconditioner (rho = r . (Pl \ r)); M = B^-1 of a
// recent step.
__global__ void pcg_dir_kernel(CgArgs a, const double *__restrict__ part, int nchunk) {
    __shared__ double red[32];
    __shared__ double beta_s;
    double acc = 0.0;
    for (int k = threadIdx.x; k < a.n; k += blockDim.x) {
        double z = 0.0;
        for (int c = 0; c < nchunk; ++c) z += part[(long long)c * a.n + k];
        a.z[k] = z;
        acc += a.r[k] * z;
    }
    const double rho = cg_block_sum(acc, red);
    if (threadIdx.x == 0) {
        beta_s = rho / a.s[8];
        a.s[8] = rho;
    }
    __syncthreads();
    const double beta = beta_s;
    for (int k = threadIdx.x; k < a.n; k += blockDim.x) a.u[k] = a.z[k] + beta * a.u[k];
}

// alpha = rho / (u . c), rho = ||r||^2 (plain) or r . z (preconditioned);
// x += alpha u; r -= alpha c; new residual and condition
__global__ void cg_update_kernel(CgArgs a, cudaGraphConditionalHandle h, int use_h) {
    __shared__ double red[32];
    __shared__ double alpha_s;
    double acc = 0.0;
    for (int k = threadIdx.x; k < a.n; k += blockDim.x) acc += a.u[k] * a.c[k];
    const double uc = cg_block_sum(acc, red);
    if (threadIdx.x == 0) alpha_s = (a.pre ? a.s[8] : a.s[0] * a.s[0]) / uc;
    __syncthreads();
    const double alpha = alpha_s;
    double rr = 0.0;
    for (int k = threadIdx.x; k < a.n; k += blockDim.x) {
        a.x[k] += alpha * a.u[k];
        const double v = a.r[k] - alpha * a.c[k];
        a.r[k] = v;
        rr += v * v;
    }
    const double t = cg_block_sum(rr, red);
    if (threadIdx.x == 0) {
        const double res = sqrt(t);
        const int it = a.it[0] + 1;
        int cont = !(it >= a.maxiter || res <= a.s[2]);
        if (!isfinite(res)) {
            a.err[2] = 1;
            cont = 0;
        }
        a.s[1] = a.s[0];
        a.s[0] = res;
        a.s[3] = cont;
        a.it[0] = it;
        if (use_h) cudaGraphSetConditional(h, cont ? 1u : 0u);
    }
}
}  // namespace

// IterativeSolvers.jl cg! as called at src/coupling.jl:198-201: plain CG from
// the initial guess x; stops when ||r|| <= max(reltol ||r0||, abstol) or after
// maxiter iterations.  precond: the same iteration with the left
// preconditioner Pl = B of a recent step, applied as z = Binv r (the reference
// passes no Pl; the stopping rule on ||r|| is unchanged).  All scalars live on
// the device.  Inside a stream
// capture the loop is a graph WHILE node whose condition the update kernel
// sets; otherwise the host reads the condition after every iteration.
template <class T>
void Engine<T>::cg(double *x, const double *b, bool have_bx, bool precond, const double *rref) {
    const int n = 2 * np;
    const int nchunk = (n + 63) / 64;
    CgArgs a{n, x, cg_r, cg_u, cg_c, b, cg_s, cg_it, err, opt.cg_maxiter, opt.cg_reltol, opt.cg_abstol, precond ? 1 : 0,
             cg_z, rref};
    // the direction: plain, or preconditioned by Binv (z = Binv r)
    auto direction = [&]() {
        if (precond) {
            binv_gemv_kernel<<<dim3(nchunk, nchunk), 256, 0, st>>>(Binv, cg_r, part, n);
            check_launch();
            pcg_dir_kernel<<<1, 256, 0, st>>>(a, part, nchunk);
        } else {
            cg_dir_kernel<<<(n + 255) / 256, 256, 0, st>>>(a);
        }
        check_launch();
    };
    if (!have_bx) apply_B(x, cg_c, n, 1);  // else cg_c already holds B x
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(st, &cs));
    if (cs == cudaStreamCaptureStatusActive) {
        cudaGraph_t gr = nullptr;
        const cudaGraphNode_t *deps = nullptr;
        size_t ndeps = 0;
        CK(cudaStreamGetCaptureInfo(st, &cs, nullptr, &gr, &deps, &ndeps));
        cudaGraphConditionalHandle hnd;
        CK(cudaGraphConditionalHandleCreate(&hnd, gr, 0, 0));
        cg_init_kernel<<<1, 256, 0, st>>>(a, hnd, 1);
        check_launch();
        CK(cudaStreamGetCaptureInfo(st, &cs, nullptr, &gr, &deps, &ndeps));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = hnd;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        CK(cudaGraphAddNode(&node, gr, deps, ndeps, &cp));
        CK(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
        // capture the loop body into the WHILE node's graph on the side stream
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        cudaStream_t main = st;
        st = st_side;
        try {
            CK(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
            direction();
            apply_B(cg_u, cg_c, n, 1);
            cg_update_kernel<<<1, 256, 0, st>>>(a, hnd, 1);
            check_launch();
            cudaGraph_t out = nullptr;
            CK(cudaStreamEndCapture(st, &out));
        } catch (...) {
            cudaGraph_t out = nullptr;
            cudaStreamEndCapture(st, &out);
            st = main;
            throw;
        }
        st = main;
        return;
    }
    cg_init_kernel<<<1, 256, 0, st>>>(a, 0, 0);
    check_launch();
    for (;;) {
        CK(cudaMemcpyAsync(cg_s_h, cg_s, sizeof(double) * 4, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (cg_s_h[3] == 0.0) break;
        direction();
        apply_B(cg_u, cg_c, n, 1);
        cg_update_kernel<<<1, 256, 0, st>>>(a, 0, 0);
        check_launch();
    }
}

// Reads the last step's CG iteration count and residual (after a stream sync).
template <class T>
void Engine<T>::cg_collect() {
    if (!cg_pending) return;
    CK(cudaMemcpyAsync(cg_s_h, cg_s, sizeof(double) * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(err_h + 2, cg_it, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(err_h + 3, err + 2, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (uses_binv_start()) CK(cudaMemcpyAsync(err_h + 1, err + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (tc) CK(cudaMemcpyAsync(err_h + 4, err + 4, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    cg_pending = false;
    last_cg_iters = err_h[2];
    last_cg_res = cg_s_h[0];
    first_cg_res = cg_s_h[4];
    // projected: directions kept; extrapolated, learned: the Galerkin coefficient
    ws_coef[0] = ws_mode != IBPM_WS_PREVIOUS && !uses_binv_start() ? cg_s_h[5] : 0.0;
    ws_coef[1] = ws_mode == IBPM_WS_LEARNED ? cg_s_h[6] : 0.0;
    if (last_cg_iters >= opt.cg_maxiter) cg_hit_maxiter = true;
    if (uses_binv_start() && err_h[1]) {
        const int k = err_h[1];
        err_h[1] = 0;
        CK(cudaMemsetAsync(err + 1, 0, sizeof(int), st));
        throw ApiError{IBPM_ERR_INVALID, "B is not positive definite (pivot " + std::to_string(k) + ")"};
    }
    if (err_h[3]) {
        CK(cudaMemsetAsync(err + 2, 0, sizeof(int), st));
        throw ApiError{IBPM_ERR_NONFINITE, "non-finite residual in CG"};
    }
    if (tc && err_h[4]) {
        err_h[4] = 0;
        CK(cudaMemsetAsync(err + 4, 0, sizeof(int), st));
        throw ApiError{IBPM_ERR_CUDA, "a tensor-core transform pass gave up waiting for its operands"};
    }
}

// advance!(::CnabSolver) (src/solver.jl:155-190)
template <class T>
void Engine<T>::step(const ibpm_step_params &sp) {
    // inc_time_index! and the host callbacks' values
    ++index;
    stage_acquire();
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
        if (uses_binv_start()) {
            if (ws_since % ws_refresh == 0) {
                direct_rebuild();
                // stale errors refer to the previous inverse
                if (ws_nvalid) CK(cudaMemsetAsync(ws_nvalid, 0, sizeof(int), st));
            }
            ++ws_since;
        }
    }
    stage_release();
    q0_zero = false;
    q0_from_user = false;
    // The rest of the step is one CUDA graph per parity of the ping-ponged
    // Gamma / nonlin buffers (gc == nc always), captured on first use; with
    // moving bodies it holds the CG loop as a WHILE node.
    if (use_graphs && !prof) {
        const int p = gc;
        if (!graph_exec[p]) {
            const int gc0 = gc, nc0 = nc;
            const long long l0 = launches;  // the capture launches nothing
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
                launches = l0;
                throw;
            }
            CK(cudaStreamEndCapture(st, &graph[p]));
            CK(cudaGraphInstantiate(&graph_exec[p], graph[p], 0));
            gc = gc0;
            nc = nc0;
            launches = l0;
        }
        CK(cudaGraphLaunch(graph_exec[p], st));
        launches += graph_launches[p];
        gc = 1 - gc;
        nc = 1 - nc;
        if (static_bodies) last_cg_iters = 0;
        cg_pending = !static_bodies;
        return;
    }
    step_body();
}

// The device work of one step after the per-step parameters are uploaded.
template <class T>
void Engine<T>::step_body() {
    if (l1d) {
        step_body_l1d();
        return;
    }
    const long long launches0 = launches;
    T *Gold = G[gc], *Gnew = G[1 - gc];
    T *N1 = nl[nc], *N2 = nl[1 - nc];
    // get_trial_state (src/fluid.jl:467-506), all levels at once: the levels
    // only read the previous step's Gamma and q.
    {
        NonlinArgs<T> a{q, Gold, N1, N2, rest, prm, g};
        const dim3 blk(kNlTX, kNlBY), grd((nx - 1 + kNlTX - 1) / kNlTX, (ny - 1 + kNlTY - 1) / kNlTY, L);
        const int pe = prof_begin();
        nonlinear_kernel<<<grd, blk, 0, st>>>(a);
        check_launch();
        prof_end(pe, IBPM_KCLASS_NONLINEAR, 8.0 * (double)(nq + 4 * ng) * L);
    }
    trial(Gold, rest, Gnew);
    nc = 1 - nc;  // _cycle!(state.nonlin)
    // couple_surface_rigid (src/coupling.jl:236-250).  The FP32 engine computes the
    // level-1 trial flux that E interpolates in FP64: B^-1 amplifies white noise in
    // E qs by its condition number (1e4..1e5), FP32 rounding would reach the forces.
    if (hi_level1) {
        vort2flux(psi, qs1, Gnew, 0, 0, 1, false, true);
        launch_regT(P, qs1_hi, 0, Ftmp, 0, 1, 1, prm, g, st);
    } else {
        vort2flux(psi, qs1, Gnew, 0, 0, 1, false, false, P.bbox);  // E reads the bbox only
        launch_regT(P, qs1, 0, Ftmp, 0, 1, 1, prm, g, st);
    }
    check_launch();
    const int n = 2 * np;
    if (static_bodies) {
        const int nchunk = (n + 63) / 64;
        binv_gemv_kernel<<<dim3(nchunk, nchunk), 256, 0, st>>>(Binv, Ftmp, part, n);
        check_launch();
        binv_reduce_kernel<<<1, 1024, 0, st>>>(part, nchunk, n, Fbt, fb, total, g.h, g.dt, 1);
        check_launch();
        last_cg_iters = 0;
    } else {
        // CG initial guess.  The reference starts from the previous solution F1
        // (src/coupling.jl:198-201).  The other modes first take the Galerkin step
        // in the B-energy norm along the last change d = F1 - F2 (x_e, from B [F1 | d]
        // in one batched application); the learned mode then maps the residual
        // b - B x_e to a correction p and takes a second Galerkin step along p.
        launch_ws_direction(Fbt, Fprev, np, ws_z, st);
        check_launch();
        if (ws_mode == IBPM_WS_PREVIOUS) {
            cg(Fbt, Ftmp);
        } else if (uses_binv_start()) {
            // x0 = B^-1 b with the inverse of this step's B (or, between rebuilds,
            // of a recent step's); CG then runs from x0, preconditioned by the
            // same inverse in IBPM_WS_PRECONDITIONED.  A relative tolerance keeps
            // the reference's value, reltol ||b - B F1|| with F1 its start (the
            // previous solution): x0's own residual is at rounding level.
            const double *rref = nullptr;
            if (opt.cg_reltol > 0) {
                apply_B(Fbt, cg_c, n, 1);
                residual_norm_kernel<<<1, 256, 0, st>>>(Ftmp, cg_c, n, cg_s + 7);
                check_launch();
                rref = cg_s + 7;
            }
            const int nchunk = (n + 63) / 64;
            binv_gemv_kernel<<<dim3(nchunk, nchunk), 256, 0, st>>>(Binv, Ftmp, part, n);
            check_launch();
            binv_reduce_kernel<<<1, 1024, 0, st>>>(part, nchunk, n, Fbt, fb, total, g.h, g.dt, 1);
            check_launch();
            if (ws_mode == IBPM_WS_PRECOND_EXTRAP) {
                stale_start_kernel<<<(n + 255) / 256, 256, 0, st>>>(Fbt, ws_x0, ws_stale, n, ws_nvalid);
                check_launch();
            }
            cg(Fbt, Ftmp, false, preconditioned(), rref);
            if (ws_mode == IBPM_WS_PRECOND_EXTRAP) {
                stale_update_kernel<<<1, 256, 0, st>>>(Fbt, ws_x0, ws_stale, n, ws_nvalid);
                check_launch();
            }
        } else if (ws_mode == IBPM_WS_PROJECTED) {
            // Galerkin over the last ws_depth solutions, B applied to all in one batch
            apply_B(ws_hist, ws_bhist, 2 * np, ws_depth);
            // slot 0 holds F1, the reference's start: its residual scales reltol
            const double *rref = nullptr;
            if (opt.cg_reltol > 0) {
                residual_norm_kernel<<<1, 256, 0, st>>>(Ftmp, ws_bhist, n, cg_s + 7);
                check_launch();
                rref = cg_s + 7;
            }
            launch_ws_projection(ws_hist, ws_bhist, Ftmp, Fbt, cg_c, 2 * np, ws_depth, ws_G, ws_h, cg_s + 5, st);
            check_launch();
            cg(Fbt, Ftmp, true, false, rref);
            launch_ws_shift(ws_hist, Fbt, 2 * np, ws_depth, st);
            check_launch();
        } else {
            apply_B(ws_z, ws_bz, 2 * np, 2);
            // ws_z's first column is F1, the reference's start: its residual scales reltol
            const double *rref = nullptr;
            if (opt.cg_reltol > 0) {
                residual_norm_kernel<<<1, 256, 0, st>>>(Ftmp, ws_bz, n, cg_s + 7);
                check_launch();
                rref = cg_s + 7;
            }
            launch_ws_galerkin(ws_z, ws_bz, Ftmp, Fbt, cg_c, ws_x2, ws_bx2, np, 1, cg_s + 5, st);
            check_launch();
            launch_ws_features(Ftmp, cg_c, ws_z, ws_z + 2 * np, P.ub, motion, pbody_d, np, ws_feat, ws_x2 + 4 * np,
                               st);
            check_launch();
            if (ws_mode == IBPM_WS_LEARNED) {
                net_forward_dev(ws, ws_feat, 1, np, ws_act, ws_y, st);
                check_launch();
                launch_ws_prediction(ws_y, ws, np, ws_x2 + 2 * np, st);
                check_launch();
                apply_B(ws_x2 + 2 * np, ws_bx2 + 2 * np, 2 * np, 1);
                launch_ws_galerkin(ws_x2, ws_bx2, Ftmp, Fbt, cg_c, nullptr, nullptr, np, 1, cg_s + 6, st);
                check_launch();
            }
            cg(Fbt, Ftmp, true, false, rref);
        }
        cg_pending = true;
        binv_reduce_kernel<<<1, 1024, 0, st>>>(nullptr, 0, n, Fbt, fb, total, g.h, g.dt, 0);
        check_launch();
    }
    // project_circ (src/coupling.jl:218-230): Gamma = Gamma_s; Gamma_1 -= Ainv_1 rot(E^T F~b)
    reg_patch(Fbt, 1);
    xpass(InRegRot<T>{Patch<T>{patch, P.bbox, patch_stride}}, out_plain(t1, ng), 1, P.bbox, 1);
    ypass(t1, t2, ng, 1, mult(MULT_AIMPL, 1, 0));
    xpass(in_plain(t2, ng), OutSub<T>{Gnew, ng, nx - 1}, 1);
    // vort2flux!(state.psi, state.q, state.Gamma)
    vort2flux(psi, q, Gnew, 0, 0, 1, true);
    gc = 1 - gc;
    graph_launches[1 - gc] = launches - launches0;
}

// IBPM_MIXED_L1's step: the body's level (level 1) in FP64 -- its Gamma, flux,
// streamfunction and nonlinear history stored and its solves run in FP64 -- and
// the coarser levels in FP32.  Level 1 feeds E (src/coupling.jl:236-250), whose
// errors B^-1 amplifies, while the coarser levels reach level 1 only through its
// boundary values, a smooth field.  Same sequence as step_body.
template <class T>
void Engine<T>::step_body_l1d() {
    const long long launches0 = launches;
    T *Gold = G[gc], *Gnew = G[1 - gc];
    T *N1 = nl[nc], *N2 = nl[1 - nc];
    double *G1o = G1[gc], *G1n = G1[1 - gc], *N11 = nl1[nc], *N12 = nl1[1 - nc];
    const dim3 blk(kNlTX, kNlBY);
    // nonlinear + rhs assembly (src/fluid.jl:467-493): level 1 in FP64, its coarser
    // level's Gamma in FP32; levels 2..L in FP32
    {
        NonlinArgs<double, T> a{q1, G1o, N11, N12, rest1, prm, g};
        a.coarse = L > 1 ? Gold + ng : nullptr;
        const dim3 grd((nx - 1 + kNlTX - 1) / kNlTX, (ny - 1 + kNlTY - 1) / kNlTY, 1);
        nonlinear_kernel<double, T, true><<<grd, blk, 0, st>>>(a);
        check_launch();
    }
    if (L > 1) {
        NonlinArgs<T> a{q + nq, Gold + ng, N1 + ng, N2 + ng, rest + ng, prm, g};
        a.lev0 = 2;
        const dim3 grd((nx - 1 + kNlTX - 1) / kNlTX, (ny - 1 + kNlTY - 1) / kNlTY, L - 1);
        nonlinear_kernel<T, T, true><<<grd, blk, 0, st>>>(a);
        check_launch();
    }
    trial_d(G1o, rest1, G1n);
    if (L > 1) trial(Gold + ng, rest + ng, Gnew + ng, L - 1, coef_coarse);
    nc = 1 - nc;  // _cycle!(state.nonlin)
    // couple_surface_rigid from the FP64 level-1 trial flux
    vort2flux_l1d(G1n, Gnew, nullptr, psi1_hi, qs1_hi, false);
    launch_regT(P, qs1_hi, 0, Ftmp, 0, 1, 1, prm, g, st);
    check_launch();
    const int n = 2 * np, nchunk = (n + 63) / 64;
    binv_gemv_kernel<<<dim3(nchunk, nchunk), 256, 0, st>>>(Binv, Ftmp, part, n);
    check_launch();
    binv_reduce_kernel<<<1, 1024, 0, st>>>(part, nchunk, n, Fbt, fb, total, g.h, g.dt, 1);
    check_launch();
    last_cg_iters = 0;
    // project_circ (src/coupling.jl:218-230) on the FP64 level 1
    launch_reg_patch<double>(P, Fbt, 2 * np, patch_d, patch_stride, 1, g, st);
    check_launch();
    xpass<double>(InRegRot<double>{Patch<double>{patch_d, P.bbox, patch_stride}}, OutPlain<double>{t1d, ng, nx - 1}, 1,
                  P.bbox, 1);
    ypass<double>(t1d, t2d, ng, 1, mult(MULT_AIMPL, 1, 0));
    xpass<double>(InPlain<double>{t2d, ng, nx - 1}, OutSub<double>{G1n, ng, nx - 1}, 1);
    // vort2flux!(state.psi, state.q, state.Gamma)
    vort2flux_l1d(G1n, Gnew, q, psi1, q1, true);
    gc = 1 - gc;
    graph_launches[1 - gc] = launches - launches0;
}

// vort2flux (src/fluid.jl:178-205) with level 1 in FP64 (G1v; psi1_out, q1_out)
// and levels 2..L in FP32 (Gm, psi, qout; level slots as in the all-float layout,
// slot 1 unused).  curl_all = false computes q at level 1 only.
template <class T>
void Engine<T>::vort2flux_l1d(const double *G1v, T *Gm, T *qout, double *psi1_out, double *q1_out, bool curl_all) {
    const int nx2 = nx / 2, ny2 = ny / 2;
    const dim3 cblk(16, 16), cgrd((nx2 + 15) / 16, (ny2 + 15) / 16, 1);
    if (L >= 2) {
        coarsify_kernel<T, double><<<cgrd, cblk, 0, st>>>(Gm + ng, G1v, 0, g);
        check_launch();
    }
    for (int lev = 3; lev <= L; ++lev) {
        coarsify_kernel<T><<<cgrd, cblk, 0, st>>>(Gm + (lev - 1) * ng, Gm + (lev - 2) * ng, 0, g);
        check_launch();
    }
    const dim3 qblk(64, 4), qgrd((nx + 1 + 63) / 64, (ny + 1 + 3) / 4, 1);
    for (int lev = L; lev >= 2; --lev) {
        T *Gl = Gm + (lev - 1) * ng, *Pl = psi + (lev - 1) * ng;
        if (lev == L)
            xpass(in_plain(Gl, 0), out_plain(t1, ng), 1);
        else
            xpass(InBC<T>{Gl, psi + lev * ng, 0, 0, g}, out_plain(t1, ng), 1);
        ypass(t1, t2, ng, 1, mult(MULT_LAPINV, 1, 0));
        xpass(in_plain(t2, ng), out_plain(Pl, 0), 1);
        if (curl_all) {
            curl_kernel<T, T, T><<<qgrd, qblk, 0, st>>>(qout + (lev - 1) * nq, 0, Pl, 0,
                                                        lev < L ? psi + lev * ng : nullptr, 0, g);
            check_launch();
        }
    }
    const T *coarse = L > 1 ? psi + ng : nullptr;
    if (coarse)
        xpass<double>(InBC<double, T>{G1v, coarse, 0, 0, g}, OutPlain<double>{t1d, ng, nx - 1}, 1);
    else
        xpass<double>(InPlain<double>{G1v, 0, nx - 1}, OutPlain<double>{t1d, ng, nx - 1}, 1);
    ypass<double>(t1d, t2d, ng, 1, mult(MULT_LAPINV, 1, 0));
    xpass<double>(InPlain<double>{t2d, ng, nx - 1}, OutPlain<double>{psi1_out, ng, nx - 1}, 1);
    curl_kernel<double, double, T><<<qgrd, qblk, 0, st>>>(q1_out, 0, psi1_out, 0, coarse, 0, g);
    check_launch();
}

namespace {
// Evaluates an X-pass prologue functor on every (i, j) of one field (diagnostics).
template <class In>
__global__ void eval_prologue_kernel(In in, double *out, int nx, int ny) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (i > nx - 1 || j > ny - 1) return;
    out[(long long)(i - 1) + (long long)(nx - 1) * (j - 1)] = in(0, i, j);
}

template <class T>
__global__ void q0_fill_kernel(T *q0, const StepDev *prm, Grid g) {
    const long long nu = (long long)(g.nx + 1) * g.ny, nq = nu + (long long)g.nx * (g.ny + 1);
    const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int lev = blockIdx.y + 1;
    if (f >= nq) return;
    double v;
    if (f < nu)
        v = base_flux_x(g, prm, lev, (int)(f % (g.nx + 1)) + 1, (int)(f / (g.nx + 1)) + 1);
    else
        v = base_flux_y(g, prm, lev, (int)((f - nu) % g.nx) + 1, (int)((f - nu) / g.nx) + 1);
    q0[(long long)blockIdx.y * nq + f] = (T)v;
}

template <class A, class B>
__global__ void convert_kernel(B *__restrict__ dst, const A *__restrict__ src, long long n) {
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        dst[k] = (B)src[k];
}
}  // namespace

template <class T>
void Engine<T>::upload(T *dst, const double *src, size_t n) {
    if (std::is_same<T, double>::value) {
        CK(cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyHostToDevice, st));
        return;
    }
    double *tmp = staging(n);
    CK(cudaMemcpyAsync(tmp, src, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    convert_kernel<double, T><<<1184, 256, 0, st>>>(dst, tmp, (long long)n);
    check_launch();
}

template <class T>
void Engine<T>::download(double *dst, const T *src, size_t n) {
    if (std::is_same<T, double>::value) {
        CK(cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
        return;
    }
    double *tmp = staging(n);
    convert_kernel<T, double><<<1184, 256, 0, st>>>(tmp, src, (long long)n);
    check_launch();
    CK(cudaMemcpyAsync(dst, tmp, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
}

template <class T>
void Engine<T>::materialise_q0() {
    if (!q0mat) q0mat = dalloc<T>(nq * L);
    if (q0_from_user) return;
    if (q0_zero) {
        CK(cudaMemsetAsync(q0mat, 0, sizeof(T) * nq * L, st));
        return;
    }
    stage_acquire();
    prm_h->fs[0] = fs_last[0];
    prm_h->fs[1] = fs_last[1];
    for (int k = 0; k < 6; ++k) prm_h->gm[k] = gm_last[k];
    CK(cudaMemcpyAsync(prm, prm_h, sizeof(StepDev), cudaMemcpyHostToDevice, st));
    stage_release();
    q0_fill_kernel<T><<<dim3((unsigned)((nq + 255) / 256), L), 256, 0, st>>>(q0mat, prm, g);
    check_launch();
}

// ---------------------------------------------------------------------------
// Engine methods behind the C ABI
// ---------------------------------------------------------------------------

template <class T>
void Engine<T>::init(const ibpm_problem *p, const ibpm_options &o) {
    opt = o;
    device = o.device;
    nx = p->nx;
    ny = p->ny;
    L = p->nlevel;
    np = p->npanel;
    nbody = p->nbody;
    nu = (long long)(p->nx + 1) * p->ny;
    nq = nu + (long long)p->nx * (p->ny + 1);
    ng = (long long)(p->nx - 1) * (p->ny - 1);
    nbc = 2LL * (p->nx + 1) + 2LL * (p->ny + 1);
    g = Grid{p->nx, p->ny, p->nlevel, p->h, p->x0, p->y0, p->Re, p->dt, p->grid_moving ? 1 : 0};
    body_kind.assign(p->body_kind, p->body_kind + p->nbody);
    body_start.assign(p->body_start, p->body_start + p->nbody + 1);
    ref_xb.assign(p->body_xb, p->body_xb + 2 * (size_t)p->npanel);
    ref_ds.assign(p->body_ds, p->body_ds + p->npanel);
    static_bodies = true;
    for (int b = 0; b < p->nbody; ++b)
        if (body_kind[b] != IBPM_BODY_STATIC) static_bodies = false;
    problem_copy = *p;
    problem_copy.body_kind = body_kind.data();
    problem_copy.body_start = body_start.data();
    problem_copy.body_xb = ref_xb.data();
    problem_copy.body_ds = ref_ds.data();
}

namespace {
// Output accessors (src/problem.jl:715-866) for one level: vorticity Gamma / hc^2,
// x_velocity (q_u + q0_u) / hc, y_velocity (q_v + q0_v) / hc.
template <class T>
__global__ void field_kernel(const T *__restrict__ G, const T *__restrict__ q, const T *__restrict__ q0, int field,
                             int lev, Grid g, double *__restrict__ out) {
    const long long nu = (long long)(g.nx + 1) * g.ny, nq = nu + (long long)g.nx * (g.ny + 1);
    const long long ng = (long long)(g.nx - 1) * (g.ny - 1);
    const long long n = field == IBPM_FIELD_VORTICITY ? ng : field == IBPM_FIELD_X_VELOCITY ? nu : nq - nu;
    const double hc = gridstep(g, lev);
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        if (field == IBPM_FIELD_VORTICITY) {
            out[k] = (double)G[(lev - 1) * ng + k] / (hc * hc);
        } else {
            const long long f = (lev - 1) * nq + (field == IBPM_FIELD_X_VELOCITY ? k : nu + k);
            out[k] = ((double)q[f] + (double)q0[f]) / hc;
        }
    }
}
}  // namespace

template <class T>
void Engine<T>::get_field(int field, int level, double *out) {
    CK(cudaSetDevice(device));
    if (level < 1 || level > L) throw ApiError{IBPM_ERR_INVALID, "level out of range"};
    long long n = 0;
    if (field == IBPM_FIELD_VORTICITY)
        n = ng;
    else if (field == IBPM_FIELD_X_VELOCITY)
        n = (long long)(nx + 1) * ny;
    else if (field == IBPM_FIELD_Y_VELOCITY)
        n = (long long)nx * (ny + 1);
    else
        throw ApiError{IBPM_ERR_INVALID, "unknown field"};
    if (!out) throw ApiError{IBPM_ERR_INVALID, "null output"};
    if (!field_d) field_d = dalloc<double>((size_t)std::max<long long>(nq, ng));
    if (field != IBPM_FIELD_VORTICITY) materialise_q0();
    if (l1d && level == 1) {
        // level 1 from its FP64 fields (q0 of the last step's callback values)
        if (field != IBPM_FIELD_VORTICITY) {
            q0_fill_kernel<double><<<dim3((unsigned)((nq + 255) / 256), 1), 256, 0, st>>>(q0d, prm, g);
            check_launch();
            if (q0_zero) CK(cudaMemsetAsync(q0d, 0, sizeof(double) * nq, st));
        }
        field_kernel<double><<<592, 256, 0, st>>>(G1[gc], q1, q0d, field, 1, g, field_d);
    } else {
        field_kernel<T><<<592, 256, 0, st>>>(G[gc], q, q0mat, field, level, g, field_d);
    }
    check_launch();
    CK(cudaMemcpyAsync(out, field_d, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
}

template <class T>
void Engine<T>::set_rebuild_transform(int products) {
    CK(cudaSetDevice(device));
    if (products != 0 && products != 1 && products != 3)
        throw ApiError{IBPM_ERR_INVALID, "the rebuild transform takes 0, 1 or 3 products"};
    if (products != 0) {
        if (!std::is_same<T, double>::value)
            throw ApiError{IBPM_ERR_INVALID, "tensor-core transforms serve the FP64 engine"};
        if (static_bodies) throw ApiError{IBPM_ERR_INVALID, "the B rebuild exists for moving bodies only"};
        if (nx != ny || (nx != 256 && nx != 512))
            throw ApiError{IBPM_ERR_INVALID, "tensor-core transforms need nx = ny in {256, 512}"};
        tc_prepare(kbatch, products);
    }
    if (products != tc_prod) {
        CK(cudaStreamSynchronize(st));
        if (binv_exec) cudaGraphExecDestroy(binv_exec);
        if (binv_graph) cudaGraphDestroy(binv_graph);
        binv_exec = nullptr;
        binv_graph = nullptr;
    }
    // back to the FP64 transforms: the plan's line buffers are released
    if (products == 0 && tc) {
        tc_destroy(tc);
        tc = nullptr;
    }
    tc_prod = products;
}

template <class T>
void Engine<T>::set_warm_start(ibpm_net *net, int mode, int depth) {
    CK(cudaSetDevice(device));
    if (static_bodies) throw ApiError{IBPM_ERR_INVALID, "the warm start applies to moving bodies (CG) only"};
    if (mode != IBPM_WS_PREVIOUS && mode != IBPM_WS_LEARNED && mode != IBPM_WS_EXTRAPOLATED &&
        mode != IBPM_WS_PROJECTED && mode != IBPM_WS_DIRECT && mode != IBPM_WS_PRECONDITIONED &&
        mode != IBPM_WS_PRECOND_EXTRAP)
        throw ApiError{IBPM_ERR_INVALID, "unknown warm-start mode"};
    if (mode == IBPM_WS_PRECOND_EXTRAP && !ws_stale) {
        ws_stale = dalloc<double>(6 * (size_t)np);
        ws_x0 = dalloc<double>(2 * (size_t)np);
        ws_nvalid = dalloc<int>(1);
    }
    if (mode == IBPM_WS_DIRECT || mode == IBPM_WS_PRECONDITIONED || mode == IBPM_WS_PRECOND_EXTRAP) {
        if (!std::is_same<T, double>::value)
            throw ApiError{IBPM_ERR_INVALID, "the direct and preconditioned starts need the FP64 engine"};
        if (depth < 1 || depth > (1 << 20)) throw ApiError{IBPM_ERR_INVALID, "the rebuild interval (depth) must be 1 .. 1048576"};
        // all 2 np columns in one batch where about 16 GB of column work allows
        const long long per_col = (2 * ng * L + nq + 2 * ng) * (long long)sizeof(T);
        grow_batch_buffers((int)std::min<long long>(2 * np, std::max(1LL, (16LL << 30) / per_col)));
        const int n = 2 * np;
        if (!Binv) Binv = dalloc<double>((size_t)n * n);
        if (!Bwork) Bwork = dalloc<double>((size_t)n * n);
        ws_refresh = depth;
        ws_since = 0;
    }
    if (mode == IBPM_WS_PROJECTED) {
        if (depth < 1 || depth > 16) throw ApiError{IBPM_ERR_INVALID, "projection depth must be 1 .. 16"};
        grow_batch_buffers(depth);
        if (!ws_hist) {
            ws_hist = dalloc<double>(2 * (size_t)np * 16);
            ws_bhist = dalloc<double>(2 * (size_t)np * 16);
            ws_G = dalloc<double>(256);
            ws_h = dalloc<double>(16);
        }
        // the history starts from the current solution alone
        CK(cudaMemsetAsync(ws_hist, 0, sizeof(double) * 2 * np * 16, st));
        CK(cudaMemcpyAsync(ws_hist, Fbt, sizeof(double) * 2 * np, cudaMemcpyDeviceToDevice, st));
        ws_depth = depth;
    }
    if (mode == IBPM_WS_LEARNED && !net) throw ApiError{IBPM_ERR_INVALID, "the learned warm start needs a network"};
    if (mode != IBPM_WS_LEARNED) net = nullptr;
    if (net) {
        if (net_device(net) != device) throw ApiError{IBPM_ERR_INVALID, "network and solver are on different devices"};
        if (net_cin(net) != kWsFeatures || net_cout(net) != kWsOutputs)
            throw ApiError{IBPM_ERR_INVALID, "the warm-start network must map 10 feature channels to 2 outputs"};
        const size_t need = net_act_floats(net, 1, np);
        if (need > ws_act_cap) {
            ws_act = dalloc<float>(need);
            ws_act_cap = need;
        }
    }
    CK(cudaStreamSynchronize(st));
    ws = net;
    ws_mode = mode;
    drop_graphs();  // the step graph holds the previous choice
}

template <class T>
void Engine<T>::warm_start_sample(float *features, float *target, float *prediction) {
    CK(cudaSetDevice(device));
    if (static_bodies) throw ApiError{IBPM_ERR_INVALID, "the warm start applies to moving bodies (CG) only"};
    if (ws_mode != IBPM_WS_EXTRAPOLATED && ws_mode != IBPM_WS_LEARNED)
        throw ApiError{IBPM_ERR_INVALID, "warm-start samples need the extrapolated or learned mode"};
    std::vector<double> f(2 * np), xe(2 * np);
    double rs = 0.0;
    CK(cudaMemcpyAsync(f.data(), Fbt, sizeof(double) * 2 * np, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(xe.data(), ws_x2, sizeof(double) * 2 * np, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&rs, ws_x2 + 4 * np, sizeof(double), cudaMemcpyDeviceToHost, st));
    if (features)
        CK(cudaMemcpyAsync(features, ws_feat, sizeof(float) * kWsFeatures * np, cudaMemcpyDeviceToHost, st));
    std::vector<double> pv(2 * np, 0.0);
    if (prediction && ws_mode == IBPM_WS_LEARNED)
        CK(cudaMemcpyAsync(pv.data(), ws_x2 + 2 * np, sizeof(double) * 2 * np, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    // the error of the extrapolated guess, converged F~b - x_e, in units of the
    // RMS of its residual (the scale of the residual feature channels)
    const double inv = rs > 0.0 ? 1.0 / rs : 0.0;
    if (target)
        for (int i = 0; i < 2 * np; ++i) target[i] = (float)((f[i] - xe[i]) * inv);
    // the network's correction as the step used it
    if (prediction)
        for (int i = 0; i < 2 * np; ++i) prediction[i] = (float)pv[i];
}

template <class T>
void Engine<T>::set_state(const ibpm_state_view *s) {
    CK(cudaSetDevice(device));
    const size_t ngL = (size_t)(ng * L), nqL = (size_t)(nq * L);
    const size_t np2 = sizeof(double) * 2 * np;
    index = s->index;
    t0 = s->t0;
    if (s->q) upload(q, s->q, nqL);
    if (s->q0) {
        if (!q0mat) q0mat = dalloc<T>(nq * L);
        upload(q0mat, s->q0, nqL);
        q0_from_user = true;
    }
    if (s->gamma) upload(G[gc], s->gamma, ngL);
    if (s->psi) upload(psi, s->psi, ngL);
    if (s->nonlin1) upload(nl[nc], s->nonlin1, ngL);
    if (s->nonlin2) upload(nl[1 - nc], s->nonlin2, ngL);
    if (l1d) {  // level 1 in FP64, exactly as given
        const size_t bg = sizeof(double) * ng, bq = sizeof(double) * nq;
        if (s->q) CK(cudaMemcpyAsync(q1, s->q, bq, cudaMemcpyHostToDevice, st));
        if (s->gamma) CK(cudaMemcpyAsync(G1[gc], s->gamma, bg, cudaMemcpyHostToDevice, st));
        if (s->psi) CK(cudaMemcpyAsync(psi1, s->psi, bg, cudaMemcpyHostToDevice, st));
        if (s->nonlin1) CK(cudaMemcpyAsync(nl1[nc], s->nonlin1, bg, cudaMemcpyHostToDevice, st));
        if (s->nonlin2) CK(cudaMemcpyAsync(nl1[1 - nc], s->nonlin2, bg, cudaMemcpyHostToDevice, st));
    }
    if (s->xb) CK(cudaMemcpyAsync(P.xb, s->xb, np2, cudaMemcpyHostToDevice, st));
    if (s->ds) CK(cudaMemcpyAsync(ds, s->ds, np2 / 2, cudaMemcpyHostToDevice, st));
    if (s->ub) CK(cudaMemcpyAsync(P.ub, s->ub, np2, cudaMemcpyHostToDevice, st));
    if (s->fbt) CK(cudaMemcpyAsync(Fbt, s->fbt, np2, cudaMemcpyHostToDevice, st));
    if (s->fbt && Fprev) CK(cudaMemcpyAsync(Fprev, Fbt, np2, cudaMemcpyDeviceToDevice, st));
    if (s->fbt && ws_hist) {
        CK(cudaMemsetAsync(ws_hist, 0, sizeof(double) * 2 * np * 16, st));
        CK(cudaMemcpyAsync(ws_hist, Fbt, np2, cudaMemcpyDeviceToDevice, st));
    }
    fs_last[0] = s->freestream[0];
    fs_last[1] = s->freestream[1];
    // update_vars! (problem.jl:676-685)
    binv_reduce_kernel<<<1, 1024, 0, st>>>(nullptr, 0, 2 * np, Fbt, fb, total, g.h, g.dt, 0);
    check_launch();
    CK(cudaStreamSynchronize(st));
}

template <class T>
void Engine<T>::get_state(ibpm_state_view *s) {
    CK(cudaSetDevice(device));
    const size_t ngL = (size_t)(ng * L), nqL = (size_t)(nq * L);
    const size_t np2 = sizeof(double) * 2 * np;
    s->index = index;
    s->t0 = t0;
    s->freestream[0] = fs_last[0];
    s->freestream[1] = fs_last[1];
    if (s->q) download(s->q, q, nqL);
    if (s->q0) {
        materialise_q0();
        download(s->q0, q0mat, nqL);
    }
    if (s->gamma) download(s->gamma, G[gc], ngL);
    if (s->psi) download(s->psi, psi, ngL);
    if (s->nonlin1) download(s->nonlin1, nl[nc], ngL);
    if (s->nonlin2) download(s->nonlin2, nl[1 - nc], ngL);
    if (l1d) {  // level 1 from its FP64 fields
        const size_t bg = sizeof(double) * ng, bq = sizeof(double) * nq;
        if (s->q) CK(cudaMemcpyAsync(s->q, q1, bq, cudaMemcpyDeviceToHost, st));
        if (s->q0 && !q0_from_user) {  // prm holds the last step's values (materialise_q0 above)
            q0_fill_kernel<double><<<dim3((unsigned)((nq + 255) / 256), 1), 256, 0, st>>>(q0d, prm, g);
            check_launch();
            if (q0_zero) CK(cudaMemsetAsync(q0d, 0, bq, st));
            CK(cudaMemcpyAsync(s->q0, q0d, bq, cudaMemcpyDeviceToHost, st));
        }
        if (s->gamma) CK(cudaMemcpyAsync(s->gamma, G1[gc], bg, cudaMemcpyDeviceToHost, st));
        if (s->psi) CK(cudaMemcpyAsync(s->psi, psi1, bg, cudaMemcpyDeviceToHost, st));
        if (s->nonlin1) CK(cudaMemcpyAsync(s->nonlin1, nl1[nc], bg, cudaMemcpyDeviceToHost, st));
        if (s->nonlin2) CK(cudaMemcpyAsync(s->nonlin2, nl1[1 - nc], bg, cudaMemcpyDeviceToHost, st));
    }
    if (s->xb) CK(cudaMemcpyAsync(s->xb, P.xb, np2, cudaMemcpyDeviceToHost, st));
    if (s->ds) CK(cudaMemcpyAsync(s->ds, ds, np2 / 2, cudaMemcpyDeviceToHost, st));
    if (s->ub) CK(cudaMemcpyAsync(s->ub, P.ub, np2, cudaMemcpyDeviceToHost, st));
    if (s->fbt) CK(cudaMemcpyAsync(s->fbt, Fbt, np2, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
}

template <class T>
bool Engine<T>::advance(int64_t nsteps, const ibpm_step_params *params) {
    CK(cudaSetDevice(device));
    cg_hit_maxiter = false;
    for (int64_t k = 0; k < nsteps; ++k) step(params[k]);
    CK(cudaStreamSynchronize(st));
    cg_collect();
    return cg_hit_maxiter;
}

template <class T>
void Engine<T>::get_forces(double *fbo, double *tot) {
    CK(cudaSetDevice(device));
    if (fbo) CK(cudaMemcpyAsync(fbo, fb, sizeof(double) * 2 * np, cudaMemcpyDeviceToHost, st));
    if (tot) CK(cudaMemcpyAsync(tot, total, sizeof(double) * 2, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
}

template <class T>
void Engine<T>::get_time(int64_t *idx, double *t) {
    if (idx) *idx = index;
    if (t) *t = t0 + g.dt * (double)(index - 1);
}

template <class T>
void Engine<T>::get_info(ibpm_info *info) {
    info->nq = nq;
    info->ng = ng;
    info->nbc = nbc;
    info->static_bodies = static_bodies ? 1 : 0;
    info->last_cg_iters = last_cg_iters;
    info->last_cg_residual = last_cg_res;
    info->first_cg_residual = first_cg_res;
    info->warm_start_coef[0] = ws_coef[0];
    info->warm_start_coef[1] = ws_coef[1];
    info->device_bytes = dev_bytes;
}

template <class T>
void Engine<T>::set_profile(int enable) {
    CK(cudaStreamSynchronize(st));
    prof = enable != 0;
    prof_recs.clear();
    ev_next = 0;
}

template <class T>
void Engine<T>::read_profile(int kclass, int64_t *launches_out, double *ms, double *bytes) {
    CK(cudaStreamSynchronize(st));
    int64_t n = 0;
    double t = 0.0, b = 0.0;
    for (const auto &r : prof_recs) {
        if (r.cls != kclass) continue;
        float e = 0.f;
        CK(cudaEventElapsedTime(&e, ev_pool[r.ev], ev_pool[r.ev + 1]));
        ++n;
        t += e;
        b += r.bytes;
    }
    if (launches_out) *launches_out = n;
    if (ms) *ms = t;
    if (bytes) *bytes = b;
}

template <class T>
void Engine<T>::diag_solve(int op, int level, const double *b, double *x) {
    if (op < 0 || op > 8 || level < 1 || level > L) throw ApiError{IBPM_ERR_INVALID, "bad diag_solve arguments"};
    CK(cudaSetDevice(device));
    const int mode = op % 3 == 0 ? MULT_LAPINV : (op % 3 == 1 ? MULT_AEXPL : MULT_AIMPL);
    if (op >= 3) {
        if constexpr (std::is_same<T, double>::value) {
            tc_prepare(1, op < 6 ? 1 : 3);
            double *bd = staging((size_t)ng);
            CK(cudaMemcpyAsync(bd, b, sizeof(double) * ng, cudaMemcpyHostToDevice, st));
            if (!tc_mult[2]) tc_mult[2] = dalloc<float>((size_t)nx * nx);
            tc_mult_table(mode, level, tc_mult[2]);
            tc_solve(InPlain<double>{bd, ng, nx - 1}, 1, tc_mult[2], rhs, ng);
            CK(cudaMemcpyAsync(x, rhs, sizeof(double) * ng, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(err_h + 4, err + 4, sizeof(int), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            if (err_h[4]) {
                err_h[4] = 0;
                CK(cudaMemsetAsync(err + 4, 0, sizeof(int), st));
                throw ApiError{IBPM_ERR_CUDA, "a tensor-core transform pass gave up waiting for its operands"};
            }
            return;
        } else {
            throw ApiError{IBPM_ERR_INVALID, "tensor-core transforms serve the FP64 engine"};
        }
    }
    upload(rhs, b, (size_t)ng);
    xpass(in_plain(rhs, ng), out_plain(t1, ng), 1);
    ypass(t1, t2, ng, 1, mult(mode, level, 0));
    xpass(in_plain(t2, ng), out_plain(rhs, ng), 1);
    download(x, rhs, (size_t)ng);
    CK(cudaStreamSynchronize(st));
}

template <class T>
void Engine<T>::diag_apply_B(const double *z, double *x) {
    CK(cudaSetDevice(device));
    const size_t bytes = sizeof(double) * 2 * np;
    CK(cudaMemcpyAsync(cg_u, z, bytes, cudaMemcpyHostToDevice, st));
    compute_bbox();
    apply_B(cg_u, cg_c, 2 * np, 1);
    CK(cudaMemcpyAsync(x, cg_c, bytes, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
}

template <class T>
void Engine<T>::diag_binv(double *out) {
    if (!Binv) throw ApiError{IBPM_ERR_INVALID, "no precomputed B^-1 (moving bodies)"};
    const size_t n = 2 * (size_t)np;
    CK(cudaMemcpyAsync(out, Binv, sizeof(double) * n * n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
}

template <class T>
void Engine<T>::diag_vort2flux(double *gamma, double *psi_out, double *q_out) {
    CK(cudaSetDevice(device));
    const size_t ngL = (size_t)(ng * L);
    // its own vorticity buffer: Gw's coarse levels must stay zero outside the
    // coarsified block (apply_B relies on it)
    if (!diag_g) diag_g = dalloc<T>(ngL);
    upload(diag_g, gamma, ngL);
    if (!diag_q) diag_q = dalloc<T>(nq * L);
    vort2flux(psiw, diag_q, diag_g, 0, 0, 1, true);
    download(gamma, diag_g, ngL);
    download(psi_out, psiw, ngL);
    download(q_out, diag_q, (size_t)(nq * L));
    CK(cudaStreamSynchronize(st));
}

template <class T>
void Engine<T>::diag_reg(const double *f, double *gamma1, const double *q1, double *fout) {
    CK(cudaSetDevice(device));
    const size_t nf = sizeof(double) * 2 * np;
    compute_bbox();
    if (f && gamma1) {
        CK(cudaMemcpyAsync(cg_u, f, nf, cudaMemcpyHostToDevice, st));
        reg_patch(cg_u, 1);
        double *out = staging((size_t)ng);
        const dim3 blk(32, 8), grd((nx - 1 + 31) / 32, (ny - 1 + 7) / 8);
        eval_prologue_kernel<<<grd, blk, 0, st>>>(InRegRot<T>{Patch<T>{patch, P.bbox, patch_stride}}, out, nx, ny);
        check_launch();
        CK(cudaMemcpyAsync(gamma1, out, sizeof(double) * ng, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
    if (q1 && fout) {
        upload(qw, q1, (size_t)nq);
        launch_regT(P, qw, 0, cg_c, 0, 1, 0, prm, g, st);
        check_launch();
        CK(cudaMemcpyAsync(fout, cg_c, nf, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
}

// ---------------------------------------------------------------------------
// Ensembles: cases of one shape stepped as one batch
// ---------------------------------------------------------------------------

// Static-body, static-grid cases of one precision with equal nx, ny, levels,
// grid step and time step (they may differ in Reynolds number, domain origin,
// bodies and freestream) are stepped together: their fields are stacked
// case-major in one allocation (batch b = case L + level - 1), and every line
// pass, the nonlinear term, the curls and the coarsening run as one launch over
// all cases, and so does the coupling (E, B^-1, E^T), each case on its own
// panels through a device table of CaseViews.  A group step is one CUDA graph.
// Each case's per-element arithmetic is that of stepping it alone, so its
// results are the same bits.  While grouped, each case's engine points at its
// slot of the stacked fields (a single advance of one case still works); the
// ensemble's destruction copies every case back into buffers of its own.
template <class T>
struct CaseGroup {
    std::vector<Engine<T> *> cs;
    Engine<T> *e0 = nullptr;  // the first case: shape, tables, launch helpers
    int C = 0, L = 0;
    long long ng = 0, nq = 0;
    int device = 0;
    cudaStream_t st = nullptr;
    T *q = nullptr, *psi = nullptr, *G[2] = {nullptr, nullptr}, *nl[2] = {nullptr, nullptr};
    T *t1 = nullptr, *t2 = nullptr, *rhs = nullptr, *rest = nullptr, *qs1 = nullptr;
    double *t1_hi = nullptr, *t2_hi = nullptr, *psi1_hi = nullptr, *qs1_hi = nullptr;
    double *coef_all = nullptr, *coef_lev1 = nullptr, *re_tab = nullptr;
    StepDev *prm_tab = nullptr;
    CaseView *views = nullptr;  // each case's panels and force-solve buffers (device)
    int *bbox_tab = nullptr;    // each case's face window, 4 ints per case (device)
    int np_max = 0;
    static constexpr int kStage = 8;
    StepDev *stage_h[kStage] = {};
    cudaEvent_t stage_ev[kStage] = {};
    bool stage_used[kStage] = {};
    int stage_next = 0;
    int gc = 0, nc = 0;
    cudaGraph_t graph[2] = {nullptr, nullptr};
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    std::vector<void *> mem;

    template <class U>
    U *alloc(size_t n) {
        void *p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(U)) != cudaSuccess) {
            (void)cudaGetLastError();
            throw ApiError{IBPM_ERR_NOMEM, "cudaMalloc of an ensemble group's fields failed"};
        }
        mem.push_back(p);
        return static_cast<U *>(p);
    }

    // true when e can join a group led by f
    static bool compatible(const Engine<T> *f, const Engine<T> *e) {
        return e->device == f->device && e->nx == f->nx && e->ny == f->ny && e->L == f->L && e->g.h == f->g.h &&
               e->g.dt == f->g.dt && e->hi_level1 == f->hi_level1;
    }
    static bool eligible(const Engine<T> *e) {
        return e->static_bodies && !e->g.grid_moving && e->Binv != nullptr && !e->prof && !e->l1d;
    }

    void bind(const std::vector<Engine<T> *> &cases) {
        cs = cases;
        C = (int)cs.size();
        e0 = cs[0];
        L = e0->L;
        ng = e0->ng;
        nq = e0->nq;
        device = e0->device;
        CK(cudaSetDevice(device));
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        for (int k = 0; k < kStage; ++k) {
            CK(cudaMallocHost(&stage_h[k], sizeof(StepDev) * C));
            CK(cudaEventCreateWithFlags(&stage_ev[k], cudaEventDisableTiming));
        }
        const size_t ngL = (size_t)(ng * L), nqL = (size_t)(nq * L);
        q = alloc<T>(nqL * C);
        psi = alloc<T>(ngL * C);
        G[0] = alloc<T>(ngL * C);
        G[1] = alloc<T>(ngL * C);
        nl[0] = alloc<T>(ngL * C);
        nl[1] = alloc<T>(ngL * C);
        t1 = alloc<T>(ngL * C);
        t2 = alloc<T>(ngL * C);
        rhs = alloc<T>(ngL * C);
        rest = alloc<T>(ngL * C);
        qs1 = alloc<T>((size_t)nq * C);
        if (e0->hi_level1) {
            t1_hi = alloc<double>((size_t)ng * C);
            t2_hi = alloc<double>((size_t)ng * C);
            psi1_hi = alloc<double>((size_t)ng * C);
            qs1_hi = alloc<double>((size_t)nq * C);
        }
        prm_tab = alloc<StepDev>(C);
        // dt / (2 Re hc^2) per (case, level), as Mult::coef forms it on the device
        std::vector<double> ca((size_t)C * L), c1(C), re(C);
        for (int c = 0; c < C; ++c) {
            const Grid &g = cs[c]->g;
            re[c] = g.Re;
            for (int lev = 1; lev <= L; ++lev) {
                const double hc = ldexp(g.h, lev - 1);
                ca[(size_t)c * L + lev - 1] = g.dt / (2 * g.Re * (hc * hc));
            }
            c1[c] = ca[(size_t)c * L];
        }
        coef_all = alloc<double>(ca.size());
        coef_lev1 = alloc<double>(C);
        re_tab = alloc<double>(C);
        CK(cudaMemcpyAsync(coef_all, ca.data(), sizeof(double) * ca.size(), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(coef_lev1, c1.data(), sizeof(double) * C, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(re_tab, re.data(), sizeof(double) * C, cudaMemcpyHostToDevice, st));
        std::vector<CaseView> hv(C);
        views = alloc<CaseView>(C);
        bbox_tab = alloc<int>(4 * (size_t)C);
        for (int c = 0; c < C; ++c) {
            Engine<T> &ec = *cs[c];
            CK(cudaStreamSynchronize(ec.st));
            hv[c] = CaseView{ec.P, ec.Ftmp, ec.part, ec.Fbt, ec.fb, ec.total, ec.Binv, ec.patch, ec.patch_stride};
            np_max = std::max(np_max, ec.np);
            CK(cudaMemcpyAsync(bbox_tab + 4 * c, ec.P.bbox, sizeof(int) * 4, cudaMemcpyDeviceToDevice, st));
        }
        CK(cudaMemcpyAsync(views, hv.data(), sizeof(CaseView) * C, cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
        e0->template tune_ypass<T>(t1, t2, C);  // the group's Y passes cover C fields
        // move every case's state into its slot and point the case there
        for (int c = 0; c < C; ++c) {
            Engine<T> &e = *cs[c];
            const size_t og = ngL * c, oq = nqL * c;
            CK(cudaMemcpyAsync(q + oq, e.q, sizeof(T) * nqL, cudaMemcpyDeviceToDevice, st));
            CK(cudaMemcpyAsync(psi + og, e.psi, sizeof(T) * ngL, cudaMemcpyDeviceToDevice, st));
            CK(cudaMemcpyAsync(G[0] + og, e.G[e.gc], sizeof(T) * ngL, cudaMemcpyDeviceToDevice, st));
            CK(cudaMemcpyAsync(G[1] + og, e.G[1 - e.gc], sizeof(T) * ngL, cudaMemcpyDeviceToDevice, st));
            CK(cudaMemcpyAsync(nl[0] + og, e.nl[e.nc], sizeof(T) * ngL, cudaMemcpyDeviceToDevice, st));
            CK(cudaMemcpyAsync(nl[1] + og, e.nl[1 - e.nc], sizeof(T) * ngL, cudaMemcpyDeviceToDevice, st));
            CK(cudaMemcpyAsync(prm_tab + c, e.prm, sizeof(StepDev), cudaMemcpyDeviceToDevice, st));
        }
        CK(cudaStreamSynchronize(st));
        for (int c = 0; c < C; ++c) {
            Engine<T> &e = *cs[c];
            e.drop_graphs();
            T *own[6] = {e.q, e.psi, e.G[0], e.G[1], e.nl[0], e.nl[1]};
            for (int k = 0; k < 6; ++k) e.dfree(own[k]);
            const size_t og = ngL * c, oq = nqL * c;
            e.q = q + oq;
            e.psi = psi + og;
            e.G[0] = G[0] + og;
            e.G[1] = G[1] + og;
            e.nl[0] = nl[0] + og;
            e.nl[1] = nl[1] + og;
            e.gc = 0;
            e.nc = 0;
        }
    }

    // a member destroyed while grouped: its slot is never touched again (the
    // group cannot step any more; the ensemble refuses to)
    void forget(const ibpm_handle *h) {
        for (auto &x : cs)
            if (x != nullptr && static_cast<const ibpm_handle *>(x) == h) x = nullptr;
        if (e0 != nullptr && static_cast<const ibpm_handle *>(e0) == h) e0 = nullptr;
    }

    // copies every case back into buffers of its own (before the group's memory goes)
    void unbind() {
        if (cs.empty()) return;
        CK(cudaSetDevice(device));
        CK(cudaStreamSynchronize(st));
        const size_t ngL = (size_t)(ng * L), nqL = (size_t)(nq * L);
        for (int c = 0; c < C; ++c) {
            if (cs[c] == nullptr) continue;
            Engine<T> &e = *cs[c];
            CK(cudaStreamSynchronize(e.st));
            e.drop_graphs();
            T *nq_ = e.template dalloc<T>(nqL), *np_ = e.template dalloc<T>(ngL);
            T *g0 = e.template dalloc<T>(ngL), *g1 = e.template dalloc<T>(ngL);
            T *n0 = e.template dalloc<T>(ngL), *n1 = e.template dalloc<T>(ngL);
            CK(cudaMemcpyAsync(nq_, e.q, sizeof(T) * nqL, cudaMemcpyDeviceToDevice, e.st));
            CK(cudaMemcpyAsync(np_, e.psi, sizeof(T) * ngL, cudaMemcpyDeviceToDevice, e.st));
            CK(cudaMemcpyAsync(g0, e.G[0], sizeof(T) * ngL, cudaMemcpyDeviceToDevice, e.st));
            CK(cudaMemcpyAsync(g1, e.G[1], sizeof(T) * ngL, cudaMemcpyDeviceToDevice, e.st));
            CK(cudaMemcpyAsync(n0, e.nl[0], sizeof(T) * ngL, cudaMemcpyDeviceToDevice, e.st));
            CK(cudaMemcpyAsync(n1, e.nl[1], sizeof(T) * ngL, cudaMemcpyDeviceToDevice, e.st));
            CK(cudaStreamSynchronize(e.st));
            e.q = nq_;
            e.psi = np_;
            e.G[0] = g0;
            e.G[1] = g1;
            e.nl[0] = n0;
            e.nl[1] = n1;
        }
        cs.clear();
    }

    ~CaseGroup() {
        try {
            unbind();
        } catch (...) {
        }
        for (int p = 0; p < 2; ++p) {
            if (exec[p]) cudaGraphExecDestroy(exec[p]);
            if (graph[p]) cudaGraphDestroy(graph[p]);
        }
        for (void *p : mem) cudaFree(p);
        for (int k = 0; k < kStage; ++k) {
            if (stage_h[k]) cudaFreeHost(stage_h[k]);
            if (stage_ev[k]) cudaEventDestroy(stage_ev[k]);
        }
        if (st) cudaStreamDestroy(st);
    }

    // Lends e0's launch helpers the group's stream and scratch for one call.
    struct Borrow {
        Engine<T> &e;
        cudaStream_t st;
        T *t1, *t2, *rhs;
        double *t1_hi, *t2_hi, *psi1_hi, *qs1_hi;
        Borrow(Engine<T> &e_, CaseGroup &gr) : e(e_) {
            st = e.st;
            t1 = e.t1;
            t2 = e.t2;
            rhs = e.rhs;
            t1_hi = e.t1_hi;
            t2_hi = e.t2_hi;
            psi1_hi = e.psi1_hi;
            qs1_hi = e.qs1_hi;
            e.st = gr.st;
            e.t1 = gr.t1;
            e.t2 = gr.t2;
            e.rhs = gr.rhs;
            e.t1_hi = gr.t1_hi;
            e.t2_hi = gr.t2_hi;
            e.psi1_hi = gr.psi1_hi;
            e.qs1_hi = gr.qs1_hi;
        }
        ~Borrow() {
            e.st = st;
            e.t1 = t1;
            e.t2 = t2;
            e.rhs = rhs;
            e.t1_hi = t1_hi;
            e.t2_hi = t2_hi;
            e.psi1_hi = psi1_hi;
            e.qs1_hi = qs1_hi;
        }
    };

    // advance! of every case (src/solver.jl:155-190), batched; e0's helpers launch
    // on the group stream (Borrow)
    void step_body() {
        Engine<T> &e = *e0;
        Borrow bw(e, *this);
        T *Gold = G[gc], *Gnew = G[1 - gc];
        T *N1 = nl[nc], *N2 = nl[1 - nc];
        const long long bsG = ng * L, bsQ = nq * L;
        {
            NonlinArgs<T> a{q, Gold, N1, N2, rest, prm_tab, e.g, re_tab, 1};
            const dim3 blk(kNlTX, kNlBY), grd((e.nx - 1 + kNlTX - 1) / kNlTX, (e.ny - 1 + kNlTY - 1) / kNlTY, C * L);
            nonlinear_kernel<T, T, true><<<grd, blk, 0, st>>>(a);
            e.check_launch();
        }
        e.trial(Gold, rest, Gnew, C * L, coef_all);
        nc = 1 - nc;
        e.vort2flux(psi, e.hi_level1 ? nullptr : qs1, Gnew, bsG, nq, C, false, e.hi_level1, nullptr);
        // per case, one launch over all cases each: E qs, F~b = B^-1 Ftmp,
        // update_vars!, E^T F~b and the X pass of its rot (zero outside each case's window)
        if (e.hi_level1)
            launch_regT_multi<double>(views, C, np_max, qs1_hi, nq, prm_tab, e.g, st);
        else
            launch_regT_multi<T>(views, C, np_max, qs1, nq, prm_tab, e.g, st);
        e.check_launch();
        const int nchunk = (2 * np_max + 63) / 64;
        binv_gemv_multi_kernel<<<dim3(nchunk, nchunk, C), 256, 0, st>>>(views);
        e.check_launch();
        binv_reduce_multi_kernel<<<C, 1024, 0, st>>>(views, e.g.h, e.g.dt);
        e.check_launch();
        launch_reg_patch_multi<T>(views, C, e.g, st);
        e.check_launch();
        e.xpass(InRegRotTab<T>{views}, e.out_plain(t1, ng), C, bbox_tab, 1, 4);
        // project_circ's solve at level 1 of every case, then vort2flux!
        Mult m = e.mult(MULT_AIMPL, 1, 0);
        m.coef_tab = coef_lev1;
        e.ypass(t1, t2, ng, C, m);
        e.xpass(e.in_plain(t2, ng), OutSub<T>{Gnew, bsG, e.nx - 1}, C);
        e.vort2flux(psi, q, Gnew, bsG, bsQ, C, true);
        gc = 1 - gc;
    }

    // one step of every case: this step's callback values, then the group's graph
    void step(const std::vector<const ibpm_step_params *> &prm) {
        CK(cudaSetDevice(device));
        const int k = stage_next;
        stage_next = (stage_next + 1) % kStage;
        if (stage_used[k]) CK(cudaEventSynchronize(stage_ev[k]));
        stage_used[k] = true;
        for (int c = 0; c < C; ++c) {
            StepDev &d = stage_h[k][c];
            d.fs[0] = prm[c]->freestream[0];
            d.fs[1] = prm[c]->freestream[1];
            for (int j = 0; j < 6; ++j) d.gm[j] = prm[c]->grid_motion[j];
        }
        CK(cudaMemcpyAsync(prm_tab, stage_h[k], sizeof(StepDev) * C, cudaMemcpyHostToDevice, st));
        CK(cudaEventRecord(stage_ev[k], st));
        const int p = gc;
        if (!exec[p]) {
            const int gc0 = gc, nc0 = nc;
            const long long l0 = e0->launches;
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
                e0->launches = l0;
                throw;
            }
            CK(cudaStreamEndCapture(st, &graph[p]));
            CK(cudaGraphInstantiate(&exec[p], graph[p], 0));
            gc = gc0;
            nc = nc0;
            e0->launches = l0;
        }
        CK(cudaGraphLaunch(exec[p], st));
        gc = 1 - gc;
        nc = 1 - nc;
        for (int c = 0; c < C; ++c) {
            Engine<T> &e = *cs[c];
            ++e.index;
            e.gc = gc;
            e.nc = nc;
            e.q0_zero = false;
            e.q0_from_user = false;
            e.last_cg_iters = 0;
            e.fs_last[0] = prm[c]->freestream[0];
            e.fs_last[1] = prm[c]->freestream[1];
            for (int j = 0; j < 6; ++j) e.gm_last[j] = prm[c]->grid_motion[j];
        }
    }

    // waits for the group's steps; each case's own parameter block gets the last step's values
    void finish() {
        CK(cudaSetDevice(device));
        for (int c = 0; c < C; ++c)
            CK(cudaMemcpyAsync(cs[c]->prm, prm_tab + c, sizeof(StepDev), cudaMemcpyDeviceToDevice, st));
        CK(cudaStreamSynchronize(st));
    }
};

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

template <class T>
static int create_engine(const ibpm_problem *p, const ibpm_options &opt, ibpm_handle **out) {
    Engine<T> *h = new Engine<T>();
    h->init(p, opt);
    const int rc = guarded(h, [&] { h->setup(); });
    if (rc != IBPM_OK) {
        g_create_error = h->last_error;
        delete h;
        return rc;
    }
    *out = h;
    return IBPM_OK;
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
    if (opt.precision != IBPM_FP64 && opt.precision != IBPM_FP32 && opt.precision != IBPM_MIXED_L1) {
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
    for (int b = 0; b < p->nbody; ++b)
        if (p->body_start[b + 1] < p->body_start[b]) {
            g_create_error = "body_start must not decrease";
            return IBPM_ERR_INVALID;
        }
    if (!std::isfinite(p->h) || !std::isfinite(p->x0) || !std::isfinite(p->y0) || !std::isfinite(p->dt) ||
        !std::isfinite(p->Re)) {
        g_create_error = "non-finite grid or fluid parameter";
        return IBPM_ERR_INVALID;
    }
    for (long long k = 0; k < 2LL * p->npanel; ++k)
        if (!std::isfinite(p->body_xb[k]) || (k < p->npanel && !std::isfinite(p->body_ds[k]))) {
            g_create_error = "non-finite body point";
            return IBPM_ERR_INVALID;
        }
    if (opt.cg_maxiter < 0 || !(opt.cg_reltol >= 0) || !(opt.cg_abstol >= 0)) {
        g_create_error = "CG options must be non-negative";
        return IBPM_ERR_INVALID;
    }
    for (int b = 0; b < p->nbody; ++b)
        if (p->body_kind[b] != IBPM_BODY_STATIC && p->body_kind[b] != IBPM_BODY_MOVING_RIGID) {
            g_create_error = "unknown body kind";
            return IBPM_ERR_INVALID;
        }
    // The reference rejects out-of-region static panels while building the
    // Regularization (coupling.jl:38-41), before any size restriction of ours.
    for (int b = 0; b < p->nbody; ++b) {
        if (p->body_kind[b] != IBPM_BODY_STATIC) continue;
        for (int k = p->body_start[b]; k < p->body_start[b + 1]; ++k) {
            const double xb = p->body_xb[k], yb = p->body_xb[p->npanel + k];
            const int ix = (int)nearbyint((xb - p->x0) / p->h + 1.0 - 0.25);
            const int iy = (int)nearbyint((yb - p->y0) / p->h + 1.0 - 0.25);
            if (!(3 < ix && ix <= p->nx - 3) || !(3 < iy && iy <= p->ny - 3)) {
                g_create_error = "Panel index=" + std::to_string(k + 1) + " at (" + jl_float(xb) + ", " +
                                 jl_float(yb) + ") outside allowed region";
                return IBPM_ERR_REGION;
            }
        }
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= opt.device) {
        g_create_error = "no CUDA device available";
        return IBPM_ERR_CUDA;
    }
    if (opt.precision == IBPM_FP32 || opt.precision == IBPM_MIXED_L1) return create_engine<float>(p, opt, out);
    return create_engine<double>(p, opt, out);
}

void ibpm_destroy(ibpm_handle *h) { delete h; }

int ibpm_set_warm_start(ibpm_handle *h, int32_t mode, ibpm_net *net, int32_t depth) {
    if (!h) return IBPM_ERR_INVALID;
    return guarded(h, [&] { h->set_warm_start(net, mode, depth); });
}

int ibpm_set_rebuild_transform(ibpm_handle *h, int32_t products) {
    if (!h) return IBPM_ERR_INVALID;
    return guarded(h, [&] { h->set_rebuild_transform(products); });
}

int ibpm_warm_start_sample(ibpm_handle *h, float *features, float *target, float *prediction) {
    if (!h) return IBPM_ERR_INVALID;
    return guarded(h, [&] { h->warm_start_sample(features, target, prediction); });
}

int ibpm_set_state(ibpm_handle *h, const ibpm_state_view *s) {
    if (!h || !s) return IBPM_ERR_INVALID;
    return guarded(h, [&] { h->set_state(s); });
}

int ibpm_get_state(ibpm_handle *h, ibpm_state_view *s) {
    if (!h || !s) return IBPM_ERR_INVALID;
    return guarded(h, [&] { h->get_state(s); });
}

int ibpm_advance(ibpm_handle *h, int64_t nsteps, const ibpm_step_params *params) {
    if (!h || nsteps < 0 || (nsteps > 0 && !params)) return IBPM_ERR_INVALID;
    bool maxiter = false;
    const int rc = guarded(h, [&] { maxiter = h->advance(nsteps, params); });
    if (rc != IBPM_OK) return rc;
    if (maxiter) {
        h->last_error = "CG reached maxiter";
        return IBPM_WARN_CG_MAXITER;
    }
    return IBPM_OK;
}

struct ibpm_ensemble {
    std::vector<ibpm_handle *> cases;
    std::vector<char> gone;  // cases destroyed while the ensemble lives
    std::string last_error;
    std::vector<std::unique_ptr<CaseGroup<double>>> g64;
    std::vector<std::unique_ptr<CaseGroup<float>>> g32;
    std::vector<std::vector<int>> members64, members32;  // case indices of each group
    std::vector<int> alone;                              // cases stepped on their own streams
    static void case_gone(ibpm_ensemble *e, ibpm_handle *h) {
        for (size_t c = 0; c < e->cases.size(); ++c)
            if (e->cases[c] == h) e->gone[c] = 1;
        for (auto &g : e->g64) g->forget(h);
        for (auto &g : e->g32) g->forget(h);
    }
    void hold() {
        gone.assign(cases.size(), 0);
        for (ibpm_handle *h : cases) h->holders.push_back({this, &ibpm_ensemble::case_gone});
    }
    ~ibpm_ensemble() {
        for (size_t c = 0; c < cases.size(); ++c) {
            if (c < gone.size() && gone[c]) continue;
            auto &v = cases[c]->holders;
            v.erase(std::remove_if(v.begin(), v.end(), [&](const auto &w) { return w.first == this; }), v.end());
        }
        g64.clear();  // each group copies its live cases back into buffers of their own
        g32.clear();
    }
};

}  // extern "C"

namespace {
// Groups the eligible cases of one precision by shape (groups of one stay alone).
template <class T>
void form_groups(ibpm_ensemble *e, std::vector<std::unique_ptr<CaseGroup<T>>> &groups,
                 std::vector<std::vector<int>> &members, std::vector<bool> &taken) {
    std::vector<std::vector<int>> lists;
    for (int c = 0; c < (int)e->cases.size(); ++c) {
        Engine<T> *x = dynamic_cast<Engine<T> *>(e->cases[c]);
        if (!x || !CaseGroup<T>::eligible(x)) continue;
        bool placed = false;
        for (auto &l : lists)
            if (CaseGroup<T>::compatible(dynamic_cast<Engine<T> *>(e->cases[l[0]]), x)) {
                l.push_back(c);
                placed = true;
                break;
            }
        if (!placed) lists.push_back({c});
    }
    for (auto &l : lists) {
        if (l.size() < 2) continue;
        std::vector<Engine<T> *> es;
        for (int c : l) es.push_back(dynamic_cast<Engine<T> *>(e->cases[c]));
        std::unique_ptr<CaseGroup<T>> gr(new CaseGroup<T>());
        gr->bind(es);
        groups.push_back(std::move(gr));
        members.push_back(l);
        for (int c : l) taken[c] = true;
    }
}

template <class T>
void step_groups(ibpm_ensemble *e, std::vector<std::unique_ptr<CaseGroup<T>>> &groups,
                 const std::vector<std::vector<int>> &members, const ibpm_step_params *params, int64_t k) {
    const int64_t n = (int64_t)e->cases.size();
    for (size_t gi = 0; gi < groups.size(); ++gi) {
        std::vector<const ibpm_step_params *> prm;
        for (int c : members[gi]) prm.push_back(&params[k * n + c]);
        groups[gi]->step(prm);
    }
}
}  // namespace

extern "C" {

int ibpm_ensemble_create(ibpm_handle *const *cases, int32_t n, ibpm_ensemble **out) {
    if (!out) return IBPM_ERR_INVALID;
    *out = nullptr;
    if (n < 1 || !cases) return IBPM_ERR_INVALID;
    for (int32_t c = 0; c < n; ++c) {
        if (!cases[c]) return IBPM_ERR_INVALID;
        for (int32_t d = 0; d < c; ++d)
            if (cases[d] == cases[c]) return IBPM_ERR_INVALID;  // a case may appear once
    }
    ibpm_ensemble *e = new ibpm_ensemble;
    e->cases.assign(cases, cases + n);
    e->hold();
    bool batch = true;
    if (const char *v = getenv("IBPM_ENSEMBLE_BATCH")) batch = v[0] != '0';
    std::vector<bool> taken(n, false);
    const int rc = guarded(nullptr, [&] {
        if (batch) {
            form_groups<double>(e, e->g64, e->members64, taken);
            form_groups<float>(e, e->g32, e->members32, taken);
        }
    });
    if (rc != IBPM_OK) {
        g_create_error = "grouping the ensemble's cases failed";
        delete e;
        return rc;
    }
    for (int c = 0; c < n; ++c)
        if (!taken[c]) e->alone.push_back(c);
    *out = e;
    return IBPM_OK;
}

void ibpm_ensemble_destroy(ibpm_ensemble *e) { delete e; }

// Each step: every group's batched step graph, and each remaining case's step on
// its own stream, all enqueued before any is waited for.
int ibpm_ensemble_advance(ibpm_ensemble *e, int64_t nsteps, const ibpm_step_params *params) {
    if (!e || nsteps < 0 || (nsteps > 0 && !params)) return IBPM_ERR_INVALID;
    for (char d : e->gone)
        if (d) {
            e->last_error = "a case of the ensemble was destroyed before it";
            return IBPM_ERR_INVALID;
        }
    const int64_t n = (int64_t)e->cases.size();
    auto finish_all = [&] {
        for (auto &g : e->g64) guarded(nullptr, [&] { g->finish(); });
        for (auto &g : e->g32) guarded(nullptr, [&] { g->finish(); });
        for (int c : e->alone) guarded(e->cases[c], [&] { e->cases[c]->finish_steps(); });
    };
    for (int64_t k = 0; k < nsteps; ++k) {
        int rc = guarded(nullptr, [&] {
            step_groups<double>(e, e->g64, e->members64, params, k);
            step_groups<float>(e, e->g32, e->members32, params, k);
        });
        if (rc != IBPM_OK) {
            e->last_error = "batched group: step failed";
            finish_all();
            return rc;
        }
        for (int c : e->alone) {
            ibpm_handle *h = e->cases[c];
            rc = guarded(h, [&] { h->enqueue_step(params[k * n + c]); });
            if (rc != IBPM_OK) {
                e->last_error = "case " + std::to_string(c) + ": " + h->last_error;
                finish_all();
                return rc;
            }
        }
    }
    int rc = guarded(nullptr, [&] {
        for (auto &g : e->g64) g->finish();
        for (auto &g : e->g32) g->finish();
    });
    if (rc != IBPM_OK) {
        e->last_error = "batched group: synchronisation failed";
        return rc;
    }
    bool maxiter = false;
    for (int c : e->alone) {
        ibpm_handle *h = e->cases[c];
        bool m = false;
        rc = guarded(h, [&] { m = h->finish_steps(); });
        if (rc != IBPM_OK) {
            e->last_error = "case " + std::to_string(c) + ": " + h->last_error;
            return rc;
        }
        maxiter = maxiter || m;
    }
    if (maxiter) {
        e->last_error = "CG reached maxiter";
        return IBPM_WARN_CG_MAXITER;
    }
    return IBPM_OK;
}

int ibpm_tune_table(char *out, int32_t len) {
    const std::string t = tune_table().dump();
    if (out && len > 0) {
        const size_t n = std::min<size_t>(t.size(), (size_t)len - 1);
        memcpy(out, t.data(), n);
        out[n] = 0;
    }
    return (int)t.size() + 1;
}

int ibpm_ensemble_groups(const ibpm_ensemble *e, int32_t *ngroups, int32_t *nbatched) {
    if (!e) return IBPM_ERR_INVALID;
    int32_t ng = 0, nb = 0;
    for (auto &m : e->members64) ++ng, nb += (int32_t)m.size();
    for (auto &m : e->members32) ++ng, nb += (int32_t)m.size();
    if (ngroups) *ngroups = ng;
    if (nbatched) *nbatched = nb;
    return IBPM_OK;
}

const char *ibpm_ensemble_last_error(const ibpm_ensemble *e) { return e ? e->last_error.c_str() : ""; }

int ibpm_get_field(ibpm_handle *h, int32_t field, int32_t level, double *out) {
    if (!h) return IBPM_ERR_INVALID;
    return guarded(h, [&] { h->get_field(field, level, out); });
}

int ibpm_get_forces(ibpm_handle *h, double *fb, double *total_force) {
    if (!h) return IBPM_ERR_INVALID;
    return guarded(h, [&] { h->get_forces(fb, total_force); });
}

int ibpm_get_time(ibpm_handle *h, int64_t *index, double *t) {
    if (!h) return IBPM_ERR_INVALID;
    h->get_time(index, t);
    return IBPM_OK;
}

int ibpm_get_info(ibpm_handle *h, ibpm_info *info) {
    if (!h || !info) return IBPM_ERR_INVALID;
    h->get_info(info);
    return IBPM_OK;
}

const char *ibpm_last_error(const ibpm_handle *h) { return h ? h->last_error.c_str() : g_create_error.c_str(); }

void *ibpm_stream(ibpm_handle *h) { return h ? h->stream_ptr() : nullptr; }

int64_t ibpm_kernel_launches(const ibpm_handle *h) { return h ? h->launch_count() : 0; }

int ibpm_diag_solve(ibpm_handle *h, int op, int level, const double *b, double *x) {
    if (!h || !b || !x) return IBPM_ERR_INVALID;
    return guarded(h, [&] { h->diag_solve(op, level, b, x); });
}

int ibpm_diag_apply_B(ibpm_handle *h, const double *z, double *x) {
    if (!h || !z || !x) return IBPM_ERR_INVALID;
    return guarded(h, [&] { h->diag_apply_B(z, x); });
}

int ibpm_diag_binv(ibpm_handle *h, double *out) {
    if (!h || !out) return IBPM_ERR_INVALID;
    return guarded(h, [&] { h->diag_binv(out); });
}

int ibpm_diag_vort2flux(ibpm_handle *h, double *gamma, double *psi, double *q) {
    if (!h || !gamma || !psi || !q) return IBPM_ERR_INVALID;
    return guarded(h, [&] { h->diag_vort2flux(gamma, psi, q); });
}

int ibpm_diag_reg(ibpm_handle *h, const double *f, double *gamma1, const double *q1, double *fout) {
    if (!h) return IBPM_ERR_INVALID;
    return guarded(h, [&] { h->diag_reg(f, gamma1, q1, fout); });
}

int ibpm_profile(ibpm_handle *h, int enable) {
    if (!h) return IBPM_ERR_INVALID;
    return guarded(h, [&] { h->set_profile(enable); });
}

int ibpm_profile_read(ibpm_handle *h, int kclass, int64_t *launches, double *ms, double *bytes) {
    if (!h || kclass < 0 || kclass >= IBPM_KCLASS_COUNT) return IBPM_ERR_INVALID;
    return guarded(h, [&] { h->read_profile(kclass, launches, ms, bytes); });
}

}  // extern "C"
