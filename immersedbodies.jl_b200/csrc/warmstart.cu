// warmstart.cu -- the learned CG warm start: a 1D convolutional network over
// the body points, with its forward, backward, loss and Adam kernels.
//
// Layer l maps C_in channels to C_out channels over the n body points of one
// sample by a cross-correlation with zero padding,
//   out[co][p] = b[co] + sum_{ci, k} W[co][ci][k] in[ci][p + k - K/2],
// followed by tanh on every layer except the last.  Inputs are normalised per
// channel, (x - in_mean) / in_std, and the last layer's output is the
// normalised target: the prediction in solver units is out_mean + out_std y.
// Parameters are one flat FP32 vector, layer by layer: W_l [C_out][C_in][K],
// then b_l [C_out].  All reductions run in a fixed order, so training is
// deterministic for a given seed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "../../include/ibpm_b200.h"
#include "warmstart.h"

struct ibpm_net {
    int device = 0, cin = 0, width = 0, ksize = 0, layers = 0, cout = 0;
    std::vector<int> lci, lco;           // channels in / out of each layer
    std::vector<long long> woff, boff;   // offsets of W_l and b_l in the parameter vector
    long long nparams = 0;
    float *params = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
    float *norm = nullptr;               // in_mean[cin], in_std[cin], out_mean[cout], out_std[cout]
    long long adam_t = 0;
    cudaStream_t st = nullptr;
    std::vector<void *> bufs;            // every device allocation, freed on destroy
    // training scratch, grown on demand
    float *act = nullptr, *dbuf = nullptr, *bt = nullptr, *loss = nullptr;
    size_t act_cap = 0, dbuf_cap = 0, bt_cap = 0;
    std::string err;
};

namespace ibpm {
namespace {

struct NetError {
    int code;
    std::string msg;
};

#define NCK(x)                                                                              \
    do {                                                                                    \
        cudaError_t e_ = (x);                                                               \
        if (e_ != cudaSuccess) throw NetError{IBPM_ERR_CUDA, cudaGetErrorString(e_)};       \
    } while (0)

thread_local std::string g_create_err;

template <class F>
int guarded(ibpm_net *net, F &&f) {
    if (!net) return IBPM_ERR_INVALID;
    try {
        NCK(cudaSetDevice(net->device));
        f();
        return IBPM_OK;
    } catch (const NetError &e) {
        net->err = e.msg;
        (void)cudaGetLastError();
        return e.code;
    } catch (const std::exception &e) {
        net->err = e.what();
        return IBPM_ERR_INVALID;
    }
}

float *net_alloc(ibpm_net *net, size_t nfloat) {
    void *p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(nfloat, 1) * sizeof(float)) != cudaSuccess)
        throw NetError{IBPM_ERR_NOMEM, "cudaMalloc failed for the network"};
    net->bufs.push_back(p);
    NCK(cudaMemsetAsync(p, 0, std::max<size_t>(nfloat, 1) * sizeof(float), net->st));
    return static_cast<float *>(p);
}

// grows a persistent scratch buffer of the network to at least nfloat floats
void ensure(ibpm_net *net, float *&buf, size_t &cap, size_t nfloat) {
    if (cap >= nfloat) return;
    if (buf) {
        NCK(cudaStreamSynchronize(net->st));
        net->bufs.erase(std::find(net->bufs.begin(), net->bufs.end(), (void *)buf));
        cudaFree(buf);
    }
    buf = net_alloc(net, nfloat);
    cap = nfloat;
}

// A device buffer that lives for one call (freed when the call returns).
struct DevTmp {
    void *p = nullptr;
    DevTmp(size_t bytes) {
        if (cudaMalloc(&p, std::max<size_t>(bytes, 1)) != cudaSuccess) {
            p = nullptr;
            throw NetError{IBPM_ERR_NOMEM, "cudaMalloc failed for the network's data"};
        }
    }
    ~DevTmp() {
        if (p) cudaFree(p);
    }
    DevTmp(const DevTmp &) = delete;
    DevTmp &operator=(const DevTmp &) = delete;
    float *f() const { return static_cast<float *>(p); }
};

uint64_t splitmix64(uint64_t &s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
double uniform01(uint64_t &s) { return (double)(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0); }

constexpr int kThreads = 256;
inline unsigned blocks_for(long long n) { return (unsigned)((n + kThreads - 1) / kThreads); }

// ---- kernels ----

// x [B][C][N] -> (x - mean[c]) / std[c]; with idx, sample s of the output is
// sample idx[s] of the input (batch gather).
__global__ void normalise_kernel(const float *__restrict__ x, const int *__restrict__ idx, float *__restrict__ out,
                                 int B, int C, int N, const float *__restrict__ mean, const float *__restrict__ sd) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)B * C * N) return;
    const int c = (int)((t / N) % C);
    const long long s = t / ((long long)C * N), r = t % ((long long)C * N);
    const long long src = (idx ? (long long)idx[s] : s) * C * N + r;
    out[t] = (x[src] - mean[c]) / sd[c];
}

__global__ void conv_fwd_kernel(const float *__restrict__ in, const float *__restrict__ W,
                                const float *__restrict__ bias, float *__restrict__ out, int B, int Ci, int Co, int N,
                                int K, int act) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)B * Co * N) return;
    const int n = (int)(t % N), co = (int)((t / N) % Co);
    const long long b = t / ((long long)N * Co);
    const int h = K / 2;
    const float *w = W + (long long)co * Ci * K;
    const float *x = in + b * Ci * N;
    float acc = bias[co];
    for (int ci = 0; ci < Ci; ++ci)
        for (int k = 0; k < K; ++k) {
            const int nn = n + k - h;
            if (nn >= 0 && nn < N) acc = fmaf(w[ci * K + k], x[(long long)ci * N + nn], acc);
        }
    out[t] = act ? tanhf(acc) : acc;
}

// din[b][ci][m] = sum_{co, k} W[co][ci][k] dout[b][co][m - k + K/2]
__global__ void conv_bwd_in_kernel(const float *__restrict__ dout, const float *__restrict__ W,
                                   float *__restrict__ din, int B, int Ci, int Co, int N, int K) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)B * Ci * N) return;
    const int m = (int)(t % N), ci = (int)((t / N) % Ci);
    const long long b = t / ((long long)N * Ci);
    const int h = K / 2;
    float acc = 0.f;
    for (int co = 0; co < Co; ++co)
        for (int k = 0; k < K; ++k) {
            const int n = m - k + h;
            if (n >= 0 && n < N) acc = fmaf(W[((long long)co * Ci + ci) * K + k], dout[(b * Co + co) * N + n], acc);
        }
    din[t] = acc;
}

// d <- d (1 - a^2): back through tanh
__global__ void tanh_bwd_kernel(float *__restrict__ d, const float *__restrict__ a, long long count) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count) d[t] *= 1.f - a[t] * a[t];
}

// One warp per gradient entry: dW[co][ci][k] = sum_{b, n} dout[b][co][n] in[b][ci][n + k - K/2],
// then db[co] = sum_{b, n} dout[b][co][n]; lanes stride over (b, n), then a fixed
// shuffle tree.
__global__ void conv_bwd_w_kernel(const float *__restrict__ dout, const float *__restrict__ in, float *__restrict__ dW,
                                  float *__restrict__ db, int B, int Ci, int Co, int N, int K) {
    const long long wid = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const long long nw = (long long)Co * Ci * K;
    if (wid >= nw + Co) return;  // uniform across the warp
    const long long tot = (long long)B * N;
    const int h = K / 2;
    float acc = 0.f;
    if (wid < nw) {
        const int k = (int)(wid % K), ci = (int)((wid / K) % Ci), co = (int)(wid / ((long long)K * Ci));
        for (long long e = lane; e < tot; e += 32) {
            const long long b = e / N;
            const int n = (int)(e % N), nn = n + k - h;
            if (nn >= 0 && nn < N) acc = fmaf(dout[(b * Co + co) * N + n], in[(b * Ci + ci) * N + nn], acc);
        }
    } else {
        const int co = (int)(wid - nw);
        for (long long e = lane; e < tot; e += 32) acc += dout[((e / N) * Co + co) * N + e % N];
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) {
        if (wid < nw)
            dW[wid] = acc;
        else
            db[wid - nw] = acc;
    }
}

// Loss over S = B cout sequences of n points, e = y - t:
//   L = (sum e^2 + sum E^2) / (S n),  E_k = (e_1 + ... + e_k) / sqrt(n),
// the pointwise squared error plus that of the running sum along the body, which
// weighs smooth error components (the ones the force operator B amplifies in the
// CG residual) about n/3 times more than point-to-point ones.  dy = dL/dy;
// loss += L.  One block, one thread per sequence, fixed reduction order.
__global__ void seq_loss_kernel(const float *__restrict__ y, const float *__restrict__ t, float *__restrict__ dy,
                                int S, int n, float *__restrict__ loss) {
    __shared__ float red[1024];
    const float inv_rn = rsqrtf((float)n), scale = 2.f / ((float)S * (float)n);
    float acc = 0.f;
    for (int q = threadIdx.x; q < S; q += blockDim.x) {
        const float *yq = y + (long long)q * n, *tq = t + (long long)q * n;
        float *dq = dy + (long long)q * n;
        float run = 0.f;
        for (int k = 0; k < n; ++k) {
            const float e = yq[k] - tq[k];
            run += e;
            const float E = run * inv_rn;
            acc = fmaf(e, e, acc);
            acc = fmaf(E, E, acc);
            dq[k] = E;
        }
        float back = 0.f;  // sum over j >= k of dL/dE_j, times dE_j/de_k = 1/sqrt(n)
        for (int k = n - 1; k >= 0; --k) {
            back += scale * dq[k] * inv_rn;
            dq[k] = scale * (yq[k] - tq[k]) + back;
        }
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *loss += red[0] / ((float)S * (float)n);
}

__global__ void adam_kernel(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, long long n, float lr, float b1, float b2, float eps, float bc1,
                            float bc2) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float gt = g[t];
    const float mt = b1 * m[t] + (1.f - b1) * gt;
    const float vt = b2 * v[t] + (1.f - b2) * gt * gt;
    m[t] = mt;
    v[t] = vt;
    p[t] -= lr * (mt / bc1) / (sqrtf(vt / bc2) + eps);
}

// Features of the warm start for every body point (channels in warmstart.h).
// One block: the residual and the last change are scaled by their own RMS over
// the sample, so every step is a unit-size example of the same linear map; the
// residual's RMS goes to scale[0].
__global__ void ws_features_kernel(const double *__restrict__ ftmp, const double *__restrict__ bx,
                                   const double *__restrict__ f1, const double *__restrict__ d,
                                   const double *__restrict__ ub, const double *__restrict__ motion,
                                   const int *__restrict__ pbody, int np, float *__restrict__ feat,
                                   double *__restrict__ scale) {
    __shared__ double red[2][32];
    __shared__ double inv_s[2];
    double rr = 0.0, dd = 0.0;
    for (int i = threadIdx.x; i < 2 * np; i += blockDim.x) {
        const double r = ftmp[i] - bx[i];
        rr += r * r;
        dd += d[i] * d[i];
    }
    for (int o = 16; o > 0; o >>= 1) {
        rr += __shfl_xor_sync(0xffffffffu, rr, o);
        dd += __shfl_xor_sync(0xffffffffu, dd, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = rr;
        red[1][threadIdx.x >> 5] = dd;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            a += red[0][w];
            b += red[1][w];
        }
        const double sr = sqrt(a / (2.0 * np)), sd = sqrt(b / (2.0 * np));
        inv_s[0] = sr > 0.0 ? 1.0 / sr : 0.0;
        inv_s[1] = sd > 0.0 ? 1.0 / sd : 0.0;
        scale[0] = sr;
    }
    __syncthreads();
    for (int p = threadIdx.x; p < np; p += blockDim.x) {
        const double ang = motion[6 * pbody[p] + 4];
        float *f = feat + p;
        f[0 * np] = (float)((ftmp[p] - bx[p]) * inv_s[0]);
        f[1 * np] = (float)((ftmp[np + p] - bx[np + p]) * inv_s[0]);
        f[2 * np] = (float)f1[p];
        f[3 * np] = (float)f1[np + p];
        f[4 * np] = (float)(d[p] * inv_s[1]);
        f[5 * np] = (float)(d[np + p] * inv_s[1]);
        f[6 * np] = (float)ub[p];
        f[7 * np] = (float)ub[np + p];
        f[8 * np] = (float)cos(ang);
        f[9 * np] = (float)sin(ang);
    }
}

// z = [f1 | d], d = f1 - f2 (the last change); then f2 <- f1.
__global__ void ws_direction_kernel(const double *__restrict__ f1, double *__restrict__ f2, int np,
                                    double *__restrict__ z) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * np) return;
    const double a = f1[i];
    z[i] = a;
    z[2 * np + i] = a - f2[i];
    f2[i] = a;
}

// p = out_mean[c] + out_std[c] y[c][p]: the network's output in solver units.
__global__ void ws_prediction_kernel(const float *__restrict__ y, const float *__restrict__ om,
                                     const float *__restrict__ os, int np, double *__restrict__ p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * np) return;
    const int c = i / np;
    p[i] = (double)om[c] + (double)os[c] * (double)y[i];
}

// One block.  z = [f1 | v_1 .. v_k], bz = B z (k = 1 or 2 directions).  Galerkin
// step in the B-energy norm: G y = h with G_ij = (v_i.B v_j + v_j.B v_i) / 2 and
// h_i = v_i.(b - B f1); x = f1 + sum y_i v_i, c = B f1 + sum y_i B v_i.  A
// system that is not positive definite falls back to the first direction alone,
// and then to y = 0 (x = f1).
__global__ void ws_galerkin_kernel(const double *__restrict__ z, const double *__restrict__ bz,
                                   const double *__restrict__ b, double *__restrict__ x, double *__restrict__ c,
                                   double *__restrict__ x2, double *__restrict__ c2, int np, int k,
                                   double *__restrict__ coef) {
    constexpr int NS = 6;  // v1.Bv1, v1.Bv2, v2.Bv1, v2.Bv2, h1, h2
    __shared__ double red[NS][32];
    __shared__ double ys[2];
    const int n = 2 * np;
    double acc[NS] = {0, 0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double r = b[i] - bz[i];
        const double v1 = z[n + i], bv1 = bz[n + i];
        acc[0] += v1 * bv1;
        acc[4] += v1 * r;
        if (k > 1) {
            const double v2 = z[2 * n + i], bv2 = bz[2 * n + i];
            acc[1] += v1 * bv2;
            acc[2] += v2 * bv1;
            acc[3] += v2 * bv2;
            acc[5] += v2 * r;
        }
    }
#pragma unroll
    for (int q = 0; q < NS; ++q) {
        double v = acc[q];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t[NS];
        for (int q = 0; q < NS; ++q) {
            t[q] = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t[q] += red[q][w];
        }
        double y1 = 0.0, y2 = 0.0;
        bool done = false;
        if (k > 1) {
            const double g11 = t[0], g22 = t[3], g12 = 0.5 * (t[1] + t[2]);
            const double det = g11 * g22 - g12 * g12;
            if (g11 > 0.0 && g22 > 0.0 && det > 1e-12 * g11 * g22) {
                y1 = (t[4] * g22 - t[5] * g12) / det;
                y2 = (t[5] * g11 - t[4] * g12) / det;
                done = isfinite(y1) && isfinite(y2);
            }
        }
        if (!done) {
            y2 = 0.0;
            y1 = t[0] > 0.0 ? t[4] / t[0] : 0.0;
            if (!isfinite(y1)) y1 = 0.0;
        }
        ys[0] = y1;
        ys[1] = y2;
        if (coef) {
            coef[0] = y1;
            if (k > 1) coef[1] = y2;
        }
    }
    __syncthreads();
    const double y1 = ys[0], y2 = ys[1];
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double xi = z[i] + y1 * z[n + i], ci = bz[i] + y1 * bz[n + i];
        if (k > 1) {
            xi += y2 * z[2 * n + i];
            ci += y2 * bz[2 * n + i];
        }
        x[i] = xi;
        c[i] = ci;
        if (x2) {
            x2[i] = xi;
            c2[i] = ci;
        }
    }
}

// Projection onto previous solutions (Fischer's method for successive right-hand
// sides).  V = hist[0 .. k) (most recent first, zero when not yet filled),
// BV = B V.  One warp per entry of the Gram system: G_ij = (v_i.Bv_j + v_j.Bv_i) / 2
// for i <= j, h_i = v_i.b; entry e < k(k+1)/2 is (i, j) in row-major upper order,
// then the k entries of h.
__global__ void ws_gram_kernel(const double *__restrict__ V, const double *__restrict__ BV,
                               const double *__restrict__ b, int n, int k, double *__restrict__ G,
                               double *__restrict__ h) {
    const int e = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    const int npair = k * (k + 1) / 2;
    if (e >= npair + k) return;  // uniform across the warp
    double a = 0.0, c = 0.0;
    if (e < npair) {
        int i = 0, r = e;
        while (r >= k - i) {
            r -= k - i;
            ++i;
        }
        const int j = i + r;
        const double *vi = V + (long long)i * n, *vj = V + (long long)j * n;
        const double *bi = BV + (long long)i * n, *bj = BV + (long long)j * n;
        for (int t = lane; t < n; t += 32) {
            a += vi[t] * bj[t];
            c += vj[t] * bi[t];
        }
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            c += __shfl_down_sync(0xffffffffu, c, o);
        }
        if (lane == 0) {
            G[i * k + j] = 0.5 * (a + c);
            G[j * k + i] = 0.5 * (a + c);
        }
    } else {
        const int i = e - npair;
        const double *vi = V + (long long)i * n;
        for (int t = lane; t < n; t += 32) a += vi[t] * b[t];
        for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
        if (lane == 0) h[i] = a;
    }
}

// One thread: G y = h by Cholesky in the given order (most recent direction
// first), dropping a direction whose pivot falls below 1e-10 of its diagonal
// (zero vectors and directions the earlier ones already span); y_i = 0 for the
// dropped ones.  Then x = sum y_i v_i and c = sum y_i B v_i (c = B x for the CG).
constexpr int kWsMaxDepth = 16;
__global__ void ws_project_kernel(const double *__restrict__ V, const double *__restrict__ BV,
                                  const double *__restrict__ G, const double *__restrict__ h, int n, int k,
                                  double *__restrict__ x, double *__restrict__ c, double *__restrict__ kept) {
    __shared__ double y[kWsMaxDepth];
    if (threadIdx.x == 0) {
        double Lm[kWsMaxDepth][kWsMaxDepth];
        bool keep[kWsMaxDepth];
        double z[kWsMaxDepth];
        int nk = 0;
        for (int i = 0; i < k; ++i) {
            keep[i] = false;
            y[i] = 0.0;
            const double gii = G[i * k + i];
            if (!(gii > 0.0)) continue;
            for (int j = 0; j < i; ++j) {
                if (!keep[j]) continue;
                double sm = G[i * k + j];
                for (int l = 0; l < j; ++l)
                    if (keep[l]) sm -= Lm[i][l] * Lm[j][l];
                Lm[i][j] = sm / Lm[j][j];
            }
            double d = gii;
            for (int l = 0; l < i; ++l)
                if (keep[l]) d -= Lm[i][l] * Lm[i][l];
            if (d > 1e-10 * gii && isfinite(d)) {
                Lm[i][i] = sqrt(d);
                keep[i] = true;
                ++nk;
            }
        }
        for (int i = 0; i < k; ++i) {  // L z = h
            if (!keep[i]) continue;
            double sm = h[i];
            for (int l = 0; l < i; ++l)
                if (keep[l]) sm -= Lm[i][l] * z[l];
            z[i] = sm / Lm[i][i];
        }
        for (int i = k - 1; i >= 0; --i) {  // L^T y = z
            if (!keep[i]) continue;
            double sm = z[i];
            for (int l = i + 1; l < k; ++l)
                if (keep[l]) sm -= Lm[l][i] * y[l];
            y[i] = sm / Lm[i][i];
        }
        if (kept) *kept = (double)nk;
    }
    __syncthreads();
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        double xv = 0.0, cv = 0.0;
        for (int i = 0; i < k; ++i) {
            xv += y[i] * V[(long long)i * n + t];
            cv += y[i] * BV[(long long)i * n + t];
        }
        x[t] = xv;
        c[t] = cv;
    }
}

// hist[j] <- hist[j-1] for j = k-1 .. 1, hist[0] <- f (vectors of n doubles).
__global__ void ws_shift_kernel(double *__restrict__ hist, const double *__restrict__ f, int n, int k) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        for (int j = k - 1; j > 0; --j) hist[(long long)j * n + t] = hist[(long long)(j - 1) * n + t];
        hist[t] = f[t];
    }
}

// ---- host-side passes ----

size_t act_floats(const ibpm_net *net, int B, int n) {
    size_t s = (size_t)net->cin;
    for (int l = 0; l < net->layers; ++l) s += (size_t)net->lco[l];
    return s * (size_t)B * (size_t)n;
}

// Forward pass storing every layer's activation in act: act[0] the normalised
// input, then the output of layer 1 .. L.  x is the raw features; idx (device,
// optional) gathers the batch.  Returns the output of the last layer.
float *forward(const ibpm_net *net, const float *x, const int *idx, int B, int n, float *act, cudaStream_t st) {
    const float *nm = net->norm;
    normalise_kernel<<<blocks_for((long long)B * net->cin * n), kThreads, 0, st>>>(x, idx, act, B, net->cin, n, nm,
                                                                                    nm + net->cin);
    float *in = act;
    for (int l = 0; l < net->layers; ++l) {
        float *out = in + (size_t)net->lci[l] * B * n;
        conv_fwd_kernel<<<blocks_for((long long)B * net->lco[l] * n), kThreads, 0, st>>>(
            in, net->params + net->woff[l], net->params + net->boff[l], out, B, net->lci[l], net->lco[l], n,
            net->ksize, l + 1 < net->layers);
        in = out;
    }
    NCK(cudaGetLastError());
    return in;
}

// Loss on the normalised targets of the batch and the gradient of the
// parameters into net->grad.  t_norm [B][cout][n] is already normalised.
void backward(ibpm_net *net, const float *y, const float *t_norm, int B, int n, cudaStream_t st) {
    size_t maxc = 0;
    for (int l = 0; l < net->layers; ++l) maxc = std::max<size_t>(maxc, (size_t)std::max(net->lci[l], net->lco[l]));
    ensure(net, net->dbuf, net->dbuf_cap, 2 * maxc * (size_t)B * n);
    float *d = net->dbuf, *dn = net->dbuf + maxc * (size_t)B * n;
    seq_loss_kernel<<<1, 1024, 0, st>>>(y, t_norm, d, B * net->cout, n, net->loss);
    // activation offsets
    std::vector<float *> a(net->layers + 1);
    a[0] = net->act;
    for (int l = 0; l < net->layers; ++l) a[l + 1] = a[l] + (size_t)net->lci[l] * B * n;
    for (int l = net->layers - 1; l >= 0; --l) {
        const int Ci = net->lci[l], Co = net->lco[l];
        if (l + 1 < net->layers)
            tanh_bwd_kernel<<<blocks_for((long long)B * Co * n), kThreads, 0, st>>>(d, a[l + 1], (long long)B * Co * n);
        const long long nwarp = (long long)Co * Ci * net->ksize + Co;
        conv_bwd_w_kernel<<<blocks_for(nwarp * 32), kThreads, 0, st>>>(d, a[l], net->grad + net->woff[l],
                                                                        net->grad + net->boff[l], B, Ci, Co, n,
                                                                        net->ksize);
        if (l > 0) {
            conv_bwd_in_kernel<<<blocks_for((long long)B * Ci * n), kThreads, 0, st>>>(
                d, net->params + net->woff[l], dn, B, Ci, Co, n, net->ksize);
            std::swap(d, dn);
        }
    }
    NCK(cudaGetLastError());
}

void adam_step(ibpm_net *net, float lr, cudaStream_t st) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    ++net->adam_t;
    const float bc1 = 1.f - (float)std::pow((double)b1, (double)net->adam_t);
    const float bc2 = 1.f - (float)std::pow((double)b2, (double)net->adam_t);
    adam_kernel<<<blocks_for(net->nparams), kThreads, 0, st>>>(net->params, net->grad, net->m, net->v, net->nparams, lr,
                                                                b1, b2, eps, bc1, bc2);
    NCK(cudaGetLastError());
}

// device copy of raw host samples for one call
void upload(ibpm_net *net, const DevTmp &buf, const float *src, size_t nfloat) {
    NCK(cudaMemcpyAsync(buf.p, src, nfloat * sizeof(float), cudaMemcpyHostToDevice, net->st));
}

}  // namespace

// ---- interface to the engine ----

size_t net_act_floats(const ibpm_net *net, int B, int n) { return act_floats(net, B, n); }
void net_forward_dev(const ibpm_net *net, const float *x, int B, int n, float *act, float *y, cudaStream_t st) {
    float *out = forward(net, x, nullptr, B, n, act, st);
    NCK(cudaMemcpyAsync(y, out, sizeof(float) * (size_t)B * net->cout * n, cudaMemcpyDeviceToDevice, st));
}
int net_device(const ibpm_net *net) { return net->device; }
int net_cin(const ibpm_net *net) { return net->cin; }
int net_cout(const ibpm_net *net) { return net->cout; }

void launch_ws_features(const double *ftmp, const double *bx, const double *f1, const double *d, const double *ub,
                        const double *motion, const int *pbody, int np, float *feat, double *scale, cudaStream_t st) {
    ws_features_kernel<<<1, 256, 0, st>>>(ftmp, bx, f1, d, ub, motion, pbody, np, feat, scale);
}
void launch_ws_direction(const double *f1, double *f2, int np, double *z, cudaStream_t st) {
    ws_direction_kernel<<<(2 * np + 127) / 128, 128, 0, st>>>(f1, f2, np, z);
}
void launch_ws_prediction(const float *y, const ibpm_net *net, int np, double *p, cudaStream_t st) {
    const float *om = net->norm + 2 * net->cin, *os = om + net->cout;
    ws_prediction_kernel<<<(2 * np + 127) / 128, 128, 0, st>>>(y, om, os, np, p);
}
void launch_ws_galerkin(const double *z, const double *bz, const double *b, double *x, double *c, double *x2,
                        double *c2, int np, int k, double *coef, cudaStream_t st) {
    ws_galerkin_kernel<<<1, 256, 0, st>>>(z, bz, b, x, c, x2, c2, np, k, coef);
}

void launch_ws_projection(const double *V, const double *BV, const double *b, double *x, double *c, int n, int k,
                          double *G, double *h, double *kept, cudaStream_t st) {
    const int items = k * (k + 1) / 2 + k;
    ws_gram_kernel<<<(items * 32 + 255) / 256, 256, 0, st>>>(V, BV, b, n, k, G, h);
    // the solve runs on thread 0 of block 0; every block then forms its share of x and c
    ws_project_kernel<<<1, 256, 0, st>>>(V, BV, G, h, n, k, x, c, kept);
}
void launch_ws_shift(double *hist, const double *f, int n, int k, cudaStream_t st) {
    ws_shift_kernel<<<(n + 255) / 256, 256, 0, st>>>(hist, f, n, k);
}

}  // namespace ibpm

using namespace ibpm;

extern "C" {

int ibpm_net_create(int32_t cin, int32_t width, int32_t kernel, int32_t layers, int32_t cout, uint64_t seed,
                    int32_t device, ibpm_net **out) {
    if (!out) return IBPM_ERR_INVALID;
    *out = nullptr;
    if (cin < 1 || width < 1 || cout < 1 || layers < 1 || kernel < 1 || kernel % 2 == 0) {
        g_create_err = "channels, width and layers must be positive and the kernel size odd";
        return IBPM_ERR_INVALID;
    }
    ibpm_net *net = new ibpm_net;
    net->device = device;
    net->cin = cin;
    net->width = width;
    net->ksize = kernel;
    net->layers = layers;
    net->cout = cout;
    try {
        NCK(cudaSetDevice(device));
        NCK(cudaStreamCreateWithFlags(&net->st, cudaStreamNonBlocking));
        for (int l = 0; l < layers; ++l) {
            net->lci.push_back(l == 0 ? cin : width);
            net->lco.push_back(l + 1 == layers ? cout : width);
            net->woff.push_back(net->nparams);
            net->nparams += (long long)net->lco[l] * net->lci[l] * kernel;
            net->boff.push_back(net->nparams);
            net->nparams += net->lco[l];
        }
        net->params = net_alloc(net, net->nparams);
        net->grad = net_alloc(net, net->nparams);
        net->m = net_alloc(net, net->nparams);
        net->v = net_alloc(net, net->nparams);
        net->norm = net_alloc(net, 2 * (cin + cout));
        net->loss = net_alloc(net, 1);
        // Glorot-uniform weights (tanh layers), the last layer scaled by 0.1 so the
        // untrained prediction is close to zero; zero biases.
        std::vector<float> w(net->nparams, 0.f);
        uint64_t s = seed;
        for (int l = 0; l < layers; ++l) {
            const double fan = (double)(net->lci[l] + net->lco[l]) * kernel;
            const double bound = std::sqrt(6.0 / fan) * (l + 1 == layers ? 0.1 : 1.0);
            for (long long k = net->woff[l]; k < net->boff[l]; ++k) w[k] = (float)((2 * uniform01(s) - 1) * bound);
        }
        NCK(cudaMemcpyAsync(net->params, w.data(), sizeof(float) * w.size(), cudaMemcpyHostToDevice, net->st));
        std::vector<float> nm(2 * (cin + cout), 0.f);
        for (int c = 0; c < cin; ++c) nm[cin + c] = 1.f;
        for (int c = 0; c < cout; ++c) nm[2 * cin + cout + c] = 1.f;
        NCK(cudaMemcpyAsync(net->norm, nm.data(), sizeof(float) * nm.size(), cudaMemcpyHostToDevice, net->st));
        NCK(cudaStreamSynchronize(net->st));
    } catch (const NetError &e) {
        g_create_err = e.msg;
        ibpm_net_destroy(net);
        (void)cudaGetLastError();
        return e.code;
    }
    *out = net;
    return IBPM_OK;
}

void ibpm_net_destroy(ibpm_net *net) {
    if (!net) return;
    cudaSetDevice(net->device);
    if (net->st) cudaStreamSynchronize(net->st);
    for (void *p : net->bufs) cudaFree(p);
    if (net->st) cudaStreamDestroy(net->st);
    delete net;
}

int64_t ibpm_net_num_params(const ibpm_net *net) { return net ? net->nparams : -1; }

const char *ibpm_net_last_error(const ibpm_net *net) { return net ? net->err.c_str() : g_create_err.c_str(); }

int ibpm_net_get_params(ibpm_net *net, float *params) {
    return guarded(net, [&] {
        if (!params) throw NetError{IBPM_ERR_INVALID, "null buffer"};
        NCK(cudaMemcpyAsync(params, net->params, sizeof(float) * net->nparams, cudaMemcpyDeviceToHost, net->st));
        NCK(cudaStreamSynchronize(net->st));
    });
}

int ibpm_net_set_params(ibpm_net *net, const float *params) {
    return guarded(net, [&] {
        if (!params) throw NetError{IBPM_ERR_INVALID, "null buffer"};
        NCK(cudaMemcpyAsync(net->params, params, sizeof(float) * net->nparams, cudaMemcpyHostToDevice, net->st));
        NCK(cudaMemsetAsync(net->m, 0, sizeof(float) * net->nparams, net->st));
        NCK(cudaMemsetAsync(net->v, 0, sizeof(float) * net->nparams, net->st));
        net->adam_t = 0;
        NCK(cudaStreamSynchronize(net->st));
    });
}

int ibpm_net_set_normalisation(ibpm_net *net, const float *in_mean, const float *in_std, const float *out_mean,
                               const float *out_std) {
    return guarded(net, [&] {
        if (!in_mean || !in_std || !out_mean || !out_std) throw NetError{IBPM_ERR_INVALID, "null buffer"};
        std::vector<float> nm;
        nm.insert(nm.end(), in_mean, in_mean + net->cin);
        nm.insert(nm.end(), in_std, in_std + net->cin);
        nm.insert(nm.end(), out_mean, out_mean + net->cout);
        nm.insert(nm.end(), out_std, out_std + net->cout);
        for (int c = 0; c < net->cin; ++c)
            if (!(in_std[c] > 0.f)) throw NetError{IBPM_ERR_INVALID, "standard deviations must be positive"};
        for (int c = 0; c < net->cout; ++c)
            if (!(out_std[c] > 0.f)) throw NetError{IBPM_ERR_INVALID, "standard deviations must be positive"};
        NCK(cudaMemcpyAsync(net->norm, nm.data(), sizeof(float) * nm.size(), cudaMemcpyHostToDevice, net->st));
        NCK(cudaStreamSynchronize(net->st));
    });
}

int ibpm_net_get_normalisation(ibpm_net *net, float *in_mean, float *in_std, float *out_mean, float *out_std) {
    return guarded(net, [&] {
        std::vector<float> nm(2 * (net->cin + net->cout));
        NCK(cudaMemcpyAsync(nm.data(), net->norm, sizeof(float) * nm.size(), cudaMemcpyDeviceToHost, net->st));
        NCK(cudaStreamSynchronize(net->st));
        const int ci = net->cin, co = net->cout;
        if (in_mean) std::copy(nm.begin(), nm.begin() + ci, in_mean);
        if (in_std) std::copy(nm.begin() + ci, nm.begin() + 2 * ci, in_std);
        if (out_mean) std::copy(nm.begin() + 2 * ci, nm.begin() + 2 * ci + co, out_mean);
        if (out_std) std::copy(nm.begin() + 2 * ci + co, nm.end(), out_std);
    });
}

int ibpm_net_forward(ibpm_net *net, const float *x, int64_t batch, int32_t n, float *y) {
    return guarded(net, [&] {
        if (!x || !y || batch < 1 || n < 1) throw NetError{IBPM_ERR_INVALID, "bad forward arguments"};
        DevTmp dx(sizeof(float) * (size_t)batch * net->cin * n);
        upload(net, dx, x, (size_t)batch * net->cin * n);
        ensure(net, net->act, net->act_cap, act_floats(net, (int)batch, n));
        const float *out = forward(net, dx.f(), nullptr, (int)batch, n, net->act, net->st);
        const size_t cnt = (size_t)batch * net->cout * n;
        std::vector<float> yn(cnt), nm(2 * (net->cin + net->cout));
        NCK(cudaMemcpyAsync(yn.data(), out, sizeof(float) * cnt, cudaMemcpyDeviceToHost, net->st));
        NCK(cudaMemcpyAsync(nm.data(), net->norm, sizeof(float) * nm.size(), cudaMemcpyDeviceToHost, net->st));
        NCK(cudaStreamSynchronize(net->st));
        const float *om = nm.data() + 2 * net->cin, *os = om + net->cout;
        for (size_t i = 0; i < cnt; ++i) {
            const int c = (int)((i / n) % net->cout);
            y[i] = om[c] + os[c] * yn[i];
        }
    });
}

int ibpm_net_loss_grad(ibpm_net *net, const float *x, const float *t, int64_t batch, int32_t n, float *loss,
                       float *grad) {
    return guarded(net, [&] {
        if (!x || !t || batch < 1 || n < 1) throw NetError{IBPM_ERR_INVALID, "bad gradient arguments"};
        const int B = (int)batch;
        DevTmp dx(sizeof(float) * (size_t)B * net->cin * n), dt(sizeof(float) * (size_t)B * net->cout * n);
        upload(net, dx, x, (size_t)B * net->cin * n);
        upload(net, dt, t, (size_t)B * net->cout * n);
        ensure(net, net->act, net->act_cap, act_floats(net, B, n));
        ensure(net, net->bt, net->bt_cap, (size_t)B * net->cout * n);
        const float *nm = net->norm;
        normalise_kernel<<<blocks_for((long long)B * net->cout * n), kThreads, 0, net->st>>>(
            dt.f(), nullptr, net->bt, B, net->cout, n, nm + 2 * net->cin, nm + 2 * net->cin + net->cout);
        const float *y = forward(net, dx.f(), nullptr, B, n, net->act, net->st);
        NCK(cudaMemsetAsync(net->loss, 0, sizeof(float), net->st));
        backward(net, y, net->bt, B, n, net->st);
        if (loss) NCK(cudaMemcpyAsync(loss, net->loss, sizeof(float), cudaMemcpyDeviceToHost, net->st));
        if (grad) NCK(cudaMemcpyAsync(grad, net->grad, sizeof(float) * net->nparams, cudaMemcpyDeviceToHost, net->st));
        NCK(cudaStreamSynchronize(net->st));
    });
}

int ibpm_net_train(ibpm_net *net, const float *x, const float *t, int64_t nsamples, int32_t n, int32_t epochs,
                   int32_t batch, float lr, uint64_t seed, float *epoch_loss) {
    return guarded(net, [&] {
        if (!x || !t || nsamples < 1 || n < 1 || epochs < 1 || batch < 1 || !(lr > 0.f))
            throw NetError{IBPM_ERR_INVALID, "bad training arguments"};
        const int B = (int)std::min<int64_t>(batch, nsamples);
        DevTmp dx(sizeof(float) * (size_t)nsamples * net->cin * n), dt(sizeof(float) * (size_t)nsamples * net->cout * n),
            didx(sizeof(int) * (size_t)nsamples);
        upload(net, dx, x, (size_t)nsamples * net->cin * n);
        upload(net, dt, t, (size_t)nsamples * net->cout * n);
        int *idx = static_cast<int *>(didx.p);
        ensure(net, net->act, net->act_cap, act_floats(net, B, n));
        ensure(net, net->bt, net->bt_cap, (size_t)B * net->cout * n);
        std::vector<int> perm(nsamples);
        uint64_t s = seed;
        const float *nm = net->norm;
        for (int e = 0; e < epochs; ++e) {
            for (int64_t i = 0; i < nsamples; ++i) perm[i] = (int)i;
            for (int64_t i = nsamples - 1; i > 0; --i) std::swap(perm[i], perm[(int64_t)(splitmix64(s) % (uint64_t)(i + 1))]);
            NCK(cudaMemcpyAsync(idx, perm.data(), sizeof(int) * nsamples, cudaMemcpyHostToDevice, net->st));
            NCK(cudaMemsetAsync(net->loss, 0, sizeof(float), net->st));
            int nb = 0;
            for (int64_t b0 = 0; b0 + B <= nsamples; b0 += B, ++nb) {  // full batches only
                normalise_kernel<<<blocks_for((long long)B * net->cout * n), kThreads, 0, net->st>>>(
                    dt.f(), idx + b0, net->bt, B, net->cout, n, nm + 2 * net->cin, nm + 2 * net->cin + net->cout);
                const float *y = forward(net, dx.f(), idx + b0, B, n, net->act, net->st);
                backward(net, y, net->bt, B, n, net->st);
                adam_step(net, lr, net->st);
            }
            float l = 0.f;
            NCK(cudaMemcpyAsync(&l, net->loss, sizeof(float), cudaMemcpyDeviceToHost, net->st));
            NCK(cudaStreamSynchronize(net->st));
            if (epoch_loss) epoch_loss[e] = nb ? l / (float)nb : 0.f;
        }
        NCK(cudaStreamSynchronize(net->st));
    });
}

}  // extern "C"
