// Dense DST-I passes on the fifth-generation tensor cores (see tc_dst.h).
//
// A tile is D[k][l] for 128 output frequencies k (rows of S) and 256 lines l of
// one field over the whole line length P, accumulated in 256 columns of tensor
// memory by tcgen05.mma (M 128, N 256, K 16; BF16 x BF16 -> FP32) from K-blocks
// of 64 elements (128-byte rows, 128-byte swizzle) that TMA brings into a ring
// of shared-memory stages; the epilogue reads its rows with tcgen05.ld and
// writes row k as line k of the next pass (rows become lines).
// Every wait on an mbarrier gives up after one second of global time, sets the
// caller's error flag and lets the CTA finish (freeing its tensor memory); no wait
// depends on another CTA.  No load here uses cluster-wide delivery.
#include "tc_dst.h"

#include <cuda.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

namespace {

constexpr int kTileM = 128;   // rows of S per CTA
constexpr int kTileN = 256;   // lines per CTA
constexpr int kBlockK = 64;   // elements per K-block: one 128-byte swizzle row
constexpr uint32_t kTmemCols = 256;
constexpr int kBytesA = kTileM * kBlockK * 2;  // 16 KB
constexpr int kBytesB = kTileN * kBlockK * 2;  // 32 KB

enum { EPI_SPLIT = 0, EPI_MULT = 1, EPI_F64 = 2 };

template <int NPROD>
struct Cfg {
    static constexpr int kParts = NPROD == 3 ? 2 : 1;
    static constexpr int kStageBytes = kParts * (kBytesA + kBytesB);
    static constexpr int kStages = NPROD == 3 ? 2 : 4;
    // the operand ring, four epilogue staging tiles and alignment slack
    static constexpr size_t kSmem = (size_t)kStages * kStageBytes + 4 * 32 * 33 * sizeof(float) + 1024;
};

struct PassArgs {
    int P;
    __nv_bfloat16 *oh, *ol;   // next pass's lines (EPI_SPLIT, EPI_MULT)
    const float *mult;        // [k][l] multipliers (EPI_MULT)
    double *out;              // result (EPI_F64)
    long long bs;
    int ld;
    TcKeep keep;              // which result elements are stored (EPI_F64)
    int *err;
};

// 0-based (x, y) of the result: stored or not
__device__ __forceinline__ bool kept(const TcKeep &k, int x, int y) {
    if (k.mode == TC_KEEP_WINDOW)
        return x >= k.win[0] - 2 && x <= k.win[1] && y >= k.win[2] - 2 && y <= k.win[3];
    if (k.mode == TC_KEEP_LINES)
        return y == k.lines[0] || y == k.lines[1] || x == k.lines[2] || x == k.lines[3];
    return true;
}

__device__ __forceinline__ uint32_t saddr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t gtime() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(b)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t *b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(saddr(b)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase of the given parity to complete; false after one second.
__device__ __forceinline__ bool mbar_wait(uint64_t *b, uint32_t parity) {
    if (mbar_try(b, parity)) return true;
    const uint64_t t0 = gtime();
    for (;;) {
        for (int i = 0; i < 32; ++i)
            if (mbar_try(b, parity)) return true;
        if (gtime() - t0 > 1000000000ull) return false;
    }
}

__device__ __forceinline__ void tma_load(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
            saddr(dst)),
        "l"((uint64_t)map), "r"(saddr(bar)), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory operand descriptor: K-major, 128-byte swizzle, 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t a) {
    uint64_t d = (uint64_t)((a & 0x3FFFFu) >> 4);
    d |= (uint64_t)1 << 16;           // leading offset (unused by swizzled K-major layouts)
    d |= (uint64_t)(1024 >> 4) << 32; // stride between 8-row groups
    d |= (uint64_t)1 << 46;           // descriptor version
    d |= (uint64_t)2 << 61;           // 128-byte swizzle
    return d;
}

// kind::f16 instruction descriptor: BF16 A and B (K-major), FP32 D, M 128, N 256
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kTileN >> 3) << 17) |
                            ((uint32_t)(kTileM >> 4) << 24);

__device__ __forceinline__ void mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
        "l"(a), "l"(b), "r"(kIdesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Rows row0 .. row0 + 31 of a tile (one warp, lane = row), columns col0 .. col0
// + 31 (v: FP32 bits from tensor memory): multiplied (EPI_MULT), then stored as
// the next pass's BF16 parts (EPI_SPLIT, EPI_MULT) or as the FP64 result
// (EPI_F64: interior elements that the selection keeps).  The warp's staging
// tile stg (32 x 33 floats, conflict-free both ways) turns the stores into
// coalesced 64-byte (BF16) and 256-byte (FP64) row segments.
constexpr int kStageLd = 33;
constexpr int kStageFloats = 32 * kStageLd;

template <int NPROD, int EPI>
__device__ __forceinline__ void epilogue_staged(const PassArgs &a, int f, int row0, int col0, const uint32_t (&v)[32],
                                                float *stg) {
    const int lane = threadIdx.x & 31, P = a.P;
    float x[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) x[j] = __uint_as_float(v[j]);
    if (EPI == EPI_MULT) {
        const float4 *mp = reinterpret_cast<const float4 *>(a.mult + (size_t)(row0 + lane) * P + col0);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const float4 m = __ldg(mp + q);
            x[4 * q] *= m.x;
            x[4 * q + 1] *= m.y;
            x[4 * q + 2] *= m.z;
            x[4 * q + 3] *= m.w;
        }
    }
#pragma unroll
    for (int j = 0; j < 32; ++j) stg[lane * kStageLd + j] = x[j];
    __syncwarp();
    if (EPI == EPI_F64) {
        const int col = col0 + lane;
        double *o = a.out + (long long)f * a.bs + col;
        for (int r = 0; r < 32; ++r) {
            const int row = row0 + r;
            if (row < P - 1 && col < P - 1 && kept(a.keep, col, row))
                o[(long long)row * a.ld] = (double)stg[r * kStageLd + lane];
        }
    } else {
        const int q = lane & 3;
#pragma unroll
        for (int it = 0; it < 4; ++it) {
            const int r = it * 8 + (lane >> 2);
            __align__(16) __nv_bfloat16 h[8];
            __align__(16) __nv_bfloat16 l[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) tc_split(stg[r * kStageLd + 8 * q + i], h[i], l[i]);
            const size_t off = ((size_t)f * P + row0 + r) * P + col0 + 8 * q;
            *reinterpret_cast<uint4 *>(a.oh + off) = *reinterpret_cast<const uint4 *>(h);
            if (NPROD == 3) *reinterpret_cast<uint4 *>(a.ol + off) = *reinterpret_cast<const uint4 *>(l);
        }
    }
    __syncwarp();
}

// One CTA per SM walks the tiles (M-tiles fastest, so the CTAs working at once
// share each line tile through L2).  Two accumulators of
// 256 tensor-memory columns let the epilogue of one tile run while the products
// of the next accumulate.  Warps: 0 producer (one lane), 1 products (one lane;
// the whole warp allocates and frees the 512 columns), 2..5 epilogue (warp w
// reads lanes 32 (w % 4) ..).
constexpr int kThreads = 192;

template <int NPROD, int EPI>
__global__ void __launch_bounds__(kThreads, 1)
    tc_dst_pass_kernel(const __grid_constant__ CUtensorMap tSh, const __grid_constant__ CUtensorMap tSl,
                             const __grid_constant__ CUtensorMap tXh, const __grid_constant__ CUtensorMap tXl,
                             PassArgs a, int nf) {
    using C = Cfg<NPROD>;
    extern __shared__ uint8_t smem_raw[];
    __shared__ uint64_t full[C::kStages], empty[C::kStages], accf[2], acce[2], fin;
    __shared__ uint32_t tmem_s;
    __shared__ int fail_s;
    uint8_t *smem = smem_raw + ((1024u - (saddr(smem_raw) & 1023u)) & 1023u);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int P = a.P, KB = P / kBlockK, MT = P / kTileM, NT = P / kTileN;
    // epilogue warp w (2..5) stages through its own tile after the operand ring
    float *stg = reinterpret_cast<float *>(smem + (size_t)C::kStages * C::kStageBytes) +
                 (warp >= 2 ? (warp - 2) * kStageFloats : 0);
    const int ntiles = nf * MT * NT;

    if (threadIdx.x == 0) {
        for (int s = 0; s < C::kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&accf[b], 1);
            mbar_init(&acce[b], 128);
        }
        mbar_init(&fin, 1);
        fail_s = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&tmem_s)),
                     "r"(2 * kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_s;

    auto stage_a = [&](int s, int part) { return smem + (size_t)s * C::kStageBytes + part * kBytesA; };
    auto stage_b = [&](int s, int part) {
        return smem + (size_t)s * C::kStageBytes + C::kParts * kBytesA + part * kBytesB;
    };

    if (warp == 0) {
        if (lane == 0) {
            int kc = 0;  // K-blocks loaded so far (the ring position)
            for (int t = blockIdx.x; t < ntiles && !fail_s; t += gridDim.x) {
                const int m0 = (t % MT) * kTileM, n0 = ((t / MT) % NT) * kTileN, f = t / (MT * NT);
                for (int kb = 0; kb < KB; ++kb, ++kc) {
                    const int s = kc % C::kStages;
                    if (kc >= C::kStages && !mbar_wait(&empty[s], ((kc / C::kStages) - 1) & 1)) {
                        atomicExch(&fail_s, 1);
                        break;
                    }
                    mbar_expect_tx(&full[s], C::kStageBytes);
                    const int x = kb * kBlockK;
                    tma_load(stage_a(s, 0), &tSh, &full[s], x, m0);
                    tma_load(stage_b(s, 0), &tXh, &full[s], x, f * P + n0);
                    if (NPROD == 3) {
                        tma_load(stage_a(s, 1), &tSl, &full[s], x, m0);
                        tma_load(stage_b(s, 1), &tXl, &full[s], x, f * P + n0);
                    }
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            int kc = 0, i = 0;
            for (int t = blockIdx.x; t < ntiles && !fail_s; t += gridDim.x, ++i) {
                const int b = i & 1, u = i >> 1;
                if (u >= 1 && !mbar_wait(&acce[b], (u - 1) & 1)) {
                    atomicExch(&fail_s, 1);
                    break;
                }
                tc_fence_after();
                const uint32_t acc = tmem + (uint32_t)(b * kTmemCols);
                bool ok = true;
                for (int kb = 0; kb < KB; ++kb, ++kc) {
                    const int s = kc % C::kStages;
                    if (!mbar_wait(&full[s], (kc / C::kStages) & 1)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint64_t ah = sw128_desc(saddr(stage_a(s, 0))), bh = sw128_desc(saddr(stage_b(s, 0)));
                    const uint64_t al = sw128_desc(saddr(stage_a(s, NPROD == 3 ? 1 : 0)));
                    const uint64_t bl = sw128_desc(saddr(stage_b(s, NPROD == 3 ? 1 : 0)));
#pragma unroll
                    for (int kk = 0; kk < kBlockK / 16; ++kk) {
                        const uint64_t o = (uint64_t)(kk * 32 >> 4);
                        mma(acc, ah + o, bh + o, (kb | kk) != 0);
                        if (NPROD == 3) {
                            mma(acc, ah + o, bl + o, 1);
                            mma(acc, al + o, bh + o, 1);
                        }
                    }
                    mma_commit(&empty[s]);
                }
                mma_commit(&accf[b]);  // the tile's products (or those issued before a failure)
                if (!ok) {
                    atomicExch(&fail_s, 1);
                    break;
                }
            }
            // every product issued here has finished before the columns are freed
            mma_commit(&fin);
            if (!mbar_wait(&fin, 0)) atomicExch(&fail_s, 1);
        }
    } else {
        const int q = warp & 3;  // the lane quarter this warp may read
        int i = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++i) {
            const int b = i & 1, u = i >> 1;
            const bool ok = mbar_wait(&accf[b], u & 1);
            tc_fence_after();
            // one decision per warp: the tensor-memory loads below are warp-wide
            if (__any_sync(0xffffffffu, !ok || fail_s)) {
                atomicExch(&fail_s, 1);
                break;
            }
            const int m0 = (t % MT) * kTileM, n0 = ((t / MT) % NT) * kTileN, f = t / (MT * NT);
            const uint32_t acc = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * kTmemCols);
            for (int c = 0; c < kTileN; c += 32) {
                uint32_t v[32];
                tmem_ld32(acc + (uint32_t)c, v);
                epilogue_staged<NPROD, EPI>(a, f, m0 + q * 32, n0 + c, v, stg);
            }
            tc_fence_before();
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(saddr(&acce[b])) : "memory");
        }
    }
    __syncwarp();
    tc_fence_before();
    __syncthreads();
    if (fail_s && threadIdx.x == 0) atomicExch(a.err, 1);
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * kTmemCols)
                     : "memory");
    }
}

// ---- host side ----

typedef CUresult (*EncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encoder() {
    static EncodeTiled fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
    }
    return fn;
}

// 2D BF16 map over rows x P (row-major), boxes of box_rows x 64 elements, 128-byte swizzle
bool make_map(CUtensorMap *m, void *base, int P, long long rows, int box_rows) {
    EncodeTiled enc = encoder();
    if (!enc) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)P, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)P * 2};
    const cuuint32_t box[2] = {(cuuint32_t)kBlockK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

uint16_t bf16_bits(float v) {
    uint32_t u;
    std::memcpy(&u, &v, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);  // round to nearest even (finite values)
    return (uint16_t)(u >> 16);
}

float bf16_value(uint16_t b) {
    const uint32_t u = (uint32_t)b << 16;
    float v;
    std::memcpy(&v, &u, 4);
    return v;
}

template <int NPROD, int EPI>
bool set_smem_attr() {
    return cudaFuncSetAttribute(tc_dst_pass_kernel<NPROD, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)Cfg<NPROD>::kSmem) == cudaSuccess;
}

}  // namespace

struct TcDstPlan {
    int P = 0, fmax = 0, nprod = 1, nsm = 148;
    __nv_bfloat16 *S[2] = {nullptr, nullptr};
    __nv_bfloat16 *X[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [buffer][hi, lo]
    CUtensorMap mS[2], mX[2][2];
};

static void tc_free(TcDstPlan *p) {
    if (!p) return;
    cudaFree(p->S[0]);
    cudaFree(p->S[1]);
    for (auto &b : p->X)
        for (auto *q : b) cudaFree(q);
    delete p;
}

TcDstPlan *tc_create(int P, int fmax, int nprod, const char **why) {
    auto fail = [&](TcDstPlan *p, const char *w) -> TcDstPlan * {
        if (why) *why = w;
        tc_free(p);
        return nullptr;
    };
    if (P != 256 && P != 512 && P != 1024) return fail(nullptr, "tensor-core transforms need nx = ny in {256, 512, 1024}");
    if (nprod != 1 && nprod != 3) return fail(nullptr, "tensor-core transforms take 1 or 3 products");
    if (fmax < 1 || (long long)fmax * P > (1LL << 31)) return fail(nullptr, "bad field count");
    int dev = 0;
    cudaDeviceProp prop{};
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess)
        return fail(nullptr, "no CUDA device");
    if (prop.major != 10 || prop.minor != 0) return fail(nullptr, "tensor-core transforms are built for sm_100a");
    if (!encoder()) return fail(nullptr, "cuTensorMapEncodeTiled is unavailable");
    TcDstPlan *p = new TcDstPlan;
    p->nsm = prop.multiProcessorCount;
    p->P = P;
    p->fmax = fmax;
    p->nprod = nprod;
    const size_t nS = (size_t)P * P, nX = (size_t)fmax * P * P;
    const int parts = nprod == 3 ? 2 : 1;
    for (int k = 0; k < parts; ++k)
        if (cudaMalloc(&p->S[k], nS * 2) != cudaSuccess) return fail(p, "out of device memory");
    for (int b = 0; b < 2; ++b)
        for (int k = 0; k < parts; ++k)
            if (cudaMalloc(&p->X[b][k], nX * 2) != cudaSuccess) return fail(p, "out of device memory");
    // S[k][j] = 2 sin(pi (k+1)(j+1) / P) on the (P-1)^2 block, zero in the padding row and column
    std::vector<uint16_t> hi(nS, 0), lo(nS, 0);
    for (int k = 0; k < P - 1; ++k)
        for (int j = 0; j < P - 1; ++j) {
            const long long t = ((long long)(k + 1) * (j + 1)) % (2LL * P);
            const double s = 2.0 * std::sin(M_PI * (double)t / (double)P);
            const uint16_t h = bf16_bits((float)s);
            hi[(size_t)k * P + j] = h;
            lo[(size_t)k * P + j] = bf16_bits((float)(s - (double)bf16_value(h)));
        }
    if (cudaMemcpy(p->S[0], hi.data(), nS * 2, cudaMemcpyHostToDevice) != cudaSuccess ||
        (parts == 2 && cudaMemcpy(p->S[1], lo.data(), nS * 2, cudaMemcpyHostToDevice) != cudaSuccess))
        return fail(p, "copy of the transform matrix failed");
    for (int k = 0; k < parts; ++k)
        if (!make_map(&p->mS[k], p->S[k], P, P, kTileM)) return fail(p, "tensor map encoding failed");
    for (int b = 0; b < 2; ++b)
        for (int k = 0; k < parts; ++k)
            if (!make_map(&p->mX[b][k], p->X[b][k], P, (long long)fmax * P, kTileN))
                return fail(p, "tensor map encoding failed");
    if (parts == 1) {
        p->mS[1] = p->mS[0];
        for (int b = 0; b < 2; ++b) p->mX[b][1] = p->mX[b][0];
    }
    const bool attrs = nprod == 3 ? (set_smem_attr<3, EPI_SPLIT>() && set_smem_attr<3, EPI_MULT>() &&
                                     set_smem_attr<3, EPI_F64>())
                                  : (set_smem_attr<1, EPI_SPLIT>() && set_smem_attr<1, EPI_MULT>() &&
                                     set_smem_attr<1, EPI_F64>());
    if (!attrs) return fail(p, "shared-memory attribute refused");
    return p;
}

void tc_destroy(TcDstPlan *p) { tc_free(p); }
int tc_P(const TcDstPlan *p) { return p->P; }
int tc_nprod(const TcDstPlan *p) { return p->nprod; }
int tc_fmax(const TcDstPlan *p) { return p->fmax; }
__nv_bfloat16 *tc_in_hi(TcDstPlan *p) { return p->X[0][0]; }
__nv_bfloat16 *tc_in_lo(TcDstPlan *p) { return p->nprod == 3 ? p->X[0][1] : nullptr; }

template <int NPROD>
static void tc_pass(TcDstPlan *p, int src, int epi, int nf, PassArgs a, cudaStream_t st) {
    const CUtensorMap &sh = p->mS[0], &sl = p->mS[1], &xh = p->mX[src][0], &xl = p->mX[src][1];
    const int ntiles = nf * (p->P / kTileM) * (p->P / kTileN);
    const int g = ntiles < p->nsm ? ntiles : p->nsm;
    const size_t sm = Cfg<NPROD>::kSmem;
    if (epi == EPI_SPLIT)
        tc_dst_pass_kernel<NPROD, EPI_SPLIT><<<g, kThreads, sm, st>>>(sh, sl, xh, xl, a, nf);
    else if (epi == EPI_MULT)
        tc_dst_pass_kernel<NPROD, EPI_MULT><<<g, kThreads, sm, st>>>(sh, sl, xh, xl, a, nf);
    else
        tc_dst_pass_kernel<NPROD, EPI_F64><<<g, kThreads, sm, st>>>(sh, sl, xh, xl, a, nf);
}

int tc_solve_tail(TcDstPlan *p, int nf, const float *mult, double *out, long long bs, int ld, TcKeep keep,
                  int *err, cudaStream_t st) {
    if (nf < 1 || nf > p->fmax) return -1;
    PassArgs a{};
    a.P = p->P;
    a.mult = mult;
    a.out = out;
    a.bs = bs;
    a.ld = ld;
    a.keep = keep;
    a.err = err;
    // (y, x) -> (kx, y) -> (ky, kx) [x m] -> (x, ky) -> (y, x)
    const int epis[4] = {EPI_SPLIT, EPI_MULT, EPI_SPLIT, EPI_F64};
    for (int k = 0; k < 4; ++k) {
        const int src = k & 1, dst = src ^ 1;
        a.oh = p->X[dst][0];
        a.ol = p->X[dst][1];
        if (p->nprod == 3)
            tc_pass<3>(p, src, epis[k], nf, a, st);
        else
            tc_pass<1>(p, src, epis[k], nf, a, st);
    }
    return 4;
}
