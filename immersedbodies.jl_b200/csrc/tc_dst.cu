// Dense DST-I passes on the fifth-generation tensor cores (see tc_dst.h).
//
// A tile is D[r][l] for 128 output frequencies r (rows of the half-length
// matrix A, block order) and the TN = P/2 lines l of one block of one field
// (the odd or the even physical indices), over the P/2 slots of the u half (odd
// frequencies) or the v half (even ones).  It accumulates in TN columns of
// tensor memory by tcgen05.mma (M 128, N TN, K 16; BF16 x BF16 -> FP32) from
// K-blocks of 32 elements (64-byte rows, 64-byte swizzle) that TMA brings into
// a ring of shared-memory stages.  One CTA per SM walks the tiles (M-tiles
// fastest, so the CTAs working at once share each line tile through L2); two
// accumulators let the epilogue of one tile run while the products of the next
// accumulate.  Warps: 0 producer (one lane), 1 products (one lane; the whole
// warp allocates and frees the tensor memory), 2..5 epilogue (warp w reads lanes
// 32 (w % 4) ..).  The epilogue turns row r into line r of the next pass: the
// tile's lines are mirror pairs c, TN - 1 - c (physical j, P - j), so a row's u
// and v values for the next pass are sums and differences of its own columns.
//
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

constexpr int kTileM = 128;   // rows of A per tile
// elements per K-block: one swizzle row of 2 kBlockK bytes (32: 64-byte swizzle;
// smaller stages keep more of them in flight than 64 with the 128-byte swizzle)
constexpr int kBlockK = 32;
constexpr int kRowBytes = 2 * kBlockK;
constexpr int kBytesA = kTileM * kBlockK * 2;  // 8 KB
constexpr int kThreads = 192;
constexpr int kStageLd = 33;
constexpr int kStageFloats = 32 * kStageLd;

// EPI_SPLIT_NAT: as EPI_SPLIT, with the next pass's lines in natural order
// (line x - 1 for frequency x, the padding last), so that the last pass's
// columns are contiguous physical positions
enum { EPI_SPLIT = 0, EPI_MULT = 1, EPI_F64 = 2, EPI_SPLIT_NAT = 3 };

template <int NPROD, int P>
struct Cfg {
    static constexpr int kTN = P / 2;                      // lines per tile, the MMA's N
    static constexpr int kBytesB = kTN * kBlockK * 2;
    static constexpr int kParts = NPROD == 3 ? 2 : 1;
    static constexpr int kStageBytes = kParts * (kBytesA + kBytesB);
    static constexpr int kStages = (192 * 1024) / kStageBytes > 8 ? 8 : (192 * 1024) / kStageBytes;
    static constexpr uint32_t kTmemCols = 2 * kTN;        // two accumulators
    static constexpr int kKB = (P / 2) / kBlockK;          // K-blocks per tile
    // the operand ring, four epilogue staging tiles and alignment slack
    static constexpr size_t kSmem = (size_t)kStages * kStageBytes + 4 * kStageFloats * sizeof(float) + 1024;
    // kind::f16 instruction descriptor: BF16 A and B (K-major), FP32 D, M 128, N kTN
    static constexpr uint32_t kIdesc =
        (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kTN >> 3) << 17) | ((uint32_t)(kTileM >> 4) << 24);
};

struct PassArgs {
    __nv_bfloat16 *oh, *ol;   // next pass's lines (EPI_SPLIT, EPI_MULT)
    const float *mult;        // [l][r] multipliers (EPI_MULT)
    double *out;              // result (EPI_F64)
    long long bs;
    int ld;
    TcKeep keep;              // which result elements are stored (EPI_F64)
    int *err;
};

// The result selection as bounds on 0-based physical (x, y): stored when
// (x in [x0, x1] and y in [y0, y1]) or y in {ya, yb} or x in {xa, xb}
struct Keep {
    int x0, x1, y0, y1, ya, yb, xa, xb;
};
__device__ __forceinline__ Keep keep_bounds(const TcKeep &k) {
    if (k.mode == TC_KEEP_WINDOW)
        return Keep{__ldg(k.win) - 2, __ldg(k.win + 1), __ldg(k.win + 2) - 2, __ldg(k.win + 3), -1, -1, -1, -1};
    if (k.mode == TC_KEEP_LINES) return Keep{0, -1, 0, -1, k.lines[0], k.lines[1], k.lines[2], k.lines[3]};
    return Keep{0, 1 << 30, 0, 1 << 30, -1, -1, -1, -1};
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

// Shared-memory operand descriptor: K-major, swizzle of one K-block row (64 or
// 128 bytes), 8-row groups 8 rows apart.
__device__ __forceinline__ uint64_t sw_desc(uint32_t a) {
    uint64_t d = (uint64_t)((a & 0x3FFFFu) >> 4);
    d |= (uint64_t)1 << 16;                       // leading offset (unused by swizzled K-major layouts)
    d |= (uint64_t)((8 * kRowBytes) >> 4) << 32;  // stride between 8-row groups
    d |= (uint64_t)1 << 46;                       // descriptor version
    d |= (uint64_t)(kRowBytes == 128 ? 2 : 4) << 61;  // 128-byte or 64-byte swizzle
    return d;
}

__device__ __forceinline__ void mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
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


// Rows row0 .. row0 + 31 (one warp, lane = row) of a 32 x 32 block staged in
// stg (32 x 33 floats, conflict-free both ways) to the next pass's lines at
// slots pos0 .. pos0 + 31, as BF16 parts in coalesced 64-byte row segments;
// row r becomes line r, or (NAT) the natural-order line of its frequency.
template <int NPROD, int P, bool NAT>
__device__ __forceinline__ void store_staged(const PassArgs &a, int f, int row0, int pos0, const float *stg) {
    const int lane = threadIdx.x & 31, q = lane & 3;
#pragma unroll
    for (int it = 0; it < 4; ++it) {
        const int r = it * 8 + (lane >> 2);
        __align__(16) __nv_bfloat16 h[8];
        __align__(16) __nv_bfloat16 l[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) tc_split(stg[r * kStageLd + 8 * q + i], h[i], l[i]);
        int line = row0 + r;
        if (NAT) {
            const int k = tc_blk(line, P);
            line = k == 0 ? P - 1 : k - 1;
        }
        const size_t off = ((size_t)f * P + line) * P + pos0 + 8 * q;
        *reinterpret_cast<uint4 *>(a.oh + off) = *reinterpret_cast<const uint4 *>(h);
        if (NPROD == 3) *reinterpret_cast<uint4 *>(a.ol + off) = *reinterpret_cast<const uint4 *>(l);
    }
}

// The epilogue of one tile for one warp: rows row0 + lane of accumulator acc
// (this warp's lane quarter, the buffer's first column), lines of block nt.
template <int NPROD, int EPI, int P>
__device__ __forceinline__ void epilogue(const PassArgs &a, int f, int row0, int nt, uint32_t acc, float *stg) {
    using C = Cfg<NPROD, P>;
    constexpr int TN = C::kTN, NCH = TN / 32;
    const int lane = threadIdx.x & 31, row = row0 + lane;
    if constexpr (EPI == EPI_F64) {
        // row flags of the warp's 32 rows (bit rr: row row0 + rr), column flags per lane
        const Keep kb = keep_bounds(a.keep);
        const int y = tc_blk(row, P) - 1;  // this thread's physical row (-1: padding)
        const unsigned live = __ballot_sync(0xffffffffu, y >= 0);
        const unsigned in_rows = __ballot_sync(0xffffffffu, y >= 0 && y >= kb.y0 && y <= kb.y1);
        const unsigned on_rows = __ballot_sync(0xffffffffu, y >= 0 && (y == kb.ya || y == kb.yb));
        double *o = a.out + (long long)f * a.bs;
        for (int k = 0; k < NCH; ++k) {
            // this lane's physical column: the lines arrive in natural order
            const int x = nt * TN + 32 * k + lane < P - 1 ? nt * TN + 32 * k + lane : -1;
            const bool cin = x >= 0 && x >= kb.x0 && x <= kb.x1, con = x >= 0 && (x == kb.xa || x == kb.xb);
            // rows with anything to store in this chunk
            const unsigned rows =
                (__any_sync(0xffffffffu, cin) ? in_rows : 0u) | on_rows | (__any_sync(0xffffffffu, con) ? live : 0u);
            if (rows == 0u) continue;
            uint32_t v[32];
            tmem_ld32(acc + (uint32_t)(32 * k), v);
#pragma unroll
            for (int i = 0; i < 32; ++i) stg[lane * kStageLd + i] = __uint_as_float(v[i]);
            __syncwarp();
            const unsigned mine = (cin ? in_rows : 0u) | on_rows | (con ? live : 0u);  // rows this lane stores
            for (unsigned rest = rows; rest;) {
                const int rr = __ffs(rest) - 1;
                rest &= rest - 1;
                const int yy = __shfl_sync(0xffffffffu, y, rr);
                if (x >= 0 && ((mine >> rr) & 1u)) o[x + a.ld * yy] = (double)stg[rr * kStageLd + lane];
            }
            __syncwarp();
        }
    } else {
        for (int k = 0; k < NCH / 2; ++k) {
            uint32_t va[32], vb[32];
            tmem_ld32(acc + (uint32_t)(32 * k), va);
            tmem_ld32(acc + (uint32_t)(32 * (NCH - 1 - k)), vb);
            float x[32], y[32];
#pragma unroll
            for (int i = 0; i < 32; ++i) {
                x[i] = __uint_as_float(va[i]);
                y[i] = __uint_as_float(vb[i]);
            }
            if (EPI == EPI_MULT) {
                // column l of the table holds the rows' multipliers contiguously
                const float *ma = a.mult + (size_t)(nt * TN + 32 * k) * P + row;
                const float *mb = a.mult + (size_t)(nt * TN + 32 * (NCH - 1 - k)) * P + row;
#pragma unroll
                for (int i = 0; i < 32; ++i) {
                    x[i] *= __ldg(ma + (size_t)i * P);
                    y[i] *= __ldg(mb + (size_t)i * P);
                }
            }
            // column 32k + i pairs with TN - 1 - (32k + i) = 32 (NCH - 1 - k) + 31 - i
            const int slot = nt * (TN / 2) + 32 * k;
#pragma unroll
            for (int i = 0; i < 32; ++i) stg[lane * kStageLd + i] = x[i] + y[31 - i];
            __syncwarp();
            store_staged<NPROD, P, EPI == EPI_SPLIT_NAT>(a, f, row0, slot, stg);
            __syncwarp();
#pragma unroll
            for (int i = 0; i < 32; ++i) stg[lane * kStageLd + i] = x[i] - y[31 - i];
            __syncwarp();
            store_staged<NPROD, P, EPI == EPI_SPLIT_NAT>(a, f, row0, P / 2 + slot, stg);
            __syncwarp();
        }
    }
}

template <int NPROD, int EPI, int P>
__global__ void __launch_bounds__(kThreads, 1)
    tc_dst_pass_kernel(const __grid_constant__ CUtensorMap tAh, const __grid_constant__ CUtensorMap tAl,
                       const __grid_constant__ CUtensorMap tXh, const __grid_constant__ CUtensorMap tXl, PassArgs a,
                       int nf) {
    using C = Cfg<NPROD, P>;
    constexpr int TN = C::kTN, MT = P / kTileM, NT = 2, KB = C::kKB;
    extern __shared__ uint8_t smem_raw[];
    __shared__ uint64_t full[C::kStages], empty[C::kStages], accf[2], acce[2], fin;
    __shared__ uint32_t tmem_s;
    __shared__ int fail_s;
    // the swizzle atoms (8 rows of one K-block) must start on 1024-byte boundaries of the shared window
    uint8_t *smem = smem_raw + ((1024u - (saddr(smem_raw) & 1023u)) & 1023u);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntiles = nf * MT * NT;
    // epilogue warp w (2..5) stages through its own tile after the operand ring
    float *stg = reinterpret_cast<float *>(smem + (size_t)C::kStages * C::kStageBytes) +
                 (warp >= 2 ? (warp - 2) * kStageFloats : 0);

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
                     "r"(C::kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_s;

    auto stage_a = [&](int s, int part) { return smem + (size_t)s * C::kStageBytes + part * kBytesA; };
    auto stage_b = [&](int s, int part) {
        return smem + (size_t)s * C::kStageBytes + C::kParts * kBytesA + part * C::kBytesB;
    };

    if (warp == 0) {
        if (lane == 0) {
            int kc = 0;  // K-blocks loaded so far (the ring position)
            for (int t = blockIdx.x; t < ntiles && !fail_s; t += gridDim.x) {
                const int m0 = (t % MT) * kTileM, n0 = ((t / MT) % NT) * TN, f = t / (MT * NT);
                const int koff = m0 < P / 2 ? 0 : P / 2;  // odd frequencies read u, even ones v
                for (int kb = 0; kb < KB; ++kb, ++kc) {
                    const int s = kc % C::kStages;
                    if (kc >= C::kStages && !mbar_wait(&empty[s], ((kc / C::kStages) - 1) & 1)) {
                        atomicExch(&fail_s, 1);
                        break;
                    }
                    mbar_expect_tx(&full[s], C::kStageBytes);
                    tma_load(stage_a(s, 0), &tAh, &full[s], kb * kBlockK, m0);
                    tma_load(stage_b(s, 0), &tXh, &full[s], koff + kb * kBlockK, f * P + n0);
                    if (NPROD == 3) {
                        tma_load(stage_a(s, 1), &tAl, &full[s], kb * kBlockK, m0);
                        tma_load(stage_b(s, 1), &tXl, &full[s], koff + kb * kBlockK, f * P + n0);
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
                const uint32_t acc = tmem + (uint32_t)(b * TN);
                bool ok = true;
                for (int kb = 0; kb < KB; ++kb, ++kc) {
                    const int s = kc % C::kStages;
                    if (!mbar_wait(&full[s], (kc / C::kStages) & 1)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint64_t ah = sw_desc(saddr(stage_a(s, 0))), bh = sw_desc(saddr(stage_b(s, 0)));
                    const uint64_t al = sw_desc(saddr(stage_a(s, NPROD == 3 ? 1 : 0)));
                    const uint64_t bl = sw_desc(saddr(stage_b(s, NPROD == 3 ? 1 : 0)));
#pragma unroll
                    for (int kk = 0; kk < kBlockK / 16; ++kk) {
                        const uint64_t o = (uint64_t)(kk * 32 >> 4);  // 16 elements = 32 B along the swizzled row
                        mma(acc, ah + o, bh + o, C::kIdesc, (kb | kk) != 0);
                        if (NPROD == 3) {
                            mma(acc, ah + o, bl + o, C::kIdesc, 1);
                            mma(acc, al + o, bh + o, C::kIdesc, 1);
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
            const int m0 = (t % MT) * kTileM, nt = (t / MT) % NT, f = t / (MT * NT);
            const uint32_t acc = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * TN);
            epilogue<NPROD, EPI, P>(a, f, m0 + q * 32, nt, acc, stg);
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
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(C::kTmemCols)
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

// 2D BF16 map over rows x cols (row-major), boxes of box_rows x kBlockK elements, swizzled like the descriptors
bool make_map(CUtensorMap *m, void *base, int cols, long long rows, int box_rows) {
    EncodeTiled enc = encoder();
    if (!enc) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
    const cuuint32_t box[2] = {(cuuint32_t)kBlockK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               kRowBytes == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
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

template <int NPROD, int P>
bool set_smem_attrs() {
    const int sm = (int)Cfg<NPROD, P>::kSmem;
    return cudaFuncSetAttribute(tc_dst_pass_kernel<NPROD, EPI_SPLIT, P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                sm) == cudaSuccess &&
           cudaFuncSetAttribute(tc_dst_pass_kernel<NPROD, EPI_MULT, P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                sm) == cudaSuccess &&
           cudaFuncSetAttribute(tc_dst_pass_kernel<NPROD, EPI_F64, P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                sm) == cudaSuccess &&
           cudaFuncSetAttribute(tc_dst_pass_kernel<NPROD, EPI_SPLIT_NAT, P>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, sm) == cudaSuccess;
}

}  // namespace

struct TcDstPlan {
    int P = 0, fmax = 0, nprod = 1, nsm = 148;
    __nv_bfloat16 *A[2] = {nullptr, nullptr};                            // hi, lo: P x P/2
    __nv_bfloat16 *X[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [buffer][hi, lo]
    CUtensorMap mA[2], mX[2][2];
};

static void tc_free(TcDstPlan *p) {
    if (!p) return;
    cudaFree(p->A[0]);
    cudaFree(p->A[1]);
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
    if (P != 256 && P != 512) return fail(nullptr, "tensor-core transforms need nx = ny in {256, 512}");
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
    const int H = P / 2;
    const size_t nA = (size_t)P * H, nX = (size_t)fmax * P * P;
    const int parts = nprod == 3 ? 2 : 1;
    for (int k = 0; k < parts; ++k)
        if (cudaMalloc(&p->A[k], nA * 2) != cudaSuccess) return fail(p, "out of device memory");
    for (int b = 0; b < 2; ++b)
        for (int k = 0; k < parts; ++k)
            if (cudaMalloc(&p->X[b][k], nX * 2) != cudaSuccess) return fail(p, "out of device memory");
    // A[r][s] = 2 sin(pi k j / P), k = tc_blk(r) (the frequency of row r) and j =
    // tc_uvj(s) (the pair of slot s); zero for the padding row and for even k at
    // j = P/2, whose v slot holds no pair
    std::vector<uint16_t> hi(nA, 0), lo(nA, 0);
    for (int r = 0; r < P; ++r) {
        const int k = tc_blk(r, P);
        if (k == 0) continue;
        for (int s = 0; s < H; ++s) {
            const int j = tc_uvj(s, P);
            if (k % 2 == 0 && j == H) continue;
            const long long t = ((long long)k * j) % (2LL * P);
            const double v = 2.0 * std::sin(M_PI * (double)t / (double)P);
            const uint16_t h = bf16_bits((float)v);
            hi[(size_t)r * H + s] = h;
            lo[(size_t)r * H + s] = bf16_bits((float)(v - (double)bf16_value(h)));
        }
    }
    if (cudaMemcpy(p->A[0], hi.data(), nA * 2, cudaMemcpyHostToDevice) != cudaSuccess ||
        (parts == 2 && cudaMemcpy(p->A[1], lo.data(), nA * 2, cudaMemcpyHostToDevice) != cudaSuccess))
        return fail(p, "copy of the transform matrix failed");
    for (int k = 0; k < parts; ++k)
        if (!make_map(&p->mA[k], p->A[k], H, P, kTileM)) return fail(p, "tensor map encoding failed");
    for (int b = 0; b < 2; ++b)
        for (int k = 0; k < parts; ++k)
            if (!make_map(&p->mX[b][k], p->X[b][k], P, (long long)fmax * P, H)) return fail(p, "tensor map encoding failed");
    if (parts == 1) {
        p->mA[1] = p->mA[0];
        for (int b = 0; b < 2; ++b) p->mX[b][1] = p->mX[b][0];
    }
    bool attrs;
    if (P == 512)
        attrs = nprod == 3 ? set_smem_attrs<3, 512>() : set_smem_attrs<1, 512>();
    else
        attrs = nprod == 3 ? set_smem_attrs<3, 256>() : set_smem_attrs<1, 256>();
    if (!attrs) return fail(p, "shared-memory attribute refused");
    return p;
}

void tc_destroy(TcDstPlan *p) { tc_free(p); }
int tc_P(const TcDstPlan *p) { return p->P; }
int tc_nprod(const TcDstPlan *p) { return p->nprod; }
int tc_fmax(const TcDstPlan *p) { return p->fmax; }
__nv_bfloat16 *tc_in_hi(TcDstPlan *p) { return p->X[0][0]; }
__nv_bfloat16 *tc_in_lo(TcDstPlan *p) { return p->nprod == 3 ? p->X[0][1] : nullptr; }

template <int NPROD, int P>
static void tc_pass(TcDstPlan *p, int src, int epi, int nf, PassArgs a, cudaStream_t st) {
    const CUtensorMap &ah = p->mA[0], &al = p->mA[1], &xh = p->mX[src][0], &xl = p->mX[src][1];
    const int ntiles = nf * (P / kTileM) * 2;
    const int g = ntiles < p->nsm ? ntiles : p->nsm;
    const size_t sm = Cfg<NPROD, P>::kSmem;
    if (epi == EPI_SPLIT)
        tc_dst_pass_kernel<NPROD, EPI_SPLIT, P><<<g, kThreads, sm, st>>>(ah, al, xh, xl, a, nf);
    else if (epi == EPI_MULT)
        tc_dst_pass_kernel<NPROD, EPI_MULT, P><<<g, kThreads, sm, st>>>(ah, al, xh, xl, a, nf);
    else if (epi == EPI_SPLIT_NAT)
        tc_dst_pass_kernel<NPROD, EPI_SPLIT_NAT, P><<<g, kThreads, sm, st>>>(ah, al, xh, xl, a, nf);
    else
        tc_dst_pass_kernel<NPROD, EPI_F64, P><<<g, kThreads, sm, st>>>(ah, al, xh, xl, a, nf);
}

int tc_solve_tail(TcDstPlan *p, int nf, const float *mult, double *out, long long bs, int ld, TcKeep keep,
                  int *err, cudaStream_t st) {
    if (nf < 1 || nf > p->fmax) return -1;
    PassArgs a{};
    a.mult = mult;
    a.out = out;
    a.bs = bs;
    a.ld = ld;
    a.keep = keep;
    a.err = err;
    // (y, x) -> (kx, y) -> (ky, kx) [x m] -> (x, ky) -> (y, x)
    const int epis[4] = {EPI_SPLIT, EPI_MULT, EPI_SPLIT_NAT, EPI_F64};
    for (int k = 0; k < 4; ++k) {
        const int src = k & 1, dst = src ^ 1;
        a.oh = p->X[dst][0];
        a.ol = p->X[dst][1];
        if (p->P == 512) {
            if (p->nprod == 3)
                tc_pass<3, 512>(p, src, epis[k], nf, a, st);
            else
                tc_pass<1, 512>(p, src, epis[k], nf, a, st);
        } else {
            if (p->nprod == 3)
                tc_pass<3, 256>(p, src, epis[k], nf, a, st);
            else
                tc_pass<1, 256>(p, src, epis[k], nf, a, st);
        }
    }
    return 4;
}
