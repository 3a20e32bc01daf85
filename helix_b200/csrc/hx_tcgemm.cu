// GEMM on the 5th-generation tensor cores: C = sum_p A_p B_p^T (one to three
// operand pairs in one accumulator) with A_p [M x K] and B_p [N x K], both
// row-major (K contiguous), BF16 (kind::f16) or TF32 (kind::tf32) operands and
// FP32 accumulation in tensor memory.  Used by the learned closure's MLP
// (hx_mlp.cu; BF16, one pair, fused bias / GELU epilogues) and by the dense-H
// stage (hx_ctx.cu; TF32, the three pairs of a split product, plain store).
// No counterpart in the reference.
//
// One CTA of four warps computes a 128 x BN tile of C (BN = 256 when N >=
// 256, else 128; 1-D grid, N tiles fastest):
//  * warp 0 allocates BN tensor-memory columns (the 128 x BN FP32
//    accumulator, one lane per row) and its lane 0 streams the K blocks of
//    every pair (128 bytes of each of the 128 rows of A and BN rows of B: 64
//    BF16 or 32 TF32) into a 192 KB shared-memory ring (6 stages at BN = 128,
//    4 at 256) with TMA tensor loads in the 128-byte swizzled layout;
//  * lane 0 of warp 1 issues tcgen05.mma (M = 128, N = BN, 32 bytes of K per
//    instruction: K = 16 BF16 or 8 TF32; four per K block, the shared-memory
//    descriptor advanced by 32 bytes inside the swizzle atom) and returns each
//    stage to the producer with tcgen05.commit on that stage's mbarrier;
//  * after the last block a commit signals the accumulator complete; every
//    warp reads its 32 lanes with tcgen05.ld (16 columns at a time) into a
//    padded shared-memory tile over the drained ring, and the CTA then stores
//    row after row of C with consecutive threads on consecutive columns,
//    applying the epilogue (bias + GELU keeping the pre-activation, bias,
//    plain store, or GELU backward).
// Out-of-range rows, columns and K are zero-filled by the tensor loads and
// masked at the stores.  Every mbarrier wait is bounded: a wait that runs
// out sets the error word, the kernel still waits (bounded) for its copies
// and MMAs in flight, frees its tensor memory and returns.

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdint>

#include "hx_internal.h"

namespace hx {

namespace {

constexpr int kBM = 128;
constexpr uint32_t kRowBytes = 128;  // one K block: 128 bytes of every row (64 BF16 or 32 TF32)
constexpr uint32_t kPoll = 1u << 22;

// Tile of BN = 128 or 256 columns: stage bytes (A then B), ring depth and
// dynamic shared memory (ring + 1024-byte alignment + barriers).
template <int BN>
struct TileCfg {
    static constexpr uint32_t kABytes = kBM * kRowBytes;
    static constexpr uint32_t kStageBytes = kABytes + BN * kRowBytes;
    static constexpr int kStages = BN == 128 ? 6 : 4;  // a 192 KB ring either way
    static constexpr uint32_t kRing = kStages * kStageBytes;
    static constexpr uint32_t kSmem = kRing + 1024 + 256;
    static_assert(kBM * (BN + 1) * 4 <= kRing, "the epilogue tile reuses the ring");
    static_assert(kSmem <= 227 * 1024, "shared memory per CTA");
};

// tcgen05.mma instruction descriptor: FP32 accumulator, A and B both BF16
// (format 1) or both TF32 (format 2), both K-major, M = 128, N = BN.
__host__ __device__ constexpr uint32_t idesc_of(uint32_t fmt, int bn)
{
    return (1u << 4) | (fmt << 7) | (fmt << 10) | (uint32_t(bn >> 3) << 17) | (uint32_t(kBM >> 4) << 24);
}

// Tensor maps of up to three operand pairs; the kernel accumulates the sum of
// their products A_p B_p^T (the terms of a split-precision product).
struct TcMaps {
    CUtensorMap a[3];
    CUtensorMap b[3];
};

__device__ __forceinline__ uint32_t saddr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// Shared-memory matrix descriptor of a K-major tile in the 128-byte swizzled
// layout: rows of 128 bytes, 8-row atoms 1024 bytes apart (stride byte
// offset), tile base 1024-byte aligned.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr)
{
    uint64_t d = static_cast<uint64_t>((addr & 0x3FFFFu) >> 4);  // start address
    d |= static_cast<uint64_t>(1) << 16;                         // leading byte offset (unused when swizzled)
    d |= static_cast<uint64_t>(1024 >> 4) << 32;                 // stride byte offset
    d |= static_cast<uint64_t>(1) << 46;                         // descriptor version of this architecture
    d |= static_cast<uint64_t>(2) << 61;                         // 128-byte swizzle
    return d;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    for (uint32_t i = 0; i < kPoll; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
            "r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tc_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ float gelu_f(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }

__device__ __forceinline__ float gelu_grad_f(float z)
{
    const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
    return cdf + z * pdf;
}

template <bool TF32, int BN>
__global__ void __launch_bounds__(128, 1)
    tc_gemm_kernel(const __grid_constant__ TcMaps maps, int M, int N, int K, int npairs, TcGemmOut o, int* err)
{
    using Cfg = TileCfg<BN>;
    constexpr int kStages = Cfg::kStages;
    constexpr uint32_t kStageBytes = Cfg::kStageBytes;
    constexpr int kBK = TF32 ? 32 : 64;  // K elements per 128-byte row
    constexpr uint32_t kIdesc = idesc_of(TF32 ? 2u : 1u, BN);
    extern __shared__ unsigned char smem_raw[];
    const uint32_t raw = saddr(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;  // swizzled tiles need 1024-byte alignment
    const uint32_t bars = base + Cfg::kRing;
    auto full_bar = [&](int s) { return bars + 8u * s; };
    auto empty_bar = [&](int s) { return bars + 8u * (kStages + s); };
    const uint32_t done_bar = bars + 8u * (2 * kStages);
    const uint32_t tslot = done_bar + 8u;
    const uint32_t cslot = tslot + 4u;  // K blocks the MMA thread consumed

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // 1-D grid, N tiles fastest: the CTAs that share a row block of A run together and read it once from HBM
    const int ntn = (N + BN - 1) / BN;
    const int m0 = static_cast<int>(blockIdx.x / ntn) * kBM, n0 = static_cast<int>(blockIdx.x % ntn) * BN;
    const int nkp = (K + kBK - 1) / kBK;  // K blocks of one operand pair
    const int nk = nkp * npairs;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(full_bar(s), 1);
            mbar_init(empty_bar(s), 1);
        }
        mbar_init(done_bar, 1);
        asm volatile("st.shared.u32 [%0], %1;" ::"r"(cslot), "r"(0) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tslot), "r"(BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    uint32_t tmem;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(tmem) : "r"(tslot) : "memory");

    // Roles are taken by whole warps: one lane issues, the other lanes of the
    // warp wait at __syncwarp (not in a polling loop that would compete with
    // the issuing lane for the warp's issue slots).
    int issued = 0;
    if (warp == 0) {
        if (lane == 0) {
            // ---- producer: TMA loads of the K blocks
            for (int kb = 0; kb < nk; ++kb) {
                const int s = kb % kStages, r = kb / kStages;
                if (r >= 1 && !mbar_wait(empty_bar(s), (r - 1) & 1)) {
                    atomicExch(err, 1);
                    break;
                }
                const uint32_t a = base + s * kStageBytes, b = a + Cfg::kABytes;
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(full_bar(s)),
                             "r"(kStageBytes)
                             : "memory");
                const int p = kb / nkp, x = (kb - p * nkp) * kBK;
                tma_load_2d(a, &maps.a[p], x, m0, full_bar(s));
                tma_load_2d(b, &maps.b[p], x, n0, full_bar(s));
                issued = kb + 1;
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            // ---- MMA issue
            int kb = 0;
            for (; kb < nk; ++kb) {
                const int s = kb % kStages, r = kb / kStages;
                if (!mbar_wait(full_bar(s), r & 1)) {
                    atomicExch(err, 1);
                    break;
                }
                tc_fence_after();
                const uint32_t a = base + s * kStageBytes, b = a + Cfg::kABytes;
#pragma unroll
                for (int k = 0; k < 4; ++k) {  // 32 bytes of K per instruction (16 BF16 or 8 TF32)
                    const uint64_t da = sw128_desc(a + 32u * k), db = sw128_desc(b + 32u * k);
                    const uint32_t accumulate = (kb > 0 || k > 0) ? 1u : 0u;
                    if constexpr (TF32)
                        asm volatile(
                            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                            "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate)
                            : "memory");
                    else
                        asm volatile(
                            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                            "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate)
                            : "memory");
                }
                tc_commit(empty_bar(s));  // the stage is free once these MMAs have read it
            }
            asm volatile("st.shared.u32 [%0], %1;" ::"r"(cslot), "r"(kb) : "memory");
            tc_commit(done_bar);  // every MMA issued above has completed
        }
        __syncwarp();
    }

    // ---- epilogue: the accumulator goes through shared memory (the ring is
    // free once every MMA has completed and every copy has landed) so that
    // each row of C is stored by consecutive threads
    const bool done = mbar_wait(done_bar, 0);
    if (!done && threadIdx.x == 0) atomicExch(err, 1);
    if (warp == 0 && lane == 0) {
        int consumed;
        asm volatile("ld.shared.u32 %0, [%1];" : "=r"(consumed) : "r"(cslot) : "memory");
        for (int kb = consumed; kb < issued; ++kb) mbar_wait(full_bar(kb % kStages), (kb / kStages) & 1);
    }
    tc_fence_after();
    __syncthreads();
    float* stile = reinterpret_cast<float*>(smem_raw + (base - raw));  // [128][BN + 1]
    constexpr int kLd = BN + 1;
    const int trow = warp * 32 + lane;
    for (int c0 = 0; c0 < BN; c0 += 16) {
        uint32_t v[16];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
            "%14, %15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c0)));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int jj = 0; jj < 16; ++jj) stile[trow * kLd + c0 + jj] = __uint_as_float(v[jj]);
    }
    __syncthreads();
    if (done) {
        for (int cc = static_cast<int>(threadIdx.x); cc < BN; cc += 128) {
            const int col = n0 + cc;
            if (col >= N) break;
            const float bias = (o.kind == kTcEpiBiasGelu || o.kind == kTcEpiBias) ? o.bias[col] : 0.0f;
            for (int rr = 0; rr < kBM; ++rr) {
                const int row = m0 + rr;
                if (row >= M) break;
                const float val = stile[rr * kLd + cc];
                const long long off = static_cast<long long>(row) * o.ldo + col;
                if (o.kind == kTcEpiBiasGelu) {
                    const float z = val + bias;
                    o.outf[off] = z;
                    static_cast<__nv_bfloat16*>(o.outh)[off] = __float2bfloat16(gelu_f(z));
                } else if (o.kind == kTcEpiBias) {
                    o.outf[off] = val + bias;
                } else if (o.kind == kTcEpiStore) {
                    o.outf[off] = val;
                } else {
                    const float g = val * gelu_grad_f(o.aux[off]);
                    static_cast<__nv_bfloat16*>(o.outh)[off] = __float2bfloat16(g);
                    if (o.outf) o.outf[off] = g;
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN) : "memory");
    }
}

// FP32 value rounded to TF32 (10 mantissa bits, to nearest, ties away from zero).
__device__ __forceinline__ float tf32_round(float v)
{
    return __uint_as_float((__float_as_uint(v) + 0x1000u) & 0xFFFFE000u);
}

// Split-product GEMM with the split of A done in shared memory:
// C = A_hi B_hi^T + A_hi B_lo^T + A_lo B_hi^T, A [M x K] FP32, B_hi / B_lo
// [N x K] exact TF32 values, FP32 accumulation (the dense-H product).
// Persistent: one CTA per SM walks the 128 x 256 tiles (N tiles fastest), with
// two accumulators in tensor memory (2 x 256 columns) so that the epilogue of
// one tile overlaps the MMAs of the next.  Each ring stage holds one K block
// of A (rounded in place to A_hi), of A_lo, of B_hi and of B_lo
// (16 + 16 + 32 + 32 KB); two stages fill 192 KB.
//  * warp 0 lane 0: TMA loads of A, B_hi, B_lo for every K block of every tile;
//  * warps 2-3: once a stage has landed, round A to A_hi in place and write
//    A_lo beside it (an elementwise map at equal offsets, so the swizzled
//    layout carries over), fence the writes to the tensor cores' proxy and
//    arrive on the stage's conversion barrier;
//  * warp 1 lane 0: twelve tcgen05.mma per stage (three products x four K
//    steps of 8; the small terms first), tcgen05.commit frees the stage, and
//    after a tile's last K block a commit marks its accumulator full;
//  * warps 4-7: each reads its 32 lanes (rows) of a full accumulator 32
//    columns at a time, transposes them through 4 KB of shared memory and
//    stores whole 128-byte row pieces, then frees the accumulator.
// A is read from HBM once and never written back in split form.  Every wait
// is bounded; a wait that runs out sets the error word and its role stops.
constexpr int kSplitBN = 256, kSplitStages = 2;
constexpr uint32_t kSplitA = kBM * kRowBytes, kSplitB = kSplitBN * kRowBytes;
constexpr uint32_t kSplitStage = 2 * kSplitA + 2 * kSplitB;
constexpr uint32_t kSplitRing = kSplitStages * kSplitStage;
constexpr int kEpiWarps = 4;
constexpr uint32_t kEpiBuf = 32 * 33 * 4;  // one epilogue warp's 32 x 32 block, padded rows
constexpr uint32_t kSplitSmem = kSplitRing + kEpiWarps * kEpiBuf + 1024 + 256;
static_assert(kSplitSmem <= 227 * 1024, "shared memory per CTA");
constexpr int kConvThreads = 64;
constexpr int kSplitThreads = 256;

__global__ void __launch_bounds__(kSplitThreads, 1)
    tc_split_gemm_kernel(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_bh,
                         const __grid_constant__ CUtensorMap map_bl, int M, int N, int K, float* out, int ldo,
                         int* err)
{
    constexpr int kBK = 32;  // TF32 per 128-byte row
    constexpr uint32_t kIdesc = idesc_of(2u, kSplitBN);
    extern __shared__ unsigned char smem_raw[];
    const uint32_t raw = saddr(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    unsigned char* gbase = smem_raw + (base - raw);  // generic pointer to the ring
    const uint32_t bars = base + kSplitRing + kEpiWarps * kEpiBuf;
    auto full_bar = [&](int s) { return bars + 8u * s; };
    auto conv_bar = [&](int s) { return bars + 8u * (2 + s); };
    auto empty_bar = [&](int s) { return bars + 8u * (4 + s); };
    auto accf_bar = [&](int x) { return bars + 8u * (6 + x); };
    auto acce_bar = [&](int x) { return bars + 8u * (8 + x); };
    const uint32_t fin_bar = bars + 8u * 10;
    const uint32_t tslot = bars + 8u * 11;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntn = (N + kSplitBN - 1) / kSplitBN;
    const int tiles = ntn * ((M + kBM - 1) / kBM);
    const int mine = tiles > static_cast<int>(blockIdx.x)
                         ? (tiles - 1 - static_cast<int>(blockIdx.x)) / static_cast<int>(gridDim.x) + 1
                         : 0;
    const int nk = (K + kBK - 1) / kBK;
    auto tile_of = [&](int i, int& m0, int& n0) {
        const int t = static_cast<int>(blockIdx.x) + i * static_cast<int>(gridDim.x);
        m0 = (t / ntn) * kBM;
        n0 = (t % ntn) * kSplitBN;
    };

    if (threadIdx.x == 0) {
        for (int s = 0; s < kSplitStages; ++s) {
            mbar_init(full_bar(s), 1);
            mbar_init(conv_bar(s), kConvThreads);
            mbar_init(empty_bar(s), 1);
        }
        for (int x = 0; x < 2; ++x) {
            mbar_init(accf_bar(x), 1);
            mbar_init(acce_bar(x), kEpiWarps);
        }
        mbar_init(fin_bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tslot),
                     "r"(2 * kSplitBN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    uint32_t tmem;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(tmem) : "r"(tslot) : "memory");

    if (warp == 0) {
        if (lane == 0) {
            // ---- producer
            long long g = 0;
            bool ok = true;
            for (int i = 0; i < mine && ok; ++i) {
                int m0, n0;
                tile_of(i, m0, n0);
                for (int kb = 0; kb < nk; ++kb, ++g) {
                    const int s = static_cast<int>(g & 1);
                    const long long r = g >> 1;
                    if (r >= 1 && !mbar_wait(empty_bar(s), static_cast<uint32_t>((r - 1) & 1))) {
                        atomicExch(err, 1);
                        ok = false;
                        break;
                    }
                    const uint32_t a = base + s * kSplitStage;
                    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(full_bar(s)),
                                 "r"(kSplitA + 2 * kSplitB)
                                 : "memory");
                    const int x = kb * kBK;
                    tma_load_2d(a, &map_a, x, m0, full_bar(s));
                    tma_load_2d(a + 2 * kSplitA, &map_bh, x, n0, full_bar(s));
                    tma_load_2d(a + 2 * kSplitA + kSplitB, &map_bl, x, n0, full_bar(s));
                }
            }
            // at most the last two issued copies can still be in flight: wait for them (bounded)
            for (long long h = g > 2 ? g - 2 : 0; h < g; ++h)
                mbar_wait(full_bar(static_cast<int>(h & 1)), static_cast<uint32_t>((h >> 1) & 1));
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            // ---- MMA issue
            long long g = 0;
            bool ok = true;
            for (int i = 0; i < mine && ok; ++i) {
                const int x = i & 1;
                if (i >= 2 && !mbar_wait(acce_bar(x), static_cast<uint32_t>(((i >> 1) - 1) & 1))) {
                    atomicExch(err, 1);
                    break;
                }
                tc_fence_after();
                const uint32_t tacc = tmem + static_cast<uint32_t>(x * kSplitBN);
                for (int kb = 0; kb < nk; ++kb, ++g) {
                    const int s = static_cast<int>(g & 1);
                    if (!mbar_wait(conv_bar(s), static_cast<uint32_t>((g >> 1) & 1))) {
                        atomicExch(err, 1);
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t ah = base + s * kSplitStage, al = ah + kSplitA, bh = ah + 2 * kSplitA,
                                   bl = bh + kSplitB;
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const uint64_t dah = sw128_desc(ah + 32u * k), dal = sw128_desc(al + 32u * k),
                                       dbh = sw128_desc(bh + 32u * k), dbl = sw128_desc(bl + 32u * k);
                        const uint32_t acc = (kb == 0 && k == 0) ? 0u : 1u;
                        asm volatile(
                            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tacc),
                            "l"(dal), "l"(dbh), "r"(kIdesc), "r"(acc)
                            : "memory");
                        asm volatile("tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, 1;" ::"r"(tacc),
                                     "l"(dah), "l"(dbl), "r"(kIdesc)
                                     : "memory");
                        asm volatile("tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, 1;" ::"r"(tacc),
                                     "l"(dah), "l"(dbh), "r"(kIdesc)
                                     : "memory");
                    }
                    tc_commit(empty_bar(s));
                }
                if (ok) tc_commit(accf_bar(x));
            }
            // every MMA issued above has completed before the teardown frees tensor memory
            tc_commit(fin_bar);
            mbar_wait(fin_bar, 0);
        }
        __syncwarp();
    } else if (warp < 4) {
        // ---- converters: A -> A_hi in place, A_lo beside it
        const int t = threadIdx.x - 64;
        const long long total = static_cast<long long>(mine) * nk;
        for (long long g = 0; g < total; ++g) {
            const int s = static_cast<int>(g & 1);
            if (!mbar_wait(full_bar(s), static_cast<uint32_t>((g >> 1) & 1))) {
                atomicExch(err, 1);
                break;
            }
            float4* ah = reinterpret_cast<float4*>(gbase + s * kSplitStage);
            float4* al = reinterpret_cast<float4*>(gbase + s * kSplitStage + kSplitA);
#pragma unroll 4
            for (int i = t; i < static_cast<int>(kSplitA / 16); i += kConvThreads) {
                const float4 v = ah[i];
                float4 h, l;
                h.x = tf32_round(v.x);
                h.y = tf32_round(v.y);
                h.z = tf32_round(v.z);
                h.w = tf32_round(v.w);
                l.x = tf32_round(v.x - h.x);
                l.y = tf32_round(v.y - h.y);
                l.z = tf32_round(v.z - h.z);
                l.w = tf32_round(v.w - h.w);
                ah[i] = h;
                al[i] = l;
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(conv_bar(s)) : "memory");
        }
    } else {
        // ---- epilogue: warp 4 + q reads tensor-memory lanes (tile rows) 32 q .. 32 q + 31
        const int q = warp - 4;
        float* buf = reinterpret_cast<float*>(gbase + kSplitRing + q * kEpiBuf);  // [32][33]
        for (int i = 0; i < mine; ++i) {
            const int x = i & 1;
            int m0, n0;
            tile_of(i, m0, n0);
            if (!mbar_wait(accf_bar(x), static_cast<uint32_t>((i >> 1) & 1))) {
                atomicExch(err, 1);
                break;
            }
            tc_fence_after();
            const uint32_t taddr = tmem + (static_cast<uint32_t>(q * 32) << 16) + static_cast<uint32_t>(x * kSplitBN);
            for (int c0 = 0; c0 < kSplitBN; c0 += 32) {
                uint32_t v[32];
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
                    "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
                    "%30, %31}, [%32];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                      "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                      "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]),
                      "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]),
                      "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                    : "r"(taddr + static_cast<uint32_t>(c0)));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int j = 0; j < 32; ++j) buf[lane * 33 + j] = __uint_as_float(v[j]);
                __syncwarp();
                const int col = n0 + c0 + lane;
                for (int rr = 0; rr < 32; ++rr) {
                    const int row = m0 + q * 32 + rr;
                    if (row < M && col < N) out[static_cast<long long>(row) * ldo + col] = buf[rr * 33 + lane];
                }
                __syncwarp();
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(acce_bar(x)) : "memory");
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * kSplitBN)
                     : "memory");
    }
}

// Row-major BF16 transpose: out[c][r] = in[r][c] for rows x cols.
__global__ void transpose_bf16_kernel(const __nv_bfloat16* __restrict__ in, int rows, int cols, int ld_in,
                                      __nv_bfloat16* __restrict__ out, int ld_out)
{
    __shared__ __nv_bfloat16 tile[32][34];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int r = r0 + i, c = c0 + threadIdx.x;
        if (r < rows && c < cols) tile[i][threadIdx.x] = in[static_cast<long long>(r) * ld_in + c];
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int c = c0 + i, r = r0 + threadIdx.x;
        if (r < rows && c < cols) out[static_cast<long long>(c) * ld_out + r] = tile[threadIdx.x][i];
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// Tensor map of a row-major matrix [rows x cols] (leading dimension ld) of
// BF16 or FP32 (read as TF32) elements, boxes of box_rows rows x 128 bytes in
// the 128-byte swizzled layout.
bool make_map(CUtensorMap* map, const void* ptr, int rows, int cols, int ld, bool fp32, int box_rows)
{
    auto fn = encode_fn();
    if (!fn) return false;
    const int esize = fp32 ? 4 : 2;
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(cols), static_cast<cuuint64_t>(rows)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(ld) * esize};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(kRowBytes / esize), static_cast<cuuint32_t>(box_rows)};
    const cuuint32_t estr[2] = {1, 1};
    return fn(map, fp32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr),
              dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <bool TF32, int BN>
bool configure()
{
    static bool configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return false;
    if (!configured[dev]) {
        if (cudaFuncSetAttribute(tc_gemm_kernel<TF32, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(TileCfg<BN>::kSmem)) != cudaSuccess)
            return false;
        configured[dev] = true;
    }
    return true;
}

template <bool TF32>
bool configure_all()
{
    return configure<TF32, 128>() && configure<TF32, 256>();
}

bool eligible(const void* A, int lda, const void* B, int ldb, int esize)
{
    const int align = 16 / esize;  // leading dimensions: multiples of 16 bytes
    return (reinterpret_cast<uintptr_t>(A) % 16 == 0) && (reinterpret_cast<uintptr_t>(B) % 16 == 0) &&
           lda % align == 0 && ldb % align == 0 && encode_fn() != nullptr;
}

}  // namespace

bool tc_gemm_eligible(const void* A, int lda, const void* B, int ldb) { return eligible(A, lda, B, ldb, 2); }

bool tc_gemm_ready(bool tf32) { return encode_fn() != nullptr && (tf32 ? configure_all<true>() : configure_all<false>()); }

bool tc_gemm(int M, int N, int K, const void* A, int lda, const void* B, int ldb, const TcGemmOut& o, int* err,
             cudaStream_t s)
{
    const TcPair pair{A, lda, B, ldb};
    return tc_gemm_sum(M, N, K, 1, &pair, false, o, err, s);
}

bool tc_gemm_sum(int M, int N, int K, int npairs, const TcPair* pairs, bool tf32, const TcGemmOut& o, int* err,
                 cudaStream_t s)
{
    if (M <= 0 || N <= 0 || K <= 0 || npairs < 1 || npairs > 3) return false;
    for (int p = 0; p < npairs; ++p)
        if (!eligible(pairs[p].A, pairs[p].lda, pairs[p].B, pairs[p].ldb, tf32 ? 4 : 2)) return false;
    if (!(tf32 ? configure_all<true>() : configure_all<false>())) return false;
    const int bn = N >= 256 ? 256 : 128;  // wide tiles halve the re-reads of A
    TcMaps maps;
    for (int p = 0; p < npairs; ++p)
        if (!make_map(&maps.a[p], pairs[p].A, M, K, pairs[p].lda, tf32, kBM) ||
            !make_map(&maps.b[p], pairs[p].B, N, K, pairs[p].ldb, tf32, bn))
            return false;
    const long long tiles = static_cast<long long>((N + bn - 1) / bn) * ((M + kBM - 1) / kBM);
    if (tiles > 0x7fffffffll) return false;
    const dim3 grid(static_cast<unsigned>(tiles));
    if (tf32 && bn == 256)
        tc_gemm_kernel<true, 256><<<grid, 128, TileCfg<256>::kSmem, s>>>(maps, M, N, K, npairs, o, err);
    else if (tf32)
        tc_gemm_kernel<true, 128><<<grid, 128, TileCfg<128>::kSmem, s>>>(maps, M, N, K, npairs, o, err);
    else if (bn == 256)
        tc_gemm_kernel<false, 256><<<grid, 128, TileCfg<256>::kSmem, s>>>(maps, M, N, K, npairs, o, err);
    else
        tc_gemm_kernel<false, 128><<<grid, 128, TileCfg<128>::kSmem, s>>>(maps, M, N, K, npairs, o, err);
    return true;
}

bool tc_split_gemm(int M, int N, int K, const float* A, int lda, const float* Bhi, const float* Blo, int ldb,
                   float* out, int ldo, int* err, cudaStream_t s)
{
    if (M <= 0 || N <= 0 || K <= 0) return false;
    if (!eligible(A, lda, Bhi, ldb, 4) || !eligible(A, lda, Blo, ldb, 4)) return false;
    static bool configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return false;
    if (!configured[dev]) {
        if (cudaFuncSetAttribute(tc_split_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(kSplitSmem)) != cudaSuccess)
            return false;
        configured[dev] = true;
    }
    CUtensorMap ma, mbh, mbl;
    if (!make_map(&ma, A, M, K, lda, true, kBM) || !make_map(&mbh, Bhi, N, K, ldb, true, kSplitBN) ||
        !make_map(&mbl, Blo, N, K, ldb, true, kSplitBN))
        return false;
    const long long tiles = static_cast<long long>((N + kSplitBN - 1) / kSplitBN) * ((M + kBM - 1) / kBM);
    if (tiles > 0x7fffffffll) return false;
    static int sms[64] = {};
    if (sms[dev] == 0 && cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return false;
    const unsigned grid = static_cast<unsigned>(tiles < sms[dev] ? tiles : sms[dev]);  // persistent: one CTA per SM
    tc_split_gemm_kernel<<<grid, kSplitThreads, kSplitSmem, s>>>(ma, mbh, mbl, M, N, K, out, ldo, err);
    return true;
}

void launch_transpose_bf16(const void* in, int rows, int cols, int ld_in, void* out, int ld_out, cudaStream_t s)
{
    const dim3 grid((cols + 31) / 32, (rows + 31) / 32), block(32, 8);
    transpose_bf16_kernel<<<grid, block, 0, s>>>(static_cast<const __nv_bfloat16*>(in), rows, cols, ld_in,
                                                 static_cast<__nv_bfloat16*>(out), ld_out);
}

}  // namespace hx
