// Persistent stage kernel for d = 64 on Hermitian-packed slabs with sigma_z
// couplings (every V_j = sigma_z of one spin): the C2 workload's hot path.
//
// Same mathematics as herm_kernel (hx_fused.cu) and stage_kernel
// (hx_stage.cu): one launch evaluates out_n = base_n + alpha L(u)_n for every
// ADO n, L being the reference right-hand side (getdRhoSparse,
// src/liouville.cu:749-869).  What differs is how the work is fed to the SMs:
//
//  * one CTA per SM; a producer warp draws ADOs from a ticket counter in index
//    order and streams, for each, its own packed slab, the packed slabs of its
//    neighbour entries and its Horner base into a ring of kRing shared-memory
//    slots with TMA bulk copies (one mbarrier per slot signals arrival,
//    another the consumers' release), so kRing slabs (130 KB) stay in flight
//    per SM whatever the consumers are doing; an L2 prefetch two ADOs per SM
//    ahead covers the DRAM latency of slabs not yet in L2;
//  * 17 consumer warps (544 threads) do the element work; thread t owns one
//    column c and four consecutive rows r0..r0+3 (r0 a multiple of 4) of the
//    upper triangle: 8 quads of packed rows x 68 column slots (rows 4q..4q+3
//    from column 4q on, then rows 60-4q..63-4q from column 60-4q on, the two
//    halves of packed rows 4q..4q+3), 2080 elements plus 48 lower-triangle
//    slots of the diagonal 4x4 blocks; every slot read is 32 consecutive
//    packed elements per warp;
//  * the two low row-bit flips of the transverse field are register moves;
//    the four higher row-bit flips and the six column-bit flips read a full
//    swizzled copy of the slab, element (r, c) in slot 64 r + (c ^ r) (every
//    flip is one XOR of the slot, every quarter-warp access touches eight
//    distinct 16-byte bank groups), written once (element and mirror);
//  * the ADO-independent diagonal term comes from two 64-entry tables:
//    Re T = -4 sum_j xi_j [bit_j(r) != bit_j(c)] (table over r ^ c) and
//    Im T = -(E_r - E_c) (the counter term vanishes for sigma_z);
//  * neighbour entries are consumed from the ring; with sigma_z couplings
//    only the elements whose commutator or anti-commutator weight is nonzero
//    are read.
// Every mbarrier wait has a poll budget; a wait that runs out sets the error
// word, and producer and consumers leave at the next ADO boundary after the
// copies in flight have landed.

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>

#include "hx_internal.h"

namespace hx {

namespace {

constexpr int kD = 64;
constexpr int kP = 2080;  // packed elements of a 64 x 64 Hermitian slab
constexpr int kRing = 4;
constexpr int kConsumerWarps = 17;
constexpr int kConsumers = 32 * kConsumerWarps;  // 8 quads x 68 column slots
constexpr int kThreads = kConsumers + 32;       // + the producer warp
constexpr uint32_t kSlabBytes = kP * sizeof(double2);
constexpr uint32_t kSpin = 1u << 22;  // poll budget of every mbarrier wait

enum ItemKind : int { kItemOwn = 0, kItemEntry = 1, kItemBase = 2, kItemEnd = 3 };

struct __align__(16) SlotMeta {
    int kind;
    int ado;
    int bit;    // entry: spin of V_j
    int count;  // own: neighbour entries that follow
    double wc;  // entry: commutator weight
    double wa;  // entry: anti-commutator weight
    double g;   // own: damping sum
    int uslot;  // own: slot in U (tier L-1 with an up-term pass) or -1
    int pad;
};

__device__ __forceinline__ uint32_t saddr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ uint64_t policy_last()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ uint64_t policy_first()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ double2 load_stream(const double2* p)
{
    double2 v;
    asm volatile("ld.global.cs.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
    return v;
}

__device__ __forceinline__ void store_stream(double2* p, double2 v)
{
    asm volatile("st.global.cs.v2.f64 [%0], {%1, %2};" ::"l"(p), "d"(v.x), "d"(v.y) : "memory");
}

__device__ __forceinline__ void prefetch_l2(const void* src, uint32_t bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ int full_slot(int r, int c) { return (r << 6) | (c ^ r); }

__device__ __forceinline__ void bar_init(uint64_t* b, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void bar_arrive(uint64_t* b)
{
    asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(saddr(b)) : "memory");
}

__device__ __forceinline__ bool bar_wait(uint64_t* b, uint32_t parity)
{
    for (uint32_t i = 0; i < kSpin; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(saddr(b)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Arm the slot's barrier for one slab and start its copy.
__device__ __forceinline__ void load_slab(void* dst, const void* src, uint64_t* b, uint64_t pol)
{
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(b)),
                 "r"(kSlabBytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::
            "r"(saddr(dst)),
        "l"(src), "r"(kSlabBytes), "r"(saddr(b)), "l"(pol)
        : "memory");
}

// Slot of the producer's next item, once the consumers released its previous
// use; -1 if that wait ran out of its budget.
__device__ __forceinline__ int acquire_slot(uint64_t* empty_bar, uint32_t it)
{
    const int k = static_cast<int>(it % kRing);
    if (it >= kRing && !bar_wait(&empty_bar[k], ((it / kRing) - 1) & 1)) return -1;
    return k;
}

__device__ __forceinline__ void consumers_sync() { asm volatile("bar.sync 1, %0;" ::"n"(kConsumers) : "memory"); }

// Barrier of the consumer warps that also returns whether any of them passed v = true.
__device__ __forceinline__ bool consumers_any(bool v)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 q, %1, 0;\n\tbar.red.or.pred p, 1, %2, q;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(r)
        : "r"(static_cast<uint32_t>(v)), "n"(kConsumers)
        : "memory");
    return r != 0;
}

// 18 warps: the busiest of the four SM sub-partitions holds 5 of them, and its
// 16K registers cap a thread at 96.
__global__ void __launch_bounds__(kThreads, 1)
    herm64_kernel(FusedArgs a, const double2* __restrict__ u, const double2* rho, double2* out, double alpha,
                  int base_kind)
{
    extern __shared__ __align__(128) unsigned char smem[];
    double2* full = reinterpret_cast<double2*>(smem);               // [64 * 64], swizzled
    double2* ring = full + kD * kD;                                  // [kRing][kP]
    SlotMeta* meta = reinterpret_cast<SlotMeta*>(ring + kRing * kP);  // [kRing]
    uint64_t* full_bar = reinterpret_cast<uint64_t*>(meta + kRing);   // [kRing]
    uint64_t* empty_bar = full_bar + kRing;                           // [kRing]
    double* sE = reinterpret_cast<double*>(empty_bar + kRing);       // [64] E_r
    double* sX = sE + kD;                                             // [64] 4 sum_j xi_j [bit_j(m)]
    double* sH = sX + kD;                                             // [8] transverse field

    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    if (tid == 0) {
        for (int k = 0; k < kRing; ++k) {
            bar_init(&full_bar[k], 1);
            bar_init(&empty_bar[k], kConsumerWarps);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (tid < kD) {
        sE[tid] = a.hdiag[tid];
        double sx = 0.0;
        for (int jj = 0; jj < a.J; ++jj)
            if ((tid >> a.vbit[jj]) & 1) sx += a.xi[jj];
        sX[tid] = 4.0 * sx;
    }
    if (tid < 6) sH[tid] = a.hflip[tid];
    __syncthreads();

    if (warp == kConsumerWarps) {
        // ---------------- producer (one thread) ----------------
        if ((tid & 31) != 0) return;
        const uint64_t keep = policy_last(), first = policy_first();
        const unsigned ahead = 2 * gridDim.x;
        uint32_t item = 0;
        bool ok = true;
        while (ok) {
            const long long n = atomicAdd(&a.ticket[0], 1);
            if (n >= a.H) break;
            if (n + ahead < a.H) {
                const long long m = a.order ? a.order[n + ahead] : n + ahead;
                prefetch_l2(u + m * kP, kSlabBytes);
                if (base_kind == kBaseRho) prefetch_l2(rho + m * kP, kSlabBytes);
            }
            const long long ado = a.order ? a.order[n] : n;
            const int Q = a.ent_count[ado];
            int k = acquire_slot(empty_bar, item);
            if (k < 0) {
                ok = false;
                break;
            }
            meta[k].kind = kItemOwn;
            meta[k].ado = static_cast<int>(ado);
            meta[k].count = Q;
            meta[k].g = a.gsum[ado];
            meta[k].uslot = a.slot ? a.slot[ado] : -1;
            load_slab(ring + k * kP, u + ado * kP, &full_bar[k], keep);
            ++item;
            for (int e = 0; e < Q; ++e) {
                const long long src = ado * 2 * a.M + e;
                k = acquire_slot(empty_bar, item);
                if (k < 0) {
                    ok = false;
                    break;
                }
                meta[k].kind = kItemEntry;
                meta[k].ado = static_cast<int>(ado);
                meta[k].bit = a.vbit[a.ent_bath[src] & 0xffff];
                meta[k].wc = a.ent_wc[src];
                meta[k].wa = a.ent_wa[src];
                load_slab(ring + k * kP, u + static_cast<long long>(a.ent_slab[src]) * kP, &full_bar[k], keep);
                ++item;
            }
            if (ok && base_kind == kBaseRho) {
                k = acquire_slot(empty_bar, item);
                if (k < 0) {
                    ok = false;
                    break;
                }
                meta[k].kind = kItemBase;
                meta[k].ado = static_cast<int>(ado);
                load_slab(ring + k * kP, rho + ado * kP, &full_bar[k], first);
                ++item;
            }
        }
        if (ok) {
            const int k = acquire_slot(empty_bar, item);
            if (k >= 0) {
                meta[k].kind = kItemEnd;
                bar_arrive(&full_bar[k]);
                ++item;
            } else {
                ok = false;
            }
        }
        if (!ok) atomicExch(a.error_flag, 1);
        // every copy this CTA started has landed before it exits
        for (uint32_t it = item > kRing ? item - kRing : 0; it < item; ++it)
            bar_wait(&full_bar[it % kRing], (it / kRing) & 1);
        // the last CTA to finish resets the ticket counter for the next launch
        __threadfence();
        if (atomicAdd(&a.ticket[1], 1) == static_cast<int>(gridDim.x) - 1) {
            a.ticket[0] = 0;
            a.ticket[1] = 0;
            __threadfence();
        }
        return;
    }

    // ---------------- consumers (544 threads) ----------------
    const int lane = tid & 31;
    const int q = tid / 68, j = tid - 68 * q;
    const bool grp_a = j < kD - 4 * q;
    const int r0 = grp_a ? 4 * q : 60 - 4 * q;
    const int c = grp_a ? 4 * q + j : j - 4;
    const int pidx = grp_a ? 64 * r0 + c : 65 * (63 - r0) + c + 1;  // packed index of (r0, c)
    const int pstep = grp_a ? 64 : -65;                               // ... per row
    const int nup = c - r0;  // row r0 + x is in the upper triangle iff x <= nup
    const double ec = sE[c];
    uint32_t item = 0;
    bool failed = false;

    // wait for an item; after a wait that ran out of its budget the thread
    // runs on without waiting until all consumers leave at the next ADO
#define HX_WAIT_ITEM(k_out)                                                 \
    do {                                                                    \
        (k_out) = static_cast<int>(item % kRing);                           \
        if (!failed && !bar_wait(&full_bar[(k_out)], (item / kRing) & 1)) { \
            failed = true;                                                  \
            atomicExch(a.error_flag, 1);                                    \
        }                                                                   \
    } while (0)
#define HX_RELEASE(k_in)                               \
    do {                                               \
        __syncwarp();                                  \
        if (lane == 0) bar_arrive(&empty_bar[(k_in)]); \
    } while (0)

    for (;;) {
        int k;
        HX_WAIT_ITEM(k);
        // one barrier: every consumer is done with the previous ADO (its reads
        // of `full`), and all leave together at the end marker or after a
        // wait that ran out of its budget
        if (consumers_any(failed || meta[k].kind == kItemEnd)) break;
        const long long n = meta[k].ado;
        const int Q = meta[k].count;
        const double g = meta[k].g;
        const int uslot = meta[k].uslot;
        double2 xv[4];
        const double2* own = ring + k * kP + pidx;
#pragma unroll
        for (int x = 0; x < 4; ++x) xv[x] = x <= nup ? own[pstep * x] : make_double2(0.0, 0.0);
#pragma unroll
        for (int x = 0; x < 4; ++x) {
            if (x <= nup) {
                const int r = r0 + x;
                full[full_slot(r, c)] = xv[x];
                if (r != c) full[full_slot(c, r)] = make_double2(xv[x].x, -xv[x].y);
            }
        }
        HX_RELEASE(k);
        ++item;
        consumers_sync();
        // lower-triangle slots of the diagonal blocks: their values (mirrors) for the register flips
#pragma unroll
        for (int x = 1; x < 4; ++x)
            if (x > nup) xv[x] = full[full_slot(r0 + x, c)];

        // ---- diagonal and transverse field: per flip bit h_b (X(r ^ 2^b, c) -
        // X(r, c ^ 2^b)); on the diagonal the two are conjugates, so the real
        // part cancels exactly and the diagonal stays real
        double2 acc[4];
#pragma unroll
        for (int x = 0; x < 4; ++x) {
            const int r = r0 + x;
            const int sl = full_slot(r, c);
            double hr = 0.0, hi = 0.0;
#pragma unroll
            for (int b = 0; b < 6; ++b) {
                const double2 rp = b < 2 ? xv[x ^ (1 << b)] : full[sl ^ ((1 << b) << 6) ^ (1 << b)];
                const double2 cp = full[sl ^ (1 << b)];
                hr += sH[b] * (rp.x - cp.x);
                hi += sH[b] * (rp.y - cp.y);
            }
            const double tr = -sX[r ^ c] - g;
            const double ti = ec - sE[r];
            acc[x].x = tr * xv[x].x - ti * xv[x].y + hi;
            acc[x].y = tr * xv[x].y + ti * xv[x].x - hr;
        }

        // ---- neighbour entries: sigma_z of spin `bit` -> v = +-1; equal bits
        // of r and c -> only {V, X} = +-2 X; different bits -> only [V, X] = +-2 X
        for (int e = 0; e < Q; ++e) {
            HX_WAIT_ITEM(k);
            const int bit = meta[k].bit;
            const double a2 = 2.0 * meta[k].wa, c2 = 2.0 * meta[k].wc;
            const bool need_same = a2 != 0.0, need_diff = c2 != 0.0;
            const double2* src = ring + k * kP + pidx;
            const int bc = (c >> bit) & 1;
#pragma unroll
            for (int x = 0; x < 4; ++x) {
                const int br = ((r0 + x) >> bit) & 1;
                const bool same = br == bc;
                if (x <= nup && (same ? need_same : need_diff)) {
                    const double2 y = src[pstep * x];
                    const double w = same ? (br ? -a2 : a2) : (br ? -c2 : c2);
                    acc[x].x += w * (same ? y.x : -y.y);
                    acc[x].y += w * (same ? y.y : y.x);
                }
            }
            HX_RELEASE(k);
            ++item;
        }
        // ---- up terms of tier L-1, when upterm_kernel summed them
        if (uslot >= 0) {
            const double2* Un = a.U + static_cast<long long>(uslot) * kP + pidx;
#pragma unroll
            for (int x = 0; x < 4; ++x) {
                if (x > nup) continue;
                const double2 w = load_stream(Un + pstep * x);
                acc[x].x += w.x;
                acc[x].y += w.y;
            }
        }
        // ---- Horner epilogue
        double2 base[4];
        if (base_kind == kBaseRho) {
            HX_WAIT_ITEM(k);
            const double2* bsrc = ring + k * kP + pidx;
#pragma unroll
            for (int x = 0; x < 4; ++x) base[x] = x <= nup ? bsrc[pstep * x] : make_double2(0.0, 0.0);
            HX_RELEASE(k);
            ++item;
        } else {
#pragma unroll
            for (int x = 0; x < 4; ++x)
                base[x] = base_kind == kBaseSelf ? full[full_slot(r0 + x, c)] : make_double2(0.0, 0.0);
        }
        double2* outn = out + n * kP + pidx;
#pragma unroll
        for (int x = 0; x < 4; ++x) {
            if (x > nup) continue;
            store_stream(outn + pstep * x, make_double2(base[x].x + alpha * acc[x].x, base[x].y + alpha * acc[x].y));
        }
    }
#undef HX_WAIT_ITEM
#undef HX_RELEASE
}

size_t herm64_smem()
{
    return size_t(kD) * kD * sizeof(double2) + size_t(kRing) * kSlabBytes + kRing * sizeof(SlotMeta) +
           2 * kRing * sizeof(uint64_t) + sizeof(double) * (2 * kD + 8);
}

}  // namespace

bool herm64_supported(int logd, int M, int J, int pauli)
{
    (void)M;
    return logd == 6 && pauli && J <= kD && herm64_smem() <= 227 * 1024;
}

bool prepare_herm64()
{
    static size_t configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return false;
    if (configured[dev] == 0) {
        if (cudaFuncSetAttribute(herm64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(herm64_smem())) != cudaSuccess)
            return false;
        // the block must fit one SM (registers and shared memory)
        cudaFuncAttributes fa{};
        if (cudaFuncGetAttributes(&fa, herm64_kernel) != cudaSuccess || fa.maxThreadsPerBlock < kThreads)
            return false;
        configured[dev] = herm64_smem();
    }
    return true;
}

bool launch_herm64(const FusedArgs& a, const double2* u, const double2* rho, double2* out, double alpha, int base_kind,
                   cudaStream_t s)
{
    if (!a.ticket || a.sms <= 0 || !prepare_herm64()) return false;
    const unsigned grid = static_cast<unsigned>(a.H < a.sms ? a.H : a.sms);
    herm64_kernel<<<grid, kThreads, herm64_smem(), s>>>(a, u, rho, out, alpha, base_kind);
    return true;
}

}  // namespace hx
