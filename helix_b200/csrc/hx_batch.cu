// Batched propagation of many independent HEOM instances (disorder averages).
//
// Instances with d >= 32 are large enough to fill the GPU on their own: they
// run as internal contexts whose up-term and fused kernels (hx_upterm.cu,
// hx_fused.cu) are issued into the same captured step on eight forked
// streams; all smaller instances are packed into the arena below.
//
// A batch holds hundreds of spin-glass instances of uneven size (Hilbert
// dimension d = 2^N, hierarchy depth, bath parameters) in one device arena.
// Every bath couples through sigma_z of one spin (V_j = sz(p_j), eigenvalues
// +-1), as in the batched disorder-average workload, so every bath term is an
// elementwise factor that follows from two bits of the element index:
//   [V_j, X]_rc = del X_rc,  {V_j, X}_rc = sig X_rc,
//   del = s(r) - s(c), sig = s(r) + s(c), s(x) = +-1 from bit p_j of x,
// and exactly one of del, sig is nonzero (2 s(r)).
//
// Layout: the states of all instances are concatenated slab by slab; the
// neighbour lists depend only on the hierarchy shape (modes, depth, modes
// per bath) and are built once per shape, grouped by bath with the Drude
// mode's down neighbour apart; per instance there is one small block of
// constants, the damping sum of every ADO and the ADO-independent diagonal
// coefficient table.  One stage of the integrator is one persistent,
// warp-specialised launch over all instances:
//
//  * the work list is a list of tiles, each a run of consecutive ADOs of one
//    instance (tile_elems / d^2 ADOs, at least one), so small slabs (d = 8:
//    1 KB) are packed into CTA-sized work items; a tile's descriptor carries
//    every offset it needs;
//  * warp 0 of every CTA is the producer: for each of the CTA's tiles it
//    fills one slot of a two-slot shared-memory ring with five TMA bulk
//    copies (the tile's slabs, its Horner base rho, the shape's neighbour
//    blocks, the instance's constants and the tile's damping sums),
//    signalled on the slot's mbarrier;
//  * warps 1-8 are the consumers: they expand the tile's entries into
//    weights (shared memory only), then a group of G threads (a warp or more
//    for d >= 8) computes one ADO at a time, so the entry loops are uniform
//    within the group; each thread keeps up to four elements in registers
//    (two row flips of the transverse field are register moves); per bath,
//    the commutator neighbours are summed unweighted by del and loaded only
//    where del != 0, and the Drude down neighbour once;
//  * per element the right-hand side is the reference's (getdRhoSparse,
//    src/liouville.cu:749-869), with the Horner epilogue of the Taylor
//    integrator (develop(), src/liouville.cu:502-590).
//
// Every wait on an mbarrier is bounded; a wait that runs out sets the error
// word, which the host reports as DeviceWaitTimeout.  One integrator step
// (its stage launches plus the disorder-average reduction of <sigma_z> of one
// spin over all instances) is captured once in a CUDA graph and replayed.
// Each Hilbert dimension present has its own persistent kernel (the
// element mapping is fixed at compile time); its tile size and variant
// (elements per thread, CTAs per SM) are picked by a timing autotuner over a
// fixed candidate list.
//
// The reference has no batched mode; its single-instance path is
// HEOMSolver::run (src/helix.cpp:723-772).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "hx_internal.h"

using hx::fail;

namespace hx {

// Host bookkeeping per instance.
struct BatchInst {
    long long state_off;  // double2 offset of ADO 0 in the state arrays
    long long ent_off;    // int offset of the shape's block of ADO 0
    long long diag_off;   // double2 offset of the instance's d x d diagonal table
    long long blk_off;    // double offset of the instance constants (even)
    long long g_off;      // double offset of the instance's damping sums (even)
    int blk_len;          // doubles in the constant block (even)
    int eba;              // ints per ADO block (multiple of 4)
    int H, M, J, logd;
};

// One work item of the stage kernel; every offset is precomputed.
struct __align__(16) BatchTile {
    long long tile_off;  // double2 offset of the tile's first element
    long long inst_off;  // double2 offset of the instance's ADO 0 (neighbour slabs)
    long long ent_off;   // int offset of the tile's first ADO block
    long long diag_off;  // double2 offset of the instance's diagonal table
    long long blk_off;   // double offset of the instance constants
    long long g_off;     // double offset of the damping sums, rounded down to even
    int nado, logd, M, J, eba, blk_len;
    int g_shift;         // 0 or 1: ADO ado0 sits at g_off + g_shift
    int g_len;           // doubles copied (even)
};

struct BatchArgs {
    const BatchTile* tiles;
    const int32_t* ent;     // per shape, per ADO block (see batch_entries_kernel)
    const double* blk;      // per instance: hflip[logd] nu[M] tcoef[M] theta_a[J] spin[J]
    const double* gsum;     // per instance: sum_m nu_m n_m of every ADO
    const double2* diag;
    int* error_flag;
    int ntiles;
    int buf_elems;          // elements of one slab buffer
    int max_tile_ados, max_M, max_J, max_eba, max_blk;
};

namespace {

constexpr int kConsumers = 256;              // consumer threads (warps 1-8)
constexpr int kThreads = kConsumers + 32;    // plus the producer warp
constexpr uint32_t kSpin = 1u << 20;         // poll budget of every mbarrier wait

__device__ __forceinline__ uint32_t sm_u32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void bar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sm_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void bar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(sm_u32(bar)) : "memory");
}

__device__ __forceinline__ void bar_arrive_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sm_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     sm_u32(dst)),
                 "l"(src), "r"(bytes), "r"(sm_u32(bar))
                 : "memory");
}

// As bulk_g2s, with the L2 evict-first policy (data read once per stage).
__device__ __forceinline__ void bulk_g2s_stream(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::
            "r"(sm_u32(dst)),
        "l"(src), "r"(bytes), "r"(sm_u32(bar)), "l"(pol)
        : "memory");
}

__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity)
{
    for (uint32_t i = 0; i < kSpin; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(sm_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void consumer_sync() { asm volatile("bar.sync 1, %0;" ::"n"(kConsumers) : "memory"); }

// ADO block of a shape (ints, length eba):
//   [0, J)            Drude down neighbour of bath j, or -1
//   [J, 2J)           n of the Drude mode of bath j (its down-coupling factor)
//   [2J, 3J+1)        start of bath j's commutator entries (entry J: their count)
//   [3J+1, 3J+1+2M)   commutator entry slab (up neighbours, down neighbours of Pade modes)
//   [3J+1+2M, 3J+1+4M) commutator entry meta = mode | up << 8 | n_mode << 16
__host__ __device__ constexpr int ent_block_ints(int M, int J) { return (3 * J + 1 + 4 * M + 3) & ~3; }

// Weights of the tile being computed, expanded by the consumers.
struct TileWeights {
    const int* ent;      // the slot's ADO blocks
    const int* cslab;    // [tile ADOs][2M] commutator slabs
    const double* cw;    // [tile ADOs][2M] commutator weights
    const double* dwc;   // [tile ADOs][J] Drude down: commutator weight
    const double* dwa;   // [tile ADOs][J] Drude down: anticommutator weight
    const double* g;     // damping sum of ADO al at g[al]
    const double* spin;  // [J] spin of bath j
    int eba, M2, J;
};

// One ADO's stage for d = 2^LOGD, computed by a group of G consumer threads.
// Element e = rd*G*EPT + lg + G*k (k < EPT): every thread keeps one column c
// (G >= d), and the k-bits of e are row bits, so those row flips of the
// transverse field are register moves.
template <int LOGD, int EMAX>
__device__ __forceinline__ void ado_stage(int al, int lg, const TileWeights& tw, const double2* xs, const double2* bs,
                                          const double2* __restrict__ Tdiag, const double* sF,
                                          const double2* __restrict__ ui, double2* o, double alpha, int base_kind)
{
    constexpr int D = 1 << LOGD, D2 = D * D;
    constexpr int E0 = D2 >= 128 ? 4 : (D2 >= 64 ? 2 : 1);
    constexpr int EPT = E0 < EMAX ? E0 : EMAX;
    constexpr int G = (D2 / EPT) < kConsumers ? (D2 / EPT) : kConsumers;
    constexpr int ROUNDS = D2 / (G * EPT);
    constexpr int GB = G == 1 ? 0 : (G == 2 ? 1 : (G == 4 ? 2 : (G == 8 ? 3 : (G == 16 ? 4 : (G == 32 ? 5 :
                       (G == 64 ? 6 : (G == 128 ? 7 : 8)))))));  // log2 G
    const int J = tw.J;
    const int* blk = tw.ent + al * tw.eba;
    const int* dslab = blk;
    const int* cstart = blk + 2 * J;
    const int* cs = tw.cslab + al * tw.M2;
    const double* cw = tw.cw + al * tw.M2;
    const double* dwc = tw.dwc + al * J;
    const double* dwa = tw.dwa + al * J;
    const double g = tw.g[al];
    const int c = lg & (D - 1);
#pragma unroll 1
    for (int rd = 0; rd < ROUNDS; ++rd) {
        const int e0 = rd * G * EPT + lg;
        double2 x[EPT], acc[EPT];
        int r[EPT];
#pragma unroll
        for (int k = 0; k < EPT; ++k) {
            r[k] = (e0 + G * k) >> LOGD;
            x[k] = xs[e0 + G * k];
        }
        // diagonal table, transverse field and damping
#pragma unroll
        for (int k = 0; k < EPT; ++k) {
            const int e = e0 + G * k;
            const double2 T = __ldg(Tdiag + e);
            double hr = 0.0, hi = 0.0;
#pragma unroll
            for (int i = 0; i < LOGD; ++i) {
                const int eb = i + LOGD;  // row bit i of the element index
                double2 p;
                if (eb >= GB && eb < GB + 2 && (1 << (eb - GB)) < EPT) p = x[k ^ (1 << (eb - GB))];
                else p = xs[e ^ (1 << eb)];
                const double2 q = xs[e ^ (1 << i)];
                hr += sF[i] * (p.x - q.x);
                hi += sF[i] * (p.y - q.y);
            }
            const double tr = T.x - g;
            acc[k].x = tr * x[k].x - T.y * x[k].y + hi;
            acc[k].y = tr * x[k].y + T.y * x[k].x - hr;
        }
        // bath terms
        for (int j = 0; j < J; ++j) {
            const int p = static_cast<int>(tw.spin[j]);
            bool mask[EPT];
            double sr2[EPT];
            double2 S[EPT];
#pragma unroll
            for (int k = 0; k < EPT; ++k) {
                mask[k] = (((r[k] ^ c) >> p) & 1) != 0;
                sr2[k] = ((r[k] >> p) & 1) ? 2.0 : -2.0;
                S[k] = make_double2(0.0, 0.0);
            }
            // Drude down neighbour: -i del wc_d X - sig wa_d X
            const int ds = dslab[j];
            if (ds >= 0) {
                const double wc = dwc[j], wa = dwa[j];
                const double2* sp = ui + (static_cast<long long>(ds) << (2 * LOGD)) + e0;
#pragma unroll
                for (int k = 0; k < EPT; ++k) {
                    const double2 y = __ldg(sp + G * k);
                    if (mask[k]) {
                        S[k].x = wc * y.x;
                        S[k].y = wc * y.y;
                    } else {
                        acc[k].x -= sr2[k] * wa * y.x;
                        acc[k].y -= sr2[k] * wa * y.y;
                    }
                }
            }
            // commutator neighbours, two at a time, loaded only where del != 0
            int q = cstart[j];
            const int qe = cstart[j + 1];
            for (; q + 1 < qe; q += 2) {
                const double w0 = cw[q], w1 = cw[q + 1];
                const double2* s0 = ui + (static_cast<long long>(cs[q]) << (2 * LOGD)) + e0;
                const double2* s1 = ui + (static_cast<long long>(cs[q + 1]) << (2 * LOGD)) + e0;
                double2 y0[EPT], y1[EPT];
#pragma unroll
                for (int k = 0; k < EPT; ++k) {
                    y0[k] = make_double2(0.0, 0.0);
                    y1[k] = make_double2(0.0, 0.0);
                    if (mask[k]) {
                        y0[k] = __ldg(s0 + G * k);
                        y1[k] = __ldg(s1 + G * k);
                    }
                }
#pragma unroll
                for (int k = 0; k < EPT; ++k) {
                    S[k].x += w0 * y0[k].x + w1 * y1[k].x;
                    S[k].y += w0 * y0[k].y + w1 * y1[k].y;
                }
            }
            if (q < qe) {
                const double w0 = cw[q];
                const double2* s0 = ui + (static_cast<long long>(cs[q]) << (2 * LOGD)) + e0;
#pragma unroll
                for (int k = 0; k < EPT; ++k) {
                    if (mask[k]) {
                        const double2 y = __ldg(s0 + G * k);
                        S[k].x += w0 * y.x;
                        S[k].y += w0 * y.y;
                    }
                }
            }
            // -i del S, del = sr2 where the bits differ (S is zero elsewhere)
#pragma unroll
            for (int k = 0; k < EPT; ++k) {
                acc[k].x += sr2[k] * S[k].y;
                acc[k].y -= sr2[k] * S[k].x;
            }
        }
        // Horner epilogue
#pragma unroll
        for (int k = 0; k < EPT; ++k) {
            const int e = e0 + G * k;
            double2 b;
            if (base_kind == kBaseSelf) b = x[k];
            else if (base_kind == kBaseRho) b = bs[e];
            else b = make_double2(0.0, 0.0);
            __stcs(o + e, make_double2(b.x + alpha * acc[k].x, b.y + alpha * acc[k].y));
        }
    }
}

template <int LOGD, int EMAX>
__device__ __forceinline__ void tile_stage(int ctid, int nado, const TileWeights& tw, const double2* sx,
                                           const double2* sb, const double2* Tdiag, const double* sF,
                                           const double2* ui, double2* out_tile, double alpha, int base_kind)
{
    constexpr int D2 = 1 << (2 * LOGD);
    constexpr int E0 = D2 >= 128 ? 4 : (D2 >= 64 ? 2 : 1);
    constexpr int EPT = E0 < EMAX ? E0 : EMAX;
    constexpr int G = (D2 / EPT) < kConsumers ? (D2 / EPT) : kConsumers;
    constexpr int NG = kConsumers / G;
    const int grp = ctid / G, lg = ctid - grp * G;
    for (int al = grp; al < nado; al += NG)
        ado_stage<LOGD, EMAX>(al, lg, tw, sx + static_cast<long long>(al) * D2, sb + static_cast<long long>(al) * D2,
                              Tdiag, sF, ui, out_tile + static_cast<long long>(al) * D2, alpha, base_kind);
}

template <int LOGD, int EMAX, int MINB>
__global__ void __launch_bounds__(kThreads, MINB)
    batch_stage_kernel(BatchArgs a, const double2* __restrict__ u, const double2* rho, double2* out, double alpha,
                       int base_kind)
{
    extern __shared__ __align__(128) unsigned char smem[];
    // two slots: slabs, base, ADO blocks, instance constants, damping sums, tile descriptor
    const size_t slab_b = static_cast<size_t>(a.buf_elems) * sizeof(double2);
    const size_t ent_b = static_cast<size_t>(a.max_tile_ados) * a.max_eba * sizeof(int);
    const size_t blk_b = static_cast<size_t>(a.max_blk) * sizeof(double);
    const size_t g_b = static_cast<size_t>((a.max_tile_ados + 3) & ~1) * sizeof(double);
    const size_t slot_b = 2 * slab_b + ent_b + blk_b + g_b + sizeof(BatchTile);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + 2 * slot_b);
    uint64_t* empty = full + 2;
    int* s_err = reinterpret_cast<int*>(empty + 2);
    const int TC = a.max_tile_ados * 2 * a.max_M;
    const int TJ = a.max_tile_ados * a.max_J;
    double* sCw = reinterpret_cast<double*>(smem + 2 * slot_b + 48);
    double* sDwc = sCw + TC;
    double* sDwa = sDwc + TJ;
    int* sCslab = reinterpret_cast<int*>(sDwa + TJ);

    const int tid = threadIdx.x;
    if (tid == 0) {
        bar_init(&full[0], 1);
        bar_init(&full[1], 1);
        bar_init(&empty[0], 1);
        bar_init(&empty[1], 1);
        *s_err = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (tid < 32) {
        // ---- producer: one lane fills the ring
        if (tid != 0) return;
        for (int t = blockIdx.x, i = 0; t < a.ntiles; t += gridDim.x, ++i) {
            const int s = i & 1;
            if (!bar_wait(&empty[s], ((i >> 1) & 1) ^ 1)) {
                atomicExch(a.error_flag, 1);
                return;
            }
            unsigned char* slot = smem + s * slot_b;
            const BatchTile tl = a.tiles[t];
            *reinterpret_cast<BatchTile*>(slot + 2 * slab_b + ent_b + blk_b + g_b) = tl;
            const uint32_t sb = static_cast<uint32_t>(static_cast<long long>(tl.nado) << (2 * tl.logd)) * 16u;
            const uint32_t eb = static_cast<uint32_t>(tl.nado * tl.eba) * 4u;
            const uint32_t bb = static_cast<uint32_t>(tl.blk_len) * 8u;
            const uint32_t gb = static_cast<uint32_t>(tl.g_len) * 8u;
            const bool with_rho = base_kind == kBaseRho;
            bar_arrive_tx(&full[s], sb * (with_rho ? 2u : 1u) + eb + bb + gb);
            bulk_g2s(slot, u + tl.tile_off, sb, &full[s]);
            if (with_rho) bulk_g2s_stream(slot + slab_b, rho + tl.tile_off, sb, &full[s]);
            bulk_g2s(slot + 2 * slab_b, a.ent + tl.ent_off, eb, &full[s]);
            bulk_g2s(slot + 2 * slab_b + ent_b, a.blk + tl.blk_off, bb, &full[s]);
            bulk_g2s(slot + 2 * slab_b + ent_b + blk_b, a.gsum + tl.g_off, gb, &full[s]);
        }
        return;
    }

    // ---- consumers
    const int ctid = tid - 32;
    for (int t = blockIdx.x, i = 0; t < a.ntiles; t += gridDim.x, ++i) {
        const int s = i & 1;
        if (!bar_wait(&full[s], (i >> 1) & 1)) atomicExch(s_err, 1);
        consumer_sync();
        if (*s_err) {
            if (ctid == 0) {
                atomicExch(a.error_flag, 1);
                // the other slot may still be receiving a tile: give it a bounded chance to land
                if (t + gridDim.x < a.ntiles) bar_wait(&full[s ^ 1], ((i + 1) >> 1) & 1);
            }
            return;
        }
        unsigned char* slot = smem + s * slot_b;
        const double2* sx = reinterpret_cast<const double2*>(slot);
        const double2* sbase = reinterpret_cast<const double2*>(slot + slab_b);
        const int* ent = reinterpret_cast<const int*>(slot + 2 * slab_b);
        const double* blk = reinterpret_cast<const double*>(slot + 2 * slab_b + ent_b);
        const double* gs = reinterpret_cast<const double*>(slot + 2 * slab_b + ent_b + blk_b);
        const BatchTile tl = *reinterpret_cast<const BatchTile*>(slot + 2 * slab_b + ent_b + blk_b + g_b);
        const int logd = tl.logd, M = tl.M, J = tl.J, M2 = 2 * M, EBA = tl.eba;
        const double* sF = blk;
        const double* nu = blk + logd;
        const double* tcoef = nu + M;
        const double* theta_a = tcoef + M;
        const double* spin = theta_a + J;
        const double* boff = spin + J;
        // expand the tile's entries into this instance's weights
        for (int idx = ctid; idx < tl.nado * M2; idx += kConsumers) {
            const int al = idx / M2, q = idx - al * M2;
            const int* eblk = ent + al * EBA;
            if (q < eblk[3 * J]) {
                const int mt = eblk[3 * J + 1 + M2 + q];
                const int m = mt & 0xff, up = (mt >> 8) & 1, nm = mt >> 16;
                sCslab[idx] = eblk[3 * J + 1 + q];
                sCw[idx] = up ? 1.0 : nu[m] * nm * tcoef[m];
            }
        }
        for (int idx = ctid; idx < tl.nado * J; idx += kConsumers) {
            const int al = idx / J, j = idx - al * J;
            const int* eblk = ent + al * EBA;
            const int m0 = static_cast<int>(boff[j]);
            const double w = nu[m0] * eblk[J + j];
            sDwc[idx] = w * tcoef[m0];
            sDwa[idx] = w * theta_a[j];
        }
        consumer_sync();
        const TileWeights twp{ent, sCslab, sCw, sDwc, sDwa, gs + tl.g_shift, spin, EBA, M2, J};
        const double2* ui = u + tl.inst_off;
        const double2* Td = a.diag + tl.diag_off;
        double2* ot = out + tl.tile_off;
        tile_stage<LOGD, EMAX>(ctid, tl.nado, twp, sx, sbase, Td, sF, ui, ot, alpha, base_kind);
        consumer_sync();  // slot and weights are free again
        if (ctid == 0) bar_arrive(&empty[s]);
    }
}

// ADO blocks of one hierarchy shape (layout at ent_block_ints): per bath, the
// Drude mode's down neighbour apart, then the bath's commutator entries in
// mode order (up neighbour, then the Pade modes' down neighbours).
__global__ void batch_entries_kernel(const int32_t* rows, const int32_t* edges, const int32_t* bath_off, long long H,
                                     int M, int J, int eba, int32_t* blocks)
{
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= H) return;
    int32_t* b = blocks + i * eba;
    int32_t* cslab = b + 3 * J + 1;
    int32_t* cmeta = cslab + 2 * M;
    int q = 0;
    for (int j = 0; j < J; ++j) {
        const int m0 = bath_off[j];
        const int dn0 = edges[i * 2 * M + M + m0];
        b[j] = dn0 < H ? dn0 : -1;
        b[J + j] = rows[i * M + m0];
        b[2 * J + j] = q;
        for (int m = m0; m < bath_off[j + 1]; ++m) {
            const int up = edges[i * 2 * M + m];
            if (up < H) {
                cslab[q] = up;
                cmeta[q] = m | (1 << 8);
                ++q;
            }
            const int dn = edges[i * 2 * M + M + m];
            if (m != m0 && dn < H) {
                cslab[q] = dn;
                cmeta[q] = m | (rows[i * M + m] << 16);
                ++q;
            }
        }
    }
    b[3 * J] = q;
    for (int k = q; k < 2 * M; ++k) {
        cslab[k] = 0;
        cmeta[k] = 0;
    }
    for (int k = 3 * J + 1 + 4 * M; k < eba; ++k) b[k] = 0;
}

// Damping sums sum_j sum_{m in bath j} nu_m n_m of every ADO of one instance.
__global__ void batch_gsum_kernel(const int32_t* rows, const int32_t* bath_off, const double* nu, long long H, int M,
                                  int J, double* g)
{
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= H) return;
    double s = 0.0;
    for (int j = 0; j < J; ++j) {
        double t = 0.0;
        for (int m = bath_off[j]; m < bath_off[j + 1]; ++m) t += nu[m] * rows[i * M + m];
        s += t;
    }
    g[i] = s;
}

// trace[*counter % cap] = sum over instances of Tr(sigma_z(spin) rho_0); then ++*counter.
// One block of 256 threads; fixed summation order, so the result does not depend on timing.
// logd[i] carries bit 8 when instance i keeps Hermitian-packed slabs.
__global__ void batch_obs_kernel(const double2* const* rho0, const int* logd, int count, int spin, double* trace,
                                 int* counter, int cap)
{
    double s = 0.0;
    for (int i = threadIdx.x; i < count; i += blockDim.x) {
        const int lg = logd[i] & 0xff;
        const bool herm = (logd[i] >> 8) & 1;
        const int D = 1 << lg;
        const double2* r0 = rho0[i];
        double v = 0.0;
        for (int r = 0; r < D; ++r) {
            const double d = r0[herm ? herm_index(r, r, lg) : static_cast<long long>(r) * D + r].x;
            v += ((r >> spin) & 1) ? d : -d;
        }
        s += v;
    }
    __shared__ double red[256];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const int t = *counter;
        trace[t % cap] = red[0];
        *counter = t + 1;
    }
}

__global__ void batch_zero_kernel(double2* rho, long long total)
{
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
        rho[i] = make_double2(0.0, 0.0);
}

// rho[pos[i]] = 1 for the n positions pos[] (element d^2 - 1 of each packed instance).
__global__ void batch_init_diag_kernel(const long long* pos, int n, double2* rho)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    rho[pos[i]] = make_double2(1.0, 0.0);
}

}  // namespace

size_t batch_smem_bytes(const BatchArgs& a)
{
    const size_t slab_b = static_cast<size_t>(a.buf_elems) * sizeof(double2);
    const size_t ent_b = static_cast<size_t>(a.max_tile_ados) * a.max_eba * sizeof(int);
    const size_t blk_b = static_cast<size_t>(a.max_blk) * sizeof(double);
    const size_t g_b = static_cast<size_t>((a.max_tile_ados + 3) & ~1) * sizeof(double);
    const size_t slot_b = 2 * slab_b + ent_b + blk_b + g_b + sizeof(BatchTile);
    const size_t TC = static_cast<size_t>(a.max_tile_ados) * 2 * a.max_M;
    const size_t TJ = static_cast<size_t>(a.max_tile_ados) * a.max_J;
    return 2 * slot_b + 48 + TC * (sizeof(double) + sizeof(int)) + 2 * TJ * sizeof(double);
}

using BatchKernel = void (*)(BatchArgs, const double2*, const double2*, double2*, double, int);
// Variants of the stage kernel the autotuner chooses from, per log2 d:
// elements per thread (register tile) and CTAs per SM the register budget
// is sized for.
constexpr int kNumBatchVariants = 3;
constexpr int kMaxBatchLogD = 6;
#define HX_BATCH_VARIANTS(L) \
    {batch_stage_kernel<L, 4, 2>, batch_stage_kernel<L, 2, 2>, batch_stage_kernel<L, 1, 3>}
const BatchKernel kBatchVariants[kMaxBatchLogD][kNumBatchVariants] = {
    HX_BATCH_VARIANTS(1), HX_BATCH_VARIANTS(2), HX_BATCH_VARIANTS(3),
    HX_BATCH_VARIANTS(4), HX_BATCH_VARIANTS(5), HX_BATCH_VARIANTS(6)};
#undef HX_BATCH_VARIANTS

}  // namespace hx

// ---------------------------------------------------------------------------
// Batch object and C ABI
// ---------------------------------------------------------------------------

constexpr int kTraceCap = 256;  // steps of the disorder-average trace buffered on the device

struct hx_batch {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    int count = 0, order = 4, spin = 0, sm_count = 0;
    double dt = 0.0;
    long long total_ados = 0, total_elems = 0;
    std::vector<hx::BatchInst> h_inst;
    // device arena
    // one persistent kernel per Hilbert dimension present, each with its own tiles and shape
    struct Class {
        hx::BatchTile* tiles = nullptr;
        int ntiles = 0, tiles_cap = 0;
        int tile_elems = 2048, variant = 1, grid = 0, max_tile_ados = 1, buf_elems = 0;
        size_t smem = 0;
        long long elems = 0;
    } cls[hx::kMaxBatchLogD + 1];
    int32_t* ent = nullptr;
    double* blk = nullptr;
    double* gsum = nullptr;
    double2* diag = nullptr;
    double2 *rho = nullptr, *ua = nullptr, *ub = nullptr;
    int* error_flag = nullptr;
    double* trace = nullptr;
    int* trace_counter = nullptr;
    int trace_cap = 0;
    double* pinned = nullptr;
    size_t device_bytes = 0;
    // instances with d >= 32 run as internal contexts through the fused and
    // up-term kernels on forked streams of the captured step
    std::vector<hx_ctx*> ctxs;
    std::vector<int> large_of;         // instance -> index in ctxs, or -1 (packed arena)
    // the context instances are spread over kGroups forked streams of the
    // captured step (balanced by state size); each context's up-term and
    // fused launches go to its group's stream
    static constexpr int kGroups = 8;
    int ngroups = 0;
    std::vector<int> group_of;         // context -> group
    std::vector<hx::FusedArgs> fargs;  // per context, error word redirected to the batch's
    cudaStream_t gstream[kGroups] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[kGroups] = {};
    cudaStream_t astream = nullptr;    // packed arena's launches, forked beside the groups
    cudaEvent_t ev_ajoin = nullptr;
    const double2** rho0_ptr = nullptr;  // per instance, for the observable
    int* logd_arr = nullptr;
    int max_M = 0, max_J = 0, max_eba = 0, max_blk = 0;
    // graph of one step
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t steps_done = 0;
    uint64_t launches = 0;
};

namespace {

template <typename T>
int balloc(hx_batch* b, T** p, size_t count)
{
    *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), count * sizeof(T));
    if (e != cudaSuccess) return hx::cuda_fail(e, "cudaMalloc (batch)");
    b->device_bytes += count * sizeof(T);
    return HX_OK;
}

void batch_release(hx_batch* b)
{
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    void* ptrs[] = {b->ent, b->blk, b->gsum, b->diag, b->rho, b->ua, b->ub,
                    b->error_flag, b->trace, b->trace_counter, b->rho0_ptr, b->logd_arr};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    for (auto& c : b->cls)
        if (c.tiles) cudaFree(c.tiles);
    for (int g = 0; g < hx_batch::kGroups; ++g) {
        if (b->gstream[g]) cudaStreamDestroy(b->gstream[g]);
        if (b->ev_join[g]) cudaEventDestroy(b->ev_join[g]);
    }
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->astream) cudaStreamDestroy(b->astream);
    if (b->ev_ajoin) cudaEventDestroy(b->ev_ajoin);
    for (hx_ctx* c : b->ctxs) hx_ctx_destroy(c);
    if (b->pinned) cudaFreeHost(b->pinned);
    if (b->own_stream) cudaStreamDestroy(b->own_stream);
    delete b;
}

hx::BatchArgs batch_args(const hx_batch* b, int lg)
{
    const hx_batch::Class& c = b->cls[lg];
    hx::BatchArgs a{};
    a.tiles = c.tiles;
    a.ent = b->ent;
    a.blk = b->blk;
    a.gsum = b->gsum;
    a.diag = b->diag;
    a.error_flag = b->error_flag;
    a.ntiles = c.ntiles;
    a.buf_elems = c.buf_elems;
    a.max_tile_ados = c.max_tile_ados;
    a.max_M = b->max_M;
    a.max_J = b->max_J;
    a.max_eba = b->max_eba;
    a.max_blk = b->max_blk;
    return a;
}

void drop_graph(hx_batch* b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

// Tile list of class lg (instances with d = 2^lg) for a tile size: instances
// in order, each cut into runs of max(1, tile_elems / d^2) consecutive ADOs.
int set_tile_shape(hx_batch* b, int lg, int tile_elems, int variant)
{
    hx_batch::Class& c = b->cls[lg];
    std::vector<hx::BatchTile> tl;
    int max_ados = 1, buf = 0;
    for (int i = 0; i < b->count; ++i) {
        const hx::BatchInst& in = b->h_inst[i];
        if (in.logd != lg || b->large_of[i] >= 0) continue;
        const int d2 = 1 << (2 * in.logd);
        const int per = std::max(1, tile_elems / d2);
        max_ados = std::max(max_ados, per);
        buf = std::max(buf, per * d2);
        for (int a0 = 0; a0 < in.H; a0 += per) {
            hx::BatchTile t{};
            t.tile_off = in.state_off + static_cast<long long>(a0) * d2;
            t.inst_off = in.state_off;
            t.ent_off = in.ent_off + static_cast<long long>(a0) * in.eba;
            t.diag_off = in.diag_off;
            t.blk_off = in.blk_off;
            t.nado = std::min(per, in.H - a0);
            t.g_shift = a0 & 1;
            t.g_off = in.g_off + a0 - t.g_shift;
            t.g_len = (t.nado + t.g_shift + 1) & ~1;
            t.logd = in.logd;
            t.M = in.M;
            t.J = in.J;
            t.eba = in.eba;
            t.blk_len = in.blk_len;
            tl.push_back(t);
        }
    }
    if (tl.empty()) return HX_OK;
    hx::BatchArgs a = batch_args(b, lg);
    a.max_tile_ados = max_ados;
    a.buf_elems = buf;
    const size_t smem = hx::batch_smem_bytes(a);
    if (smem > 227 * 1024) return fail(HX_ERR_UNSUPPORTED_EXECUTION, "batch tile shape exceeds shared memory");
    int per_sm = 0;
    const hx::BatchKernel fn = hx::kBatchVariants[lg - 1][variant];
    HX_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    HX_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, hx::kThreads, smem));
    if (per_sm < 1) return fail(HX_ERR_UNSUPPORTED_EXECUTION, "batch kernel does not fit on an SM");
    if (static_cast<int>(tl.size()) > c.tiles_cap) {
        if (c.tiles) {
            cudaFree(c.tiles);
            b->device_bytes -= static_cast<size_t>(c.tiles_cap) * sizeof(hx::BatchTile);
        }
        c.tiles = nullptr;
        c.tiles_cap = 0;
        int rc = balloc(b, &c.tiles, tl.size());
        if (rc != HX_OK) return rc;
        c.tiles_cap = static_cast<int>(tl.size());
    }
    HX_CUDA_TRY(cudaMemcpyAsync(c.tiles, tl.data(), tl.size() * sizeof(hx::BatchTile), cudaMemcpyHostToDevice,
                                b->stream));
    HX_CUDA_TRY(cudaStreamSynchronize(b->stream));
    c.ntiles = static_cast<int>(tl.size());
    c.tile_elems = tile_elems;
    c.variant = variant;
    c.max_tile_ados = max_ados;
    c.buf_elems = buf;
    c.smem = smem;
    c.grid = std::max(1, std::min(c.ntiles, per_sm * b->sm_count));
    drop_graph(b);  // the captured step refers to the old tile list and launch shape
    return HX_OK;
}

void launch_class_stage(hx_batch* b, int lg, const double2* u, double2* out, double alpha, int base, cudaStream_t s)
{
    const hx_batch::Class& c = b->cls[lg];
    if (c.ntiles == 0) return;
    hx::kBatchVariants[lg - 1][c.variant]<<<c.grid, hx::kThreads, c.smem, s>>>(batch_args(b, lg), u, b->rho, out,
                                                                             alpha, base);
}

// One stage from state buffer in_id to out_id (0 = rho, 1 = ua, 2 = ub): one
// persistent launch per Hilbert dimension of the packed instances, and the
// up-term and fused launches of every context instance on its group's stream.
void launch_batch_stage(hx_batch* b, int in_id, int out_id, double alpha, int base, cudaStream_t s)
{
    double2* bufs[3] = {b->rho, b->ua, b->ub};
    const bool fork = b->ngroups > 0;
    cudaStream_t sa = fork ? b->astream : s;
    if (fork) {
        cudaEventRecord(b->ev_fork, s);
        cudaStreamWaitEvent(sa, b->ev_fork, 0);
        for (int g = 1; g < b->ngroups; ++g) cudaStreamWaitEvent(b->gstream[g], b->ev_fork, 0);
    }
    for (int lg = 1; lg <= hx::kMaxBatchLogD; ++lg) launch_class_stage(b, lg, bufs[in_id], bufs[out_id], alpha, base, sa);
    for (size_t k = 0; k < b->ctxs.size(); ++k) {
        hx_ctx* c = b->ctxs[k];
        const int g = b->group_of[k];
        cudaStream_t sg = g == 0 ? s : b->gstream[g];
        double2* cb[3] = {c->rho, c->ua, c->ub};
        if (c->up_slots > 0) hx::launch_upterm(hx::upterm_args_of(c), cb[in_id], c->U, sg);
        hx::launch_fused(b->fargs[k], cb[in_id], c->rho, cb[out_id], alpha, base, sg);
    }
    for (int g = 1; g < b->ngroups; ++g) {
        cudaEventRecord(b->ev_join[g], b->gstream[g]);
        cudaStreamWaitEvent(s, b->ev_join[g], 0);
    }
    if (fork) {
        cudaEventRecord(b->ev_ajoin, sa);
        cudaStreamWaitEvent(s, b->ev_ajoin, 0);
    }
}

int kernels_per_stage(const hx_batch* b)
{
    int k = 0;
    for (int lg = 1; lg <= hx::kMaxBatchLogD; ++lg) k += b->cls[lg].ntiles > 0 ? 1 : 0;
    for (const hx_ctx* c : b->ctxs) k += 1 + (c->up_slots > 0 ? 1 : 0);
    return k;
}

// One Horner step (as enqueue_step in hx_ctx.cu) plus the observable.
void enqueue_batch_step(hx_batch* b, cudaStream_t s)
{
    const int m = b->order;
    if (m == 1) {
        // neighbours are read from the input: write ua, then copy back
        launch_batch_stage(b, 0, 1, b->dt, hx::kBaseSelf, s);
        cudaMemcpyAsync(b->rho, b->ua, b->total_elems * sizeof(double2), cudaMemcpyDeviceToDevice, s);
        for (hx_ctx* c : b->ctxs)
            cudaMemcpyAsync(c->rho, c->ua, static_cast<size_t>(c->H) * c->slab_store * sizeof(double2),
                            cudaMemcpyDeviceToDevice, s);
    } else {
        int in = 0;
        for (int st = 1; st <= m; ++st) {
            const double alpha = b->dt / static_cast<double>(m - st + 1);
            const int out = (st == m) ? 0 : 1 + ((st - 1) & 1);
            launch_batch_stage(b, in, out, alpha, st == 1 ? hx::kBaseSelf : hx::kBaseRho, s);
            in = out;
        }
    }
    hx::batch_obs_kernel<<<1, 256, 0, s>>>(b->rho0_ptr, b->logd_arr, b->count, b->spin, b->trace, b->trace_counter,
                                          b->trace_cap);
}

int ensure_graph(hx_batch* b)
{
    if (b->exec) return HX_OK;
    HX_CUDA_TRY(cudaStreamSynchronize(b->stream));
    HX_CUDA_TRY(cudaStreamBeginCapture(b->own_stream, cudaStreamCaptureModeThreadLocal));
    enqueue_batch_step(b, b->own_stream);
    cudaError_t e = cudaStreamEndCapture(b->own_stream, &b->graph);
    if (e != cudaSuccess) return hx::cuda_fail(e, "capture of the batch step");
    HX_CUDA_TRY(cudaGraphInstantiate(&b->exec, b->graph, 0));
    return HX_OK;
}

int batch_check_flag(hx_batch* b)
{
    int flag = 0;
    HX_CUDA_TRY(cudaMemcpyAsync(&flag, b->error_flag, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
    HX_CUDA_TRY(cudaStreamSynchronize(b->stream));
    if (flag) {
        cudaMemsetAsync(b->error_flag, 0, sizeof(int), b->stream);
        return fail(HX_ERR_DEVICE_TIMEOUT, "a device-side wait ran out of its iteration budget");
    }
    return HX_OK;
}

// Streams of the context instances (groups balanced by state size, largest
// first), their fused-kernel arguments and the observable's rho_0 pointers.
int build_context_launches(hx_batch* b)
{
    const int nc = static_cast<int>(b->ctxs.size());
    b->ngroups = std::min(nc, static_cast<int>(hx_batch::kGroups));
    b->group_of.assign(nc, 0);
    std::vector<int> order(nc);
    for (int k = 0; k < nc; ++k) order[k] = k;
    std::sort(order.begin(), order.end(), [&](int x, int y) {
        return b->ctxs[x]->H * b->ctxs[x]->slab_store > b->ctxs[y]->H * b->ctxs[y]->slab_store;
    });
    std::vector<long long> load(std::max(1, b->ngroups), 0);
    for (int k : order) {
        const int g = static_cast<int>(std::min_element(load.begin(), load.end()) - load.begin());
        b->group_of[k] = g;
        load[g] += b->ctxs[k]->H * static_cast<long long>(b->ctxs[k]->slab_store);
    }
    b->fargs.resize(nc);
    for (int k = 0; k < nc; ++k) {
        b->fargs[k] = hx::fused_args_of(b->ctxs[k]);
        b->fargs[k].error_flag = b->error_flag;
        // the kernel's shared-memory limit is raised here, outside any stream capture
        if (!hx::prepare_fused(b->ctxs[k]->logd, b->ctxs[k]->M, b->ctxs[k]->J, b->ctxs[k]->herm ? 1 : 0))
            return fail(HX_ERR_UNSUPPORTED_EXECUTION, "fused kernel tables exceed shared memory");
    }
    for (int g = 1; g < b->ngroups; ++g) {
        HX_CUDA_TRY(cudaStreamCreateWithFlags(&b->gstream[g], cudaStreamNonBlocking));
        HX_CUDA_TRY(cudaEventCreateWithFlags(&b->ev_join[g], cudaEventDisableTiming));
    }
    if (b->ngroups > 0) {
        HX_CUDA_TRY(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
        HX_CUDA_TRY(cudaEventCreateWithFlags(&b->ev_ajoin, cudaEventDisableTiming));
        HX_CUDA_TRY(cudaStreamCreateWithFlags(&b->astream, cudaStreamNonBlocking));
    }
    std::vector<const double2*> rp(b->count);
    std::vector<int> lgs(b->count);
    for (int i = 0; i < b->count; ++i) {
        const int k = b->large_of[i];
        rp[i] = k >= 0 ? b->ctxs[k]->rho : b->rho + b->h_inst[i].state_off;
        lgs[i] = b->h_inst[i].logd | ((k >= 0 && b->ctxs[k]->herm) ? 1 << 8 : 0);
    }
    int rc = HX_OK;
    if ((rc = balloc(b, &b->rho0_ptr, b->count)) || (rc = balloc(b, &b->logd_arr, b->count))) return rc;
    HX_CUDA_TRY(cudaMemcpyAsync(b->rho0_ptr, rp.data(), b->count * sizeof(const double2*), cudaMemcpyHostToDevice,
                                b->stream));
    HX_CUDA_TRY(cudaMemcpyAsync(b->logd_arr, lgs.data(), b->count * sizeof(int), cudaMemcpyHostToDevice, b->stream));
    HX_CUDA_TRY(cudaStreamSynchronize(b->stream));
    return HX_OK;
}


}  // namespace

extern "C" {

int hx_batch_create(const hx_problem* problems, uint32_t count, const hx_batch_options* opt, hx_batch** out)
{
    if (!out) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL batch output");
    *out = nullptr;
    if (!problems || count == 0) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "empty batch");
    const double dt = problems[0].time_step;
    const uint32_t order = problems[0].integration_order;
    for (uint32_t i = 0; i < count; ++i) {
        const hx_problem& p = problems[i];
        const uint32_t d = p.dim;
        if (d < 2 || (d & (d - 1)) != 0 || d > 64)
            return fail(HX_ERR_INVALID_DIMENSION, "batched instances need dim = 2^k with 2 <= dim <= 64");
        if (!p.h_diag) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "h_diag is NULL");
        if (p.h_csr) return fail(HX_ERR_UNSUPPORTED_EXECUTION, "batched instances take diagonal plus flip Hamiltonians");
        if (p.precision != HX_PRECISION_DOUBLE) return fail(HX_ERR_UNSUPPORTED_PRECISION, "batches propagate in double precision");
        if (p.time_step != dt || p.integration_order != order)
            return fail(HX_ERR_INVALID_RUNTIME_OPTION, "all instances of a batch share time_step and integration_order");
        if (!(dt > 0.0) || !std::isfinite(dt)) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "time_step must be positive");
        if (order < 1 || order > 8) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "integration_order must be in 1..8");
        if (p.n_baths == 0 || !p.baths || p.n_baths > 16) return fail(HX_ERR_UNSUPPORTED_BATH, "batched instances need 1..16 baths");
        if (p.max_depth < 1) return fail(HX_ERR_UNSUPPORTED_HIERARCHY, "max_depth must be >= 1");
        if ((p.flags & ~HX_FLAG_FULL_STATE) != 0) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "unknown flags");
        for (uint32_t j = 0; j < p.n_baths; ++j) {
            const hx_bath& bb = p.baths[j];
            if (!bb.coupling_diag || bb.coupling_csr)
                return fail(HX_ERR_UNSUPPORTED_BATH, "batched instances need sigma_z coupling diagonals");
            if (bb.coupling_flip)
                for (uint32_t k = 0; (1u << k) < d; ++k)
                    if (bb.coupling_flip[k] != 0.0)
                        return fail(HX_ERR_UNSUPPORTED_EXECUTION, "batched instances need sigma_z couplings");
            if (hx::pauli_spin(bb.coupling_diag, static_cast<int>(d)) < 0)
                return fail(HX_ERR_UNSUPPORTED_EXECUTION, "batched instances need sigma_z couplings (+-1 by one spin bit)");
        }
    }
    const int spin = opt ? static_cast<int>(opt->observable_spin) : 0;
    for (uint32_t i = 0; i < count; ++i)
        if (spin > 30 || (1u << spin) >= problems[i].dim)
            return fail(HX_ERR_INVALID_RUNTIME_OPTION, "observable_spin is not a spin of every instance");
    const int te = (opt && opt->tile_elems) ? static_cast<int>(opt->tile_elems) : 2048;
    if (te < 64 || te > 8192 || (te & (te - 1)) != 0)
        return fail(HX_ERR_INVALID_RUNTIME_OPTION, "tile_elems must be a power of two in 64..8192");
    if (opt && opt->threads && opt->threads != static_cast<uint32_t>(hx::kConsumers))
        return fail(HX_ERR_INVALID_RUNTIME_OPTION, "the batched stage kernel computes with 256 threads per CTA");

    hx_batch* b = new (std::nothrow) hx_batch();
    if (!b) return fail(HX_ERR_OUT_OF_MEMORY, "host allocation failed");
    auto bail = [&](int rc) {
        batch_release(b);
        return rc;
    };
    cudaGetDevice(&b->device);
    cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, b->device);
    cudaError_t e = cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(hx::cuda_fail(e, "cudaStreamCreate"));
    b->stream = b->own_stream;
    b->count = static_cast<int>(count);
    b->order = static_cast<int>(order);
    b->dt = dt;
    b->spin = spin;

    // instances with d >= 32 whose context takes the fused path run as contexts
    b->large_of.assign(count, -1);
    for (uint32_t i = 0; i < count; ++i) {
        if (problems[i].dim < 32) continue;
        hx_ctx* c = nullptr;
        const int rc = hx_ctx_create(&problems[i], &c);
        if (rc != HX_OK) return bail(rc);
        if (!c->use_fused) {
            hx_ctx_destroy(c);
            continue;
        }
        b->large_of[i] = static_cast<int>(b->ctxs.size());
        b->ctxs.push_back(c);
    }

    // host layout: shapes (modes, depth, modes per bath), per-instance offsets and constants
    struct ShapeInfo {
        long long ent_off, H;
        int M, depth, J, eba;
        std::vector<int32_t> boff;
        std::vector<uint32_t> members;
    };
    std::map<std::vector<int>, ShapeInfo> shapes;
    long long n_ent = 0, n_diag = 0, n_state = 0, n_g = 0;
    std::vector<double> blk;    // kernel constant blocks
    std::vector<double> dsrc;   // per instance: hdiag[d] vdiag[J][d] xi[J] kappa[J] (diagonal-table input)
    std::vector<long long> dsrc_off(count), nu_off(count);
    b->h_inst.resize(count);
    for (uint32_t i = 0; i < count; ++i) {
        const hx_problem& p = problems[i];
        const int J = static_cast<int>(p.n_baths), D = static_cast<int>(p.dim);
        int logd = 0;
        while ((1 << logd) < D) ++logd;
        std::vector<hx::BathConst> bc(J);
        std::vector<int> key;
        int M = 0;
        for (int j = 0; j < J; ++j) {
            const hx_bath& bb = p.baths[j];
            if (!(bb.inverse_temperature > 0.0) || !(bb.damping > 0.0) || !std::isfinite(bb.coupling_strength) ||
                bb.pade_terms > 32 ||
                !hx::bath_constants(bb.inverse_temperature, bb.damping, bb.coupling_strength,
                                    static_cast<int>(bb.pade_terms), bc[j]))
                return bail(fail(HX_ERR_UNSUPPORTED_BATH, "bath coefficients are not finite"));
            bc[j].offset = M;
            M += static_cast<int>(bb.pade_terms) + 1;
            key.push_back(static_cast<int>(bb.pade_terms) + 1);
        }
        if (M > 64) return bail(fail(HX_ERR_UNSUPPORTED_HIERARCHY, "batched instances need at most 64 modes"));
        if (p.max_depth > 32767) return bail(fail(HX_ERR_UNSUPPORTED_HIERARCHY, "hierarchy too deep for a batch"));
        uint64_t H = 0;
        int rc = hx_hierarchy_size(static_cast<uint32_t>(M), p.max_depth, &H);
        if (rc != HX_OK) return bail(rc);
        if (H == 0 || H >= (1ull << 31)) return bail(fail(HX_ERR_UNSUPPORTED_HIERARCHY, "hierarchy size out of range"));
        hx::BatchInst& in = b->h_inst[i];
        in.H = static_cast<int>(H);
        in.M = M;
        in.J = J;
        in.logd = logd;
        in.eba = hx::ent_block_ints(M, J);
        if (b->large_of[i] >= 0) {
            b->total_ados += static_cast<long long>(H);
            continue;
        }
        key.push_back(-static_cast<int>(p.max_depth));
        auto it = shapes.find(key);
        if (it == shapes.end()) {
            ShapeInfo si;
            si.ent_off = n_ent;
            si.H = static_cast<long long>(H);
            si.M = M;
            si.depth = static_cast<int>(p.max_depth);
            si.J = J;
            si.eba = in.eba;
            for (int j = 0; j < J; ++j) si.boff.push_back(bc[j].offset);
            si.boff.push_back(M);
            it = shapes.emplace(key, si).first;
            n_ent += static_cast<long long>(H) * in.eba;
        }
        it->second.members.push_back(i);
        in.ent_off = it->second.ent_off;
        in.diag_off = n_diag;
        n_diag += static_cast<long long>(D) * D;
        in.state_off = n_state;
        n_state += static_cast<long long>(H) * D * D;
        in.g_off = n_g;
        n_g += (static_cast<long long>(H) + 1) & ~1ll;
        // constant block: hflip[logd] nu[M] tcoef[M] theta_a[J] spin[J] bath_off[J+1]
        in.blk_off = static_cast<long long>(blk.size());
        for (int k = 0; k < logd; ++k) blk.push_back(p.h_flip ? p.h_flip[k] : 0.0);
        std::vector<double> nu(M), tc(M);
        for (int j = 0; j < J; ++j)
            for (int k = 0; k <= bc[j].K; ++k) {
                const int m = bc[j].offset + k;
                nu[m] = bc[j].nu[k];
                tc[m] = (k == 0) ? bc[j].theta_c : bc[j].phi[k - 1];
            }
        nu_off[i] = static_cast<long long>(blk.size());
        blk.insert(blk.end(), nu.begin(), nu.end());
        blk.insert(blk.end(), tc.begin(), tc.end());
        for (int j = 0; j < J; ++j) blk.push_back(bc[j].theta_a);
        for (int j = 0; j < J; ++j) blk.push_back(hx::pauli_spin(p.baths[j].coupling_diag, D));
        for (int j = 0; j < J; ++j) blk.push_back(bc[j].offset);
        blk.push_back(M);
        if (blk.size() & 1) blk.push_back(0.0);  // 16-byte aligned blocks
        in.blk_len = static_cast<int>(blk.size() - in.blk_off);
        // diagonal-table input
        dsrc_off[i] = static_cast<long long>(dsrc.size());
        for (int r = 0; r < D; ++r) dsrc.push_back(p.h_diag[r]);
        for (int j = 0; j < J; ++j)
            for (int r = 0; r < D; ++r) dsrc.push_back(p.baths[j].coupling_diag[r]);
        for (int j = 0; j < J; ++j) dsrc.push_back(bc[j].xi);
        for (int j = 0; j < J; ++j) dsrc.push_back(bc[j].counter);
        for (size_t k = in.blk_off; k < blk.size(); ++k)
            if (!std::isfinite(blk[k])) return bail(fail(HX_ERR_INVALID_RUNTIME_OPTION, "instance constants are not finite"));
        for (size_t k = dsrc_off[i]; k < dsrc.size(); ++k)
            if (!std::isfinite(dsrc[k])) return bail(fail(HX_ERR_INVALID_RUNTIME_OPTION, "instance operators are not finite"));
        b->max_M = std::max(b->max_M, M);
        b->max_J = std::max(b->max_J, J);
        b->max_eba = std::max(b->max_eba, in.eba);
        b->max_blk = std::max(b->max_blk, in.blk_len);
        b->total_ados += static_cast<long long>(H);
    }
    b->total_elems = n_state;
    int rc = HX_OK;
    double* ddsrc = nullptr;
    if ((rc = balloc(b, &b->ent, n_ent)) || (rc = balloc(b, &b->blk, blk.size())) ||
        (rc = balloc(b, &b->gsum, n_g + 2)) || (rc = balloc(b, &b->diag, n_diag)) || (rc = balloc(b, &b->rho, n_state)) ||
        (rc = balloc(b, &b->ua, n_state)) || (rc = balloc(b, &b->ub, n_state)) || (rc = balloc(b, &b->error_flag, 1)) ||
        (rc = balloc(b, &b->trace_counter, 1)) || (rc = balloc(b, &b->trace, kTraceCap)))
        return bail(rc);
    b->trace_cap = kTraceCap;
    e = cudaMallocHost(&b->pinned, kTraceCap * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&ddsrc, dsrc.size() * sizeof(double));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->blk, blk.data(), blk.size() * sizeof(double), cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ddsrc, dsrc.data(), dsrc.size() * sizeof(double), cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->gsum, 0, (n_g + 2) * sizeof(double), b->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->error_flag, 0, sizeof(int), b->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->trace_counter, 0, sizeof(int), b->stream);
    if (e == cudaSuccess) {
        // per-instance diagonal coefficient tables
        for (uint32_t i = 0; i < count; ++i) {
            if (b->large_of[i] >= 0) continue;
            const hx::BatchInst& in = b->h_inst[i];
            const int D = 1 << in.logd;
            const double* o = ddsrc + dsrc_off[i];
            hx::launch_diag_table(o, o + D, o + D + in.J * D, o + D + in.J * D + in.J, D, in.J,
                                  b->diag + in.diag_off, b->stream);
        }
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    cudaFree(ddsrc);
    if (e != cudaSuccess) return bail(hx::cuda_fail(e, "batch upload"));

    // ADO blocks per shape (from the device-built reference tables) and the
    // damping sums of every instance of that shape
    for (auto& kv : shapes) {
        const ShapeInfo& si = kv.second;
        const int M = si.M, J = si.J;
        const long long H = si.H;
        int32_t *rows = nullptr, *edges = nullptr, *dboff = nullptr;
        e = cudaMalloc(&rows, static_cast<size_t>(H) * M * sizeof(int32_t));
        if (e == cudaSuccess) e = cudaMalloc(&edges, static_cast<size_t>(H) * 2 * M * sizeof(int32_t));
        if (e == cudaSuccess) e = cudaMalloc(&dboff, (J + 1) * sizeof(int32_t));
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(dboff, si.boff.data(), (J + 1) * sizeof(int32_t), cudaMemcpyHostToDevice, b->stream);
        if (e != cudaSuccess) rc = hx::cuda_fail(e, "batch tables");
        if (rc == HX_OK) rc = hx::build_tables_device(M, si.depth, H, rows, edges, b->stream);
        if (rc == HX_OK) {
            const unsigned grid = static_cast<unsigned>((H + 127) / 128);
            hx::batch_entries_kernel<<<grid, 128, 0, b->stream>>>(rows, edges, dboff, H, M, J, si.eba,
                                                                 b->ent + si.ent_off);
            for (uint32_t i : si.members)
                hx::batch_gsum_kernel<<<grid, 128, 0, b->stream>>>(rows, dboff, b->blk + nu_off[i], H, M, J,
                                                                  b->gsum + b->h_inst[i].g_off);
            e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
            if (e != cudaSuccess) rc = hx::cuda_fail(e, "batch entry blocks");
        }
        cudaFree(rows);
        cudaFree(edges);
        cudaFree(dboff);
        if (rc != HX_OK) return bail(rc);
    }
    // initial state |d-1><d-1| in ADO 0 of every packed instance (contexts set their own)
    std::vector<long long> pos;
    for (uint32_t i = 0; i < count; ++i)
        if (b->large_of[i] < 0) {
            const long long D = 1ll << b->h_inst[i].logd;
            pos.push_back(b->h_inst[i].state_off + D * D - 1);
        }
    if (!pos.empty()) {
        long long* dpos = nullptr;
        e = cudaMalloc(&dpos, pos.size() * sizeof(long long));
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(dpos, pos.data(), pos.size() * sizeof(long long), cudaMemcpyHostToDevice, b->stream);
        if (e == cudaSuccess) {
            hx::batch_zero_kernel<<<148 * 4, 256, 0, b->stream>>>(b->rho, b->total_elems);
            hx::batch_init_diag_kernel<<<static_cast<unsigned>((pos.size() + 127) / 128), 128, 0, b->stream>>>(
                dpos, static_cast<int>(pos.size()), b->rho);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
        cudaFree(dpos);
        if (e != cudaSuccess) return bail(hx::cuda_fail(e, "batch set-up kernels"));
    }

    for (uint32_t i = 0; i < count; ++i)
        if (b->large_of[i] < 0)
            b->cls[b->h_inst[i].logd].elems += static_cast<long long>(b->h_inst[i].H) << (2 * b->h_inst[i].logd);
    // streams and arguments of the context instances, and the observable's pointer table
    if ((rc = build_context_launches(b)) != HX_OK) return bail(rc);
    for (int lg = 1; lg <= hx::kMaxBatchLogD; ++lg)
        if ((rc = set_tile_shape(b, lg, te, 1)) != HX_OK) return bail(rc);
    if (opt && opt->tune) {
        uint32_t a = 0, c = 0;
        if ((rc = hx_batch_tune(b, &a, &c)) != HX_OK) return bail(rc);
    }
    *out = b;
    return HX_OK;
}

void hx_batch_destroy(hx_batch* b) { batch_release(b); }

int hx_batch_set_stream(hx_batch* b, void* stream)
{
    if (!b) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL batch");
    HX_CUDA_TRY(cudaStreamSynchronize(b->stream));
    b->stream = stream ? static_cast<cudaStream_t>(stream) : b->own_stream;
    return HX_OK;
}

int hx_batch_info(const hx_batch* b, hx_batch_stats* info)
{
    if (!b || !info) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL argument");
    info->count = static_cast<uint32_t>(b->count);
    info->total_ados = static_cast<uint64_t>(b->total_ados);
    uint64_t ctx_bytes = 0;
    for (const hx_ctx* c : b->ctxs) ctx_bytes += static_cast<uint64_t>(c->H) * c->slab_store * sizeof(double2);
    info->state_bytes = static_cast<uint64_t>(b->total_elems) * sizeof(double2) + ctx_bytes;
    info->device_bytes = b->device_bytes;
    for (const hx_ctx* c : b->ctxs) info->device_bytes += c->device_bytes;
    info->steps_done = b->steps_done;
    // tile shape of the class with the most elements; tiles summed over classes
    int big = 1;
    uint32_t tiles = 0;
    for (int lg = 1; lg <= hx::kMaxBatchLogD; ++lg) {
        if (b->cls[lg].elems > b->cls[big].elems) big = lg;
        tiles += static_cast<uint32_t>(b->cls[lg].ntiles);
    }
    info->tile_elems = static_cast<uint32_t>(b->cls[big].tile_elems);
    info->threads = static_cast<uint32_t>(hx::kConsumers);
    info->tiles = tiles;
    info->grid = static_cast<uint32_t>(b->cls[big].grid);
    info->kernel_launches = b->launches;
    info->kernels_per_step = static_cast<uint32_t>(b->order * kernels_per_stage(b) + 1);
    return HX_OK;
}

int hx_batch_tune(hx_batch* b, uint32_t* tile_elems, uint32_t* threads)
{
    if (!b) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL batch");
    static const int tiles[] = {512, 1024, 2048, 4096};
    constexpr int nt = static_cast<int>(sizeof(tiles) / sizeof(tiles[0]));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    HX_CUDA_TRY(cudaEventCreate(&e0));
    HX_CUDA_TRY(cudaEventCreate(&e1));
    int rc = HX_OK;
    for (int lg = 1; lg <= hx::kMaxBatchLogD && rc == HX_OK; ++lg) {
        if (b->cls[lg].ntiles == 0) continue;
        float best = 1e30f;
        int bi = -1;
        for (int k = 0; k < nt * hx::kNumBatchVariants; ++k) {
            if (set_tile_shape(b, lg, tiles[k % nt], k / nt) != HX_OK) continue;  // shape does not fit: skip it
            // time stages that read rho and write the scratch buffer ua (the state is untouched)
            launch_class_stage(b, lg, b->rho, b->ua, b->dt, hx::kBaseRho, b->stream);
            cudaEventRecord(e0, b->stream);
            for (int r = 0; r < 3; ++r) launch_class_stage(b, lg, b->rho, b->ua, b->dt, hx::kBaseRho, b->stream);
            cudaEventRecord(e1, b->stream);
            cudaError_t e = cudaEventSynchronize(e1);
            if (e == cudaSuccess) e = cudaGetLastError();
            if (e != cudaSuccess) {
                rc = hx::cuda_fail(e, "autotune launch");
                break;
            }
            b->launches += 4;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best) {
                best = ms;
                bi = k;
            }
        }
        if (rc == HX_OK && bi < 0) rc = fail(HX_ERR_UNSUPPORTED_EXECUTION, "no tile shape fits this batch");
        if (rc == HX_OK) rc = set_tile_shape(b, lg, tiles[bi % nt], bi / nt);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != HX_OK) return rc;
    hx_batch_stats st{};
    hx_batch_info(b, &st);
    if (tile_elems) *tile_elems = st.tile_elems;
    if (threads) *threads = static_cast<uint32_t>(hx::kConsumers);
    return batch_check_flag(b);
}

int hx_batch_step(hx_batch* b, uint64_t nsteps, double* sz_sum_trace)
{
    if (!b) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL batch");
    int rc = ensure_graph(b);
    if (rc != HX_OK) return rc;
    const int cap = b->trace_cap;
    uint64_t done = 0;
    while (done < nsteps) {
        const int chunk = static_cast<int>(std::min<uint64_t>(nsteps - done, cap));
        HX_CUDA_TRY(cudaMemsetAsync(b->trace_counter, 0, sizeof(int), b->stream));
        for (int t = 0; t < chunk; ++t) HX_CUDA_TRY(cudaGraphLaunch(b->exec, b->stream));
        b->launches += static_cast<uint64_t>(chunk) * (b->order * kernels_per_stage(b) + 1);
        if (sz_sum_trace) {
            HX_CUDA_TRY(cudaMemcpyAsync(b->pinned, b->trace, chunk * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
            HX_CUDA_TRY(cudaStreamSynchronize(b->stream));
            std::memcpy(sz_sum_trace + done, b->pinned, chunk * sizeof(double));
        }
        done += chunk;
    }
    b->steps_done += nsteps;
    if (!sz_sum_trace) return HX_OK;
    return batch_check_flag(b);
}

int hx_batch_sync(hx_batch* b)
{
    if (!b) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL batch");
    HX_CUDA_TRY(cudaStreamSynchronize(b->stream));
    return batch_check_flag(b);
}

int hx_batch_read_rho0(hx_batch* b, uint32_t instance, double* out, uint64_t n)
{
    if (!b || !out) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL argument");
    if (instance >= static_cast<uint32_t>(b->count)) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "instance out of range");
    const hx::BatchInst& in = b->h_inst[instance];
    const size_t d2 = size_t(1) << (2 * in.logd);
    if (n < 2 * d2) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "output buffer too small");
    const int k = b->large_of[instance];
    const double2* src = k >= 0 ? b->ctxs[k]->rho : b->rho + in.state_off;
    if (k >= 0 && b->ctxs[k]->herm) {
        std::vector<double2> pk(b->ctxs[k]->slab_store);
        HX_CUDA_TRY(cudaMemcpyAsync(pk.data(), src, pk.size() * sizeof(double2), cudaMemcpyDeviceToHost, b->stream));
        HX_CUDA_TRY(cudaStreamSynchronize(b->stream));
        hx::unpack_herm_host(pk.data(), in.logd, out);
        return batch_check_flag(b);
    }
    HX_CUDA_TRY(cudaMemcpyAsync(out, src, d2 * sizeof(double2), cudaMemcpyDeviceToHost, b->stream));
    HX_CUDA_TRY(cudaStreamSynchronize(b->stream));
    return batch_check_flag(b);
}

}  // extern "C"
