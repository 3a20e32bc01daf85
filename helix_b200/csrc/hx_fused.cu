// Multi-CTA fused stage kernels for d = 32 and d = 64 (FP64), on full or on
// Hermitian-packed slabs.
//
// Same mathematics as stage_kernel (hx_stage.cu): one launch evaluates
// out_n = base_n + alpha L(u)_n for every ADO n, L being the reference
// right-hand side (getdRhoSparse, src/liouville.cu:749-869) for diagonal
// couplings.  Layout chosen for latency hiding on B200:
//
//  * one CTA per ADO, 256 threads, one slab of shared memory, two or more
//    CTAs resident per SM so their load / compute phases overlap;
//  * the slab arrives by one TMA bulk copy (evict_last in L2 for slabs below
//    the top tier, which are re-read as neighbours);
//  * thread t owns elements e_k = t + 256 k, all accumulated in registers;
//    step A (diagonal + transverse field) runs in chunks of 4 elements so
//    two row-flip bits are register moves;
//  * once step A has read the slab, a second TMA copy streams the Horner base
//    rho_n into the same buffer (evict_first) while step B gathers the
//    neighbour terms, so the base read overlaps the neighbour loads;
//  * the ADO-independent diagonal table is read through L1/L2;
//  * neighbour entries are consumed two at a time, 8 independent element
//    loads per thread per batch;
//  * the up term of tier L-1 (neighbours in the top tier L) is not gathered
//    here: upterm_kernel (hx_upterm.cu) sums it tile by tile beforehand and
//    this kernel adds the result.

#include <cuda_runtime.h>

#include <cstdint>

#include "hx_internal.h"

namespace hx {

namespace {

__device__ __forceinline__ uint32_t s_addr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ uint64_t pol_last()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ uint64_t pol_normal()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ double2 ldg_hint(const double2* p, uint64_t pol)
{
    double2 v;
    asm volatile("ld.global.nc.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(v.x), "=d"(v.y) : "l"(p), "l"(pol));
    return v;
}

__device__ __forceinline__ double2 ldg_stream(const double2* p)
{
    double2 v;
    asm volatile("ld.global.cs.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
    return v;
}

__device__ __forceinline__ void stg_stream(double2* p, double2 v)
{
    asm volatile("st.global.cs.v2.f64 [%0], {%1, %2};" ::"l"(p), "d"(v.x), "d"(v.y) : "memory");
}

constexpr uint32_t kSpinLimit = 1u << 20;

__device__ __forceinline__ uint64_t pol_first()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar, uint64_t pol)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(s_addr(bar)), "r"(bytes) : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::
            "r"(s_addr(dst)),
        "l"(src), "r"(bytes), "r"(s_addr(bar)), "l"(pol)
        : "memory");
}

// Start pulling `bytes` at src into L2 (no completion to wait for).
__device__ __forceinline__ void prefetch_l2(const void* src, uint32_t bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

// Bounded wait on an mbarrier phase; false if the poll budget ran out.
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity)
{
    for (uint32_t i = 0; i < kSpinLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(s_addr(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// The stage of ADO n: out_n = base_n + alpha L(u)_n (one CTA of 256 threads).
template <int LOGD>
__device__ __forceinline__ void fused_ado(const FusedArgs& a, long long n, const double2* __restrict__ u,
                                          const double2* rho, double2* out, double alpha, int base_kind)
{
    constexpr int D = 1 << LOGD, D2 = D * D, T = 256;
    constexpr int E = D2 / T;         // elements per thread
    constexpr int CH = 4;             // chunk: register flips of 2 row bits, load batches
    constexpr int RSTEP = 8 - LOGD;   // k advances the row by 2^RSTEP
    static_assert(E % CH == 0, "chunk must divide the elements per thread");
    extern __shared__ __align__(128) unsigned char smem[];
    double2* slab = reinterpret_cast<double2*>(smem);  // own slab, then the rho slab
    uint64_t* bar = reinterpret_cast<uint64_t*>(slab + D2);
    double* sV = reinterpret_cast<double*>(bar + 2);  // [J][D]
    double* sH = sV + a.J * D;                        // [LOGD]
    double* sWc = sH + LOGD;                          // [2M]
    double* sWa = sWc + 2 * a.M;                      // [2M]
    int* sSlab = reinterpret_cast<int*>(sWa + 2 * a.M);
    int* sBath = sSlab + 2 * a.M;

    const int tid = threadIdx.x;
    const uint64_t pk = pol_last(), pn = pol_normal();
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(s_addr(&bar[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(s_addr(&bar[1])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) bulk_g2s(slab, u + n * D2, D2 * sizeof(double2), &bar[0], a.ado_keep[n] ? pk : pn);
    const int Q = a.ent_count[n];
    for (int i = tid; i < a.J * D; i += T) sV[i] = a.vdiag[i];
    if (tid < LOGD) sH[tid] = a.hflip[tid];
    for (int q = tid; q < Q; q += T) {
        const long long src = n * 2 * a.M + q;
        sSlab[q] = a.ent_slab[src];
        sBath[q] = a.ent_bath[src];
        sWc[q] = a.ent_wc[src];
        sWa[q] = a.ent_wa[src];
    }
    const double g = a.gsum[n];
    const int slot = a.slot ? a.slot[n] : -1;
    __syncthreads();
    if (__syncthreads_or(!bar_wait(&bar[0], 0))) {
        if (tid == 0) atomicExch(a.error_flag, 1);
        return;
    }

    const int c = tid & (D - 1);
    const int r0 = tid >> LOGD;
    double2 acc[E];

    // ---- step A: diagonal (table in L1/L2) and transverse field (shared memory)
#pragma unroll
    for (int k0 = 0; k0 < E; k0 += CH) {
        double2 x[CH], t[CH];
#pragma unroll
        for (int kk = 0; kk < CH; ++kk) {
            x[kk] = slab[tid + T * (k0 + kk)];
            t[kk] = __ldg(a.diag + tid + T * (k0 + kk));
        }
#pragma unroll
        for (int kk = 0; kk < CH; ++kk) {
            const int e = tid + T * (k0 + kk);
            double hr = 0.0, hi = 0.0;
#pragma unroll
            for (int i = 0; i < LOGD; ++i) {
                const double h = sH[i];
                double2 rowp;
                if (i >= RSTEP && i < RSTEP + 2) rowp = x[kk ^ (1 << (i - RSTEP))];
                else rowp = slab[e ^ (D << i)];
                const double2 colp = slab[e ^ (1 << i)];
                hr += h * (rowp.x - colp.x);
                hi += h * (rowp.y - colp.y);
            }
            const double tr = t[kk].x - g;
            acc[k0 + kk].x = tr * x[kk].x - t[kk].y * x[kk].y + hi;
            acc[k0 + kk].y = tr * x[kk].y + t[kk].y * x[kk].x - hr;
        }
    }

    // ---- the own slab is no longer needed (except as the stage-1 base): stream rho into the same buffer
    __syncthreads();
    if (base_kind == kBaseRho && tid == 0)
        bulk_g2s(slab, rho + n * D2, D2 * sizeof(double2), &bar[1], pol_first());

    // ---- step B: neighbour entries, two at a time, CH elements per load batch
    const double2* ubase = u + tid;
    int q = 0;
    for (; q + 1 < Q; q += 2) {
        const int jb0 = sBath[q], jb1 = sBath[q + 1];
        const int j0 = jb0 & 0xffff, j1 = jb1 & 0xffff;
        const uint64_t p0 = (jb0 >> 16) ? pk : pn, p1 = (jb1 >> 16) ? pk : pn;
        const double wc0 = sWc[q], wa0 = sWa[q], wc1 = sWc[q + 1], wa1 = sWa[q + 1];
        const double vc0 = sV[j0 * D + c], vc1 = sV[j1 * D + c];
        const double2* s0 = ubase + static_cast<long long>(sSlab[q]) * D2;
        const double2* s1 = ubase + static_cast<long long>(sSlab[q + 1]) * D2;
#pragma unroll
        for (int k0 = 0; k0 < E; k0 += CH) {
            double2 y0[CH], y1[CH];
#pragma unroll
            for (int kk = 0; kk < CH; ++kk) {
                const int r = r0 + ((k0 + kk) << RSTEP);
                const double vr0 = sV[j0 * D + r], vr1 = sV[j1 * D + r];
                y0[kk] = make_double2(0.0, 0.0);
                y1[kk] = make_double2(0.0, 0.0);
                if ((vr0 + vc0) * wa0 != 0.0 || (vr0 - vc0) * wc0 != 0.0) y0[kk] = ldg_hint(s0 + T * (k0 + kk), p0);
                if ((vr1 + vc1) * wa1 != 0.0 || (vr1 - vc1) * wc1 != 0.0) y1[kk] = ldg_hint(s1 + T * (k0 + kk), p1);
            }
#pragma unroll
            for (int kk = 0; kk < CH; ++kk) {
                const int r = r0 + ((k0 + kk) << RSTEP);
                const double vr0 = sV[j0 * D + r], vr1 = sV[j1 * D + r];
                const double ar0 = -(vr0 + vc0) * wa0, ai0 = -(vr0 - vc0) * wc0;
                const double ar1 = -(vr1 + vc1) * wa1, ai1 = -(vr1 - vc1) * wc1;
                acc[k0 + kk].x += ar0 * y0[kk].x - ai0 * y0[kk].y + ar1 * y1[kk].x - ai1 * y1[kk].y;
                acc[k0 + kk].y += ar0 * y0[kk].y + ai0 * y0[kk].x + ar1 * y1[kk].y + ai1 * y1[kk].x;
            }
        }
    }
    if (q < Q) {
        const int jb0 = sBath[q];
        const int j0 = jb0 & 0xffff;
        const uint64_t p0 = (jb0 >> 16) ? pk : pn;
        const double wc0 = sWc[q], wa0 = sWa[q];
        const double vc0 = sV[j0 * D + c];
        const double2* s0 = ubase + static_cast<long long>(sSlab[q]) * D2;
#pragma unroll
        for (int k0 = 0; k0 < E; k0 += CH) {
            double2 y0[CH];
#pragma unroll
            for (int kk = 0; kk < CH; ++kk) {
                const int r = r0 + ((k0 + kk) << RSTEP);
                const double vr0 = sV[j0 * D + r];
                y0[kk] = make_double2(0.0, 0.0);
                if ((vr0 + vc0) * wa0 != 0.0 || (vr0 - vc0) * wc0 != 0.0) y0[kk] = ldg_hint(s0 + T * (k0 + kk), p0);
            }
#pragma unroll
            for (int kk = 0; kk < CH; ++kk) {
                const int r = r0 + ((k0 + kk) << RSTEP);
                const double vr0 = sV[j0 * D + r];
                const double ar0 = -(vr0 + vc0) * wa0, ai0 = -(vr0 - vc0) * wc0;
                acc[k0 + kk].x += ar0 * y0[kk].x - ai0 * y0[kk].y;
                acc[k0 + kk].y += ar0 * y0[kk].y + ai0 * y0[kk].x;
            }
        }
    }
    // ---- up term of tier L-1 (neighbours in the top tier), summed by upterm_kernel
    if (slot >= 0) {
        const double2* Un = a.U + static_cast<long long>(slot) * D2 + tid;
#pragma unroll
        for (int k = 0; k < E; ++k) {
            const double2 w = ldg_stream(Un + T * k);
            acc[k].x += w.x;
            acc[k].y += w.y;
        }
    }

    // ---- Horner epilogue: out = base + alpha * L(u)
    if (base_kind == kBaseRho && __syncthreads_or(!bar_wait(&bar[1], 0))) {
        if (tid == 0) atomicExch(a.error_flag, 1);
        return;
    }
    double2* out_n = out + n * D2 + tid;
#pragma unroll
    for (int k = 0; k < E; ++k) {
        const double2 b = (base_kind == kBaseZero) ? make_double2(0.0, 0.0) : slab[tid + T * k];
        stg_stream(out_n + T * k, make_double2(b.x + alpha * acc[k].x, b.y + alpha * acc[k].y));
    }
}

template <int LOGD, int MINB>
__global__ void __launch_bounds__(256, MINB)
    fused_kernel(FusedArgs a, const double2* __restrict__ u, const double2* rho, double2* out, double alpha,
                 int base_kind)
{
    const long long n = a.order ? static_cast<long long>(a.order[blockIdx.x]) : static_cast<long long>(blockIdx.x);
    fused_ado<LOGD>(a, n, u, rho, out, alpha, base_kind);
}

// ---------------------------------------------------------------------------
// Hermitian-packed variant.  Slabs, the Horner base, neighbours, up terms,
// the diagonal table and the output are packed upper triangles (herm_index
// in hx_internal.h), so every stream moves d(d+1)/2 elements instead of d^2.
// Thread t owns packed elements t + T k; a warp's 32 elements are
// consecutive in the packed slab, so neighbour, up-term, base and output
// accesses coalesce, and they are runs of consecutive columns of at most two
// matrix rows.
//
// The CTA unpacks its own slab into a full d x d copy in shared memory for
// the transverse-field flips, element (r, c) in slot r d + (c ^ (r & 7)).
// With that swizzle every flip is one XOR of the slot with a constant
// (row bit b: d 2^b, plus 2^b when b < 3; column bit b: 2^b), and the
// accesses stay free of bank conflicts: a run of consecutive columns of one
// row, its row flips and its column flips each cover eight distinct
// 16-byte bank groups per quarter-warp, and so do the mirrored writes (c, r)
// of the unpack, one column of consecutive rows.  With PAULI every coupling
// operator is sigma_z of one spin: v_r = +1 or -1 from a bit of r, and of
// [V, X] and {V, X} exactly one is nonzero at each element.
template <int LOGD> struct HermShape;
template <> struct HermShape<5> { static constexpr int T = 192, MINB = 4; };  // 528 elements: 3 per thread
template <> struct HermShape<6> { static constexpr int T = 416, MINB = 2; };  // 2080 elements: 5 per thread

constexpr unsigned kPrefetchAhead = 148;  // CTAs per resident wave per unit of HermShape::MINB

template <int LOGD>
__device__ __forceinline__ int herm_slot(int r, int c)
{
    return (r << LOGD) | (c ^ (r & 7));
}

template <int LOGD, bool PAULI>
__device__ __forceinline__ void herm_ado(const FusedArgs& a, long long n, const double2* __restrict__ u,
                                         const double2* rho, double2* out, double alpha, int base_kind)
{
    constexpr int D = 1 << LOGD, HALF = D / 2, P = HALF * (D + 1);
    constexpr int T = HermShape<LOGD>::T, E = (P + T - 1) / T;
    constexpr bool kExact = (P % T) == 0;
    extern __shared__ __align__(128) unsigned char smem[];
    double2* full = reinterpret_cast<double2*>(smem);  // [D * D] own slab, unpacked and swizzled
    double2* pk = full + D * D;                         // [P] own packed slab, then the packed rho slab
    uint64_t* bar = reinterpret_cast<uint64_t*>(pk + P);
    double* sV = reinterpret_cast<double*>(bar + 2);   // [J][D] (general couplings)
    double* sH = sV + a.J * D;                          // [LOGD]
    double* sWc = sH + LOGD;                            // [2M]
    double* sWa = sWc + 2 * a.M;                        // [2M]
    int* sSlab = reinterpret_cast<int*>(sWa + 2 * a.M);
    int* sBath = sSlab + 2 * a.M;
    int* sBit = sBath + 2 * a.M;                        // [J] (PAULI)

    const int tid = threadIdx.x;
    const uint64_t pkeep = pol_last(), pn = pol_normal();
    // thread 0 alone owns the two mbarriers (init, copies, waits); the others
    // learn of a completed copy from the block barrier that follows its wait
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(s_addr(&bar[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(s_addr(&bar[1])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        bulk_g2s(pk, u + n * P, P * sizeof(double2), &bar[0], a.ado_keep[n] ? pkeep : pn);
    }
    const int Q = a.ent_count[n];
    if (PAULI) {
        if (tid < a.J) sBit[tid] = a.vbit[tid];
    } else {
        for (int i = tid; i < a.J * D; i += T) sV[i] = a.vdiag[i];
    }
    if (tid < LOGD) sH[tid] = a.hflip[tid];
    for (int q = tid; q < Q; q += T) {
        const long long src = n * 2 * a.M + q;
        sSlab[q] = a.ent_slab[src];
        sBath[q] = a.ent_bath[src];
        sWc[q] = a.ent_wc[src];
        sWa[q] = a.ent_wa[src];
    }
    const double g = a.gsum[n];
    const int slot = a.slot ? a.slot[n] : -1;
    // one barrier publishes the tables above and the arrival of the slab
    if (__syncthreads_or(tid == 0 && !bar_wait(&bar[0], 0))) {
        if (tid == 0) atomicExch(a.error_flag, 1);
        return;
    }

    // ---- unpack the own slab: (r, c) and its mirror (c, r) = conj
    int rc[E];
#pragma unroll
    for (int k = 0; k < E; ++k) {
        const int i = tid + T * k;
        int r = 0, c = 0;
        if (kExact || i < P) {
            herm_coords(i, LOGD, r, c);
            const double2 v = pk[i];
            full[herm_slot<LOGD>(r, c)] = v;
            if (r != c) full[herm_slot<LOGD>(c, r)] = make_double2(v.x, -v.y);
        }
        rc[k] = (r << 8) | c;
    }
    __syncthreads();
    // the packed copy is still the stage-1 base; otherwise stream rho_n into it
    if (base_kind == kBaseRho && tid == 0) bulk_g2s(pk, rho + n * P, P * sizeof(double2), &bar[1], pol_first());

    // ---- step A: diagonal (packed table) and transverse field (unpacked slab)
    double2 acc[E];
#pragma unroll
    for (int k = 0; k < E; ++k) {
        const int i = tid + T * k;
        acc[k] = make_double2(0.0, 0.0);
        if (!kExact && i >= P) continue;
        const int sl = herm_slot<LOGD>(rc[k] >> 8, rc[k] & 255);
        const double2 x = full[sl];
        const double2 t = __ldg(a.diag + i);
        double hr = 0.0, hi = 0.0;
#pragma unroll
        for (int b = 0; b < LOGD; ++b) {
            const double h = sH[b];
            const double2 rowp = full[sl ^ ((1 << b) << LOGD) ^ (b < 3 ? (1 << b) : 0)];
            const double2 colp = full[sl ^ (1 << b)];
            hr += h * (rowp.x - colp.x);
            hi += h * (rowp.y - colp.y);
        }
        const double tr = t.x - g;
        acc[k].x = tr * x.x - t.y * x.y + hi;
        acc[k].y = tr * x.y + t.y * x.x - hr;
    }

    // ---- step B: neighbour entries, E loads in flight per thread
    const double2* ubase = u + tid;
    for (int q = 0; q < Q; ++q) {
        const int jb = sBath[q];
        const int j = jb & 0xffff;
        const uint64_t pol = (jb >> 16) ? pkeep : pn;
        const double wc = sWc[q], wa = sWa[q];
        const double2* src = ubase + static_cast<long long>(sSlab[q]) * P;
        double2 y[E];
        if (PAULI) {
            // v = +-1 from bit `bit`: equal bits of r and c -> only {V, X} = +-2 X;
            // different bits -> only [V, X] = +-2 X (sign + when bit r is set)
            const int bit = sBit[j];
            const bool need_same = wa != 0.0, need_diff = wc != 0.0;
#pragma unroll
            for (int k = 0; k < E; ++k) {
                const int br = (rc[k] >> (8 + bit)) & 1, bc = (rc[k] >> bit) & 1;
                y[k] = make_double2(0.0, 0.0);
                if ((kExact || tid + T * k < P) && (br == bc ? need_same : need_diff))
                    y[k] = ldg_hint(src + T * k, pol);
            }
            const double a2 = 2.0 * wa, c2 = 2.0 * wc;
#pragma unroll
            for (int k = 0; k < E; ++k) {
                const int br = (rc[k] >> (8 + bit)) & 1, bc = (rc[k] >> bit) & 1;
                const bool same = br == bc;
                // -(vr + vc) wa {V,.} term (real weight) or -i (vr - vc) wc [V,.] term
                const double w = same ? (br ? -a2 : a2) : (br ? -c2 : c2);
                const double px = same ? y[k].x : -y[k].y;
                const double py = same ? y[k].y : y[k].x;
                acc[k].x += w * px;
                acc[k].y += w * py;
            }
        } else {
            const double* vj = sV + j * D;
#pragma unroll
            for (int k = 0; k < E; ++k) {
                const double vr = vj[rc[k] >> 8], vc = vj[rc[k] & 255];
                y[k] = make_double2(0.0, 0.0);
                if ((kExact || tid + T * k < P) && ((vr + vc) * wa != 0.0 || (vr - vc) * wc != 0.0))
                    y[k] = ldg_hint(src + T * k, pol);
            }
#pragma unroll
            for (int k = 0; k < E; ++k) {
                const double vr = vj[rc[k] >> 8], vc = vj[rc[k] & 255];
                const double ar = -(vr + vc) * wa, ai = -(vr - vc) * wc;
                acc[k].x += ar * y[k].x - ai * y[k].y;
                acc[k].y += ar * y[k].y + ai * y[k].x;
            }
        }
    }
    // ---- up term of tier L-1, summed by upterm_kernel
    if (slot >= 0) {
        const double2* Un = a.U + static_cast<long long>(slot) * P + tid;
#pragma unroll
        for (int k = 0; k < E; ++k) {
            if (!kExact && tid + T * k >= P) continue;
            const double2 w = ldg_stream(Un + T * k);
            acc[k].x += w.x;
            acc[k].y += w.y;
        }
    }

    // ---- Horner epilogue
    if (base_kind == kBaseRho && __syncthreads_or(tid == 0 && !bar_wait(&bar[1], 0))) {
        if (tid == 0) atomicExch(a.error_flag, 1);
        return;
    }
    double2* out_n = out + n * P + tid;
#pragma unroll
    for (int k = 0; k < E; ++k) {
        if (!kExact && tid + T * k >= P) continue;
        const double2 b = (base_kind == kBaseZero) ? make_double2(0.0, 0.0) : pk[tid + T * k];
        stg_stream(out_n + T * k, make_double2(b.x + alpha * acc[k].x, b.y + alpha * acc[k].y));
    }
}

template <int LOGD, bool PAULI>
__global__ void __launch_bounds__(HermShape<LOGD>::T, HermShape<LOGD>::MINB)
    herm_kernel(FusedArgs a, const double2* __restrict__ u, const double2* rho, double2* out, double alpha,
                int base_kind)
{
    const long long n = a.order ? static_cast<long long>(a.order[blockIdx.x]) : static_cast<long long>(blockIdx.x);
    // The CTA that starts one resident wave later (MINB CTAs on each of 148
    // SMs) finds its slab and its Horner base in L2 instead of waiting on DRAM.
    constexpr unsigned ahead = kPrefetchAhead * HermShape<LOGD>::MINB;
    if (threadIdx.x == 0 && blockIdx.x + ahead < gridDim.x) {
        constexpr uint32_t bytes = (1u << (LOGD - 1)) * ((1u << LOGD) + 1) * sizeof(double2);
        const long long m = a.order ? a.order[blockIdx.x + ahead] : blockIdx.x + ahead;
        prefetch_l2(u + m * (bytes / sizeof(double2)), bytes);
        if (base_kind == kBaseRho) prefetch_l2(rho + m * (bytes / sizeof(double2)), bytes);
    }
    herm_ado<LOGD, PAULI>(a, n, u, rho, out, alpha, base_kind);
}

// Shared memory of herm_kernel (the operator table sV is reserved in both
// forms; the PAULI form leaves it unused).
template <int LOGD>
size_t herm_smem(int M, int J)
{
    const size_t D = size_t(1) << LOGD;
    const size_t P = (D / 2) * (D + 1);
    return (D * D + P) * sizeof(double2) + 16 + sizeof(double) * (J * D + LOGD + 4 * M) +
           sizeof(int) * (4 * M + J);
}

template <int LOGD, bool PAULI>
bool prepare_herm_t(int M, int J)
{
    const size_t smem = herm_smem<LOGD>(M, J);
    if (smem > 227 * 1024) return false;
    static size_t configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && configured[dev] < smem) {
        if (cudaFuncSetAttribute(herm_kernel<LOGD, PAULI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)) != cudaSuccess)
            return false;
        configured[dev] = smem;
    }
    return true;
}

template <int LOGD>
bool prepare_herm(int M, int J)
{
    return prepare_herm_t<LOGD, true>(M, J) && prepare_herm_t<LOGD, false>(M, J);
}

template <int LOGD>
bool launch_herm(const FusedArgs& a, const double2* u, const double2* rho, double2* out, double alpha, int base,
                 cudaStream_t s)
{
    if (!prepare_herm<LOGD>(a.M, a.J)) return false;
    const size_t smem = herm_smem<LOGD>(a.M, a.J);
    const unsigned grid = static_cast<unsigned>(a.H);
    if (a.pauli)
        herm_kernel<LOGD, true><<<grid, HermShape<LOGD>::T, smem, s>>>(a, u, rho, out, alpha, base);
    else
        herm_kernel<LOGD, false><<<grid, HermShape<LOGD>::T, smem, s>>>(a, u, rho, out, alpha, base);
    return true;
}

template <int LOGD>
size_t fused_smem(int M, int J)
{
    const size_t D = size_t(1) << LOGD;
    return D * D * sizeof(double2) + 16 + sizeof(double) * (J * D + LOGD + 4 * M) + sizeof(int) * 4 * M;
}

// Raise the kernel's dynamic shared-memory limit to what (M, J) needs, once
// per device (a function attribute; must not happen during stream capture).
template <int LOGD, int MINB>
bool prepare3(int M, int J)
{
    const size_t smem = fused_smem<LOGD>(M, J);
    if (smem > 227 * 1024) return false;
    static size_t configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && configured[dev] < smem) {
        if (cudaFuncSetAttribute(fused_kernel<LOGD, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)) != cudaSuccess)
            return false;
        configured[dev] = smem;
    }
    return true;
}

template <int LOGD, int MINB>
bool launch3(const FusedArgs& a, const double2* u, const double2* rho, double2* out, double alpha, int base,
             cudaStream_t s)
{
    const size_t smem = fused_smem<LOGD>(a.M, a.J);
    if (!prepare3<LOGD, MINB>(a.M, a.J)) return false;
    fused_kernel<LOGD, MINB><<<static_cast<unsigned>(a.H), 256, smem, s>>>(a, u, rho, out, alpha, base);
    return true;
}

// Per-ADO neighbour entries, grouped by bath: for each mode m of bath j,
//   up present, below the top tier: (slab n+e_m, j, w_comm = 1, w_anti = 0)
//   down present: (slab n-e_m, j, w_comm = a_{n,m},  w_anti = b_{n,j} if m is the Drude mode else 0)
__global__ void entries_kernel(const int32_t* rows, const int32_t* edges, const double* acoef, const double* bcoef,
                               const int32_t* bath_off, long long H, int M, int J, int top_tier, int* count,
                               int32_t* slab, int32_t* bath, double* wc, double* wa, int8_t* keep)
{
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= H) return;
    auto tier_of = [&](long long a) {
        int t = 0;
        for (int m = 0; m < M; ++m) t += rows[a * M + m];
        return t;
    };
    const int tier = tier_of(i);
    keep[i] = tier < top_tier ? 1 : 0;
    int q = 0;
    const long long o = i * 2 * M;
    for (int j = 0; j < J; ++j) {
        for (int m = bath_off[j]; m < bath_off[j + 1]; ++m) {
            const int up = edges[i * 2 * M + m];
            // up neighbours in the top tier are summed by upterm_kernel (hx_upterm.cu)
            if (up < H && tier + 1 < top_tier) {
                slab[o + q] = up;
                bath[o + q] = j | (1 << 16);
                wc[o + q] = 1.0;
                wa[o + q] = 0.0;
                ++q;
            }
            const int dn = edges[i * 2 * M + M + m];
            if (dn < H) {
                slab[o + q] = dn;
                bath[o + q] = j | (1 << 16);  // down neighbours are below the top tier
                wc[o + q] = acoef[i * M + m];
                wa[o + q] = (m == bath_off[j]) ? bcoef[i * J + j] : 0.0;
                ++q;
            }
        }
    }
    count[i] = q;
}

// T[r][c] = -sum_j xi_j (v_r - v_c)^2 - i[(E_r - E_c) + sum_j kappa_j (v_r - v_c)(v_r + v_c)]
__global__ void diag_table_kernel(const double* hdiag, const double* vdiag, const double* xi, const double* kappa,
                                  int D, int J, double2* T)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= D * D) return;
    const int r = e / D, c = e % D;
    double re = 0.0, im = -(hdiag[r] - hdiag[c]);
    for (int j = 0; j < J; ++j) {
        const double vr = vdiag[j * D + r], vc = vdiag[j * D + c];
        const double del = vr - vc, sig = vr + vc;
        re -= xi[j] * del * del;
        im -= kappa[j] * del * sig;
    }
    T[e] = make_double2(re, im);
}

}  // namespace

bool launch_fused(const FusedArgs& a, const double2* u, const double2* rho, double2* out, double alpha,
                   int base_kind, cudaStream_t s)
{
    if (a.herm) {
        switch (a.logd) {
        case 5: return launch_herm<5>(a, u, rho, out, alpha, base_kind, s);
        case 6: return launch_herm<6>(a, u, rho, out, alpha, base_kind, s);
        default: return false;
        }
    }
    switch (a.logd) {
    case 5: return launch3<5, 3>(a, u, rho, out, alpha, base_kind, s);
    case 6: return launch3<6, 2>(a, u, rho, out, alpha, base_kind, s);
    default: return false;
    }
}

bool prepare_fused(int logd, int M, int J, int herm)
{
    switch (logd) {
    case 5: return herm ? prepare_herm<5>(M, J) : prepare3<5, 3>(M, J);
    case 6: return herm ? prepare_herm<6>(M, J) : prepare3<6, 2>(M, J);
    default: return false;
    }
}

bool fused_supported(int logd, int M, int J, int herm)
{
    if (logd == 5) return (herm ? herm_smem<5>(M, J) : fused_smem<5>(M, J)) <= 227 * 1024;
    if (logd == 6) return (herm ? herm_smem<6>(M, J) : fused_smem<6>(M, J)) <= 227 * 1024;
    return false;
}

void launch_entries(const int32_t* rows, const int32_t* edges, const double* acoef, const double* bcoef,
                    const int32_t* bath_off, long long H, int M, int J, int max_depth, int* count, int32_t* slab,
                    int32_t* bath, double* wc, double* wa, int8_t* keep, cudaStream_t s)
{
    if (H <= 0) return;
    const int block = 128;
    entries_kernel<<<static_cast<unsigned>((H + block - 1) / block), block, 0, s>>>(
        rows, edges, acoef, bcoef, bath_off, H, M, J, max_depth - 1, count, slab, bath, wc, wa, keep);
}

void launch_diag_table(const double* hdiag, const double* vdiag, const double* xi, const double* kappa, int D, int J,
                       double2* T, cudaStream_t s)
{
    const int n = D * D;
    diag_table_kernel<<<(n + 255) / 256, 256, 0, s>>>(hdiag, vdiag, xi, kappa, D, J, T);
}

}  // namespace hx
