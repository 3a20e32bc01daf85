// Stage kernels for Hilbert dimension 128 <= d <= 1024 with diagonal couplings,
// in double precision (the plain propagator) or in single precision with
// complex64 storage (the mixed-precision propagator, whose tier-0 ADO runs in
// double precision in ado0_kernel).
//
// Mathematics as in fused_kernel (hx_fused.cu): out_n = base_n + alpha L(u)_n
// with L the reference right-hand side (getdRhoSparse, src/liouville.cu:749-869)
// for diagonal couplings V_j and H = diag(E) + sum_i h_i sigma_x(i).  A slab of
// d = 256 is 1 MB in double precision, too large for shared memory, so:
//
//  * one CTA computes one band of 4096 elements (4096/d whole rows) of one
//    ADO; the band arrives by one TMA bulk copy; consecutive CTAs take the
//    bands of one ADO, so the rest of its slab is in L2 while they run;
//  * column flips of the transverse field and row flips inside the band read
//    shared memory; row flips across bands read the slab through L2;
//  * neighbour terms are elementwise (diagonal V) and read through L2, two
//    entries at a time; the up term of tier L-1 (neighbours in the top tier)
//    comes from large_upterm_kernel, which walks the top tier tile by tile.
//
// With a dense H (HX_FLAG_DENSE_H, complex64 path) the diagonal table keeps
// the real diagonal of H and the commutator with the rest of H (no flip
// terms) comes from the product Y_n = X_n H_off of every ADO, computed before
// the stage by the tensor-core GEMM (hx_tcgemm.cu) as one [H d x 2d] x
// [2d x 2d] real product in 3-term TF32 split form.  Every ADO is Hermitian,
// so H_off X_n = Y_n^dagger and -i[H_off, X_n]_rc = -i(conj(Y_cr) - Y_rc): one
// product per ADO, not two.
//
// The reference has no precision other than the compiled one
// (src/legacy_compile_options.h:6); the complex64 path is the
// mixed-precision extension of this propagator.

#include <cuda_runtime.h>

#include <cstdint>

#include "hx_internal.h"

namespace hx {

namespace {

__device__ __forceinline__ uint32_t l_addr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

constexpr uint32_t kLargeSpin = 1u << 20;

template <typename R>
__device__ __forceinline__ C2<R> mk(R x, R y)
{
    C2<R> v;
    v.x = x;
    v.y = y;
    return v;
}

// Threads of a full-slab band CTA: complex64 bands take twice the threads
// (8 elements each instead of 16), so twice the warps per SM hide the
// neighbour gathers' latency at the same shared memory per CTA.
template <typename R> struct LargeThreads { static constexpr int T = 256; };
template <> struct LargeThreads<float> { static constexpr int T = 512; };

template <typename R, int LOGD>
__global__ void __launch_bounds__(LargeThreads<R>::T, 2)
    large_kernel(LargeArgs<R> a, const C2<R>* __restrict__ u, const C2<R>* rho, C2<R>* out, double alpha_d,
                 int base_kind)
{
    using C = C2<R>;
    constexpr int D = 1 << LOGD, T = LargeThreads<R>::T, BE = 4096, E = BE / T, CH = 4;
    constexpr long long D2 = static_cast<long long>(D) * D;
    constexpr int NB = static_cast<int>(D2 / BE);  // bands per slab
    extern __shared__ __align__(128) unsigned char smem[];
    C* sx = reinterpret_cast<C*>(smem);                       // [BE] the band
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + BE * sizeof(C));
    double* sWc = reinterpret_cast<double*>(bar + 2);         // [2M]
    double* sWa = sWc + 2 * a.M;                              // [2M]
    R* sV = reinterpret_cast<R*>(sWa + 2 * a.M);              // [J][D]
    R* sH = sV + a.J * D;                                     // [LOGD]
    int* sSlab = reinterpret_cast<int*>(sH + LOGD + 1);       // [2M]
    int* sBath = sSlab + 2 * a.M;                             // [2M]
    constexpr int RB = BE / D, RBP = RB + 1;                  // rows of the band; padded strip row
    C* sYT = reinterpret_cast<C*>((reinterpret_cast<uintptr_t>(sBath + 2 * a.M) + 15) & ~uintptr_t(15));  // [D][RBP]

    const int tid = threadIdx.x;
    const long long n = a.first_ado + static_cast<long long>(blockIdx.x) / NB;
    const long long be = static_cast<long long>(blockIdx.x % NB) * BE;  // band's first element in the slab
    const int r0 = static_cast<int>(be >> LOGD);                        // band's first row
    const C* un = u + n * D2;
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(l_addr(bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(l_addr(bar)),
                     "r"(static_cast<uint32_t>(BE * sizeof(C)))
                     : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                         l_addr(sx)),
                     "l"(un + be), "r"(static_cast<uint32_t>(BE * sizeof(C))), "r"(l_addr(bar))
                     : "memory");
    }
    const int Q = a.ent_count[n];
    for (int i = tid; i < a.J * D; i += T) sV[i] = a.vdiag[i];
    if (tid < LOGD) sH[tid] = a.hflip[tid];
    for (int q = tid; q < Q; q += T) {
        const long long src = n * 2 * a.M + q;
        sSlab[q] = a.ent_slab[src];
        sBath[q] = a.ent_bath[src] & 0xffff;
        sWc[q] = a.ent_wc[src];
        sWa[q] = a.ent_wa[src];
    }
    if (a.dense_y) {
        // dense H: the strip Y_n[c][r0 .. r0 + RB) of every column c (coalesced row pieces, asynchronous
        // 8-byte copies that overlap the table loads) for the transposed elements Y_cr of this band
        const C* yn = a.dense_y + n * D2;
#pragma unroll
        for (int k = 0; k < BE / T; ++k) {
            const int i = tid + k * T, cc = i / RB, j = i - cc * RB;
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(l_addr(sYT + cc * RBP + j)),
                         "l"(yn + (static_cast<long long>(cc) << LOGD) + r0 + j)
                         : "memory");
        }
    }
    const R g = static_cast<R>(a.gsum[n]);
    const int slot = a.slot ? a.slot[n] : -1;
    const R alpha = static_cast<R>(alpha_d);
    if (a.dense_y) asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    bool ok = false;
    for (uint32_t it = 0; it < kLargeSpin && !ok; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\tselp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(l_addr(bar))
            : "memory");
        ok = done != 0;
    }
    if (__syncthreads_or(!ok)) {
        if (tid == 0) atomicExch(a.error_flag, 1);
        return;
    }

    C acc[E];
    // ---- diagonal table and transverse field
#pragma unroll
    for (int k0 = 0; k0 < E; k0 += CH) {
        C x[CH], t[CH];
#pragma unroll
        for (int kk = 0; kk < CH; ++kk) {
            x[kk] = sx[tid + T * (k0 + kk)];
            t[kk] = __ldg(a.diag + be + tid + T * (k0 + kk));
        }
#pragma unroll
        for (int kk = 0; kk < CH; ++kk) {
            const int e = tid + T * (k0 + kk);
            const long long ge = be + e;
            R hr = 0, hi = 0;
#pragma unroll
            for (int i = 0; i < LOGD; ++i) {
                if (sH[i] == R(0)) continue;  // no field on this spin (every spin with a dense H): no gathers
                constexpr long long one = 1;
                const long long fb = static_cast<long long>(D) << i;  // row bit i of the element index
                C rowp;
                if (fb < BE) rowp = sx[e ^ static_cast<int>(fb)];
                else rowp = __ldg(un + (ge ^ fb));
                const C colp = sx[e ^ static_cast<int>(one << i)];
                hr += sH[i] * (rowp.x - colp.x);
                hi += sH[i] * (rowp.y - colp.y);
            }
            const R tr = t[kk].x - g;
            acc[k0 + kk].x = tr * x[kk].x - t[kk].y * x[kk].y + hi;
            acc[k0 + kk].y = tr * x[kk].y + t[kk].y * x[kk].x - hr;
            if (a.dense_y) {
                // -i [H_off, X] = -i (conj(Y_cr) - Y_rc) from the tensor-core product Y = X H_off
                const int r = static_cast<int>(ge >> LOGD), c = static_cast<int>(ge & (D - 1));
                const C yrc = __ldg(a.dense_y + n * D2 + ge), ycr = sYT[c * RBP + (r - r0)];
                acc[k0 + kk].x -= yrc.y + ycr.y;
                acc[k0 + kk].y += yrc.x - ycr.x;
            }
        }
    }
    // ---- neighbour entries, two at a time, CH elements per load batch
    const C* ub = u + be + tid;
    int q = 0;
    for (; q + 1 < Q; q += 2) {
        const int j0 = sBath[q], j1 = sBath[q + 1];
        const R wc0 = static_cast<R>(sWc[q]), wa0 = static_cast<R>(sWa[q]);
        const R wc1 = static_cast<R>(sWc[q + 1]), wa1 = static_cast<R>(sWa[q + 1]);
        const C* s0 = ub + static_cast<long long>(sSlab[q]) * D2;
        const C* s1 = ub + static_cast<long long>(sSlab[q + 1]) * D2;
#pragma unroll
        for (int k0 = 0; k0 < E; k0 += CH) {
            C y0[CH], y1[CH];
            R ar0[CH], ai0[CH], ar1[CH], ai1[CH];
#pragma unroll
            for (int kk = 0; kk < CH; ++kk) {
                const long long ge = be + tid + T * (k0 + kk);
                const int r = static_cast<int>(ge >> LOGD), c = static_cast<int>(ge & (D - 1));
                const R vr0 = sV[j0 * D + r], vc0 = sV[j0 * D + c];
                const R vr1 = sV[j1 * D + r], vc1 = sV[j1 * D + c];
                ar0[kk] = -(vr0 + vc0) * wa0;
                ai0[kk] = -(vr0 - vc0) * wc0;
                ar1[kk] = -(vr1 + vc1) * wa1;
                ai1[kk] = -(vr1 - vc1) * wc1;
                y0[kk] = mk<R>(0, 0);
                y1[kk] = mk<R>(0, 0);
                if (ar0[kk] != R(0) || ai0[kk] != R(0)) y0[kk] = __ldg(s0 + T * (k0 + kk));
                if (ar1[kk] != R(0) || ai1[kk] != R(0)) y1[kk] = __ldg(s1 + T * (k0 + kk));
            }
#pragma unroll
            for (int kk = 0; kk < CH; ++kk) {
                acc[k0 + kk].x += ar0[kk] * y0[kk].x - ai0[kk] * y0[kk].y + ar1[kk] * y1[kk].x - ai1[kk] * y1[kk].y;
                acc[k0 + kk].y += ar0[kk] * y0[kk].y + ai0[kk] * y0[kk].x + ar1[kk] * y1[kk].y + ai1[kk] * y1[kk].x;
            }
        }
    }
    if (q < Q) {
        const int j0 = sBath[q];
        const R wc0 = static_cast<R>(sWc[q]), wa0 = static_cast<R>(sWa[q]);
        const C* s0 = ub + static_cast<long long>(sSlab[q]) * D2;
#pragma unroll
        for (int k = 0; k < E; ++k) {
            const long long ge = be + tid + T * k;
            const int r = static_cast<int>(ge >> LOGD), c = static_cast<int>(ge & (D - 1));
            const R vr0 = sV[j0 * D + r], vc0 = sV[j0 * D + c];
            const R ar = -(vr0 + vc0) * wa0, ai = -(vr0 - vc0) * wc0;
            C y = mk<R>(0, 0);
            if (ar != R(0) || ai != R(0)) y = __ldg(s0 + T * k);
            acc[k].x += ar * y.x - ai * y.y;
            acc[k].y += ar * y.y + ai * y.x;
        }
    }
    // ---- up term of tier L-1 (neighbours in the top tier), summed by large_upterm_kernel
    if (slot >= 0) {
        const C* Un = a.U + static_cast<long long>(slot) * D2 + be + tid;
#pragma unroll
        for (int k = 0; k < E; ++k) {
            const C w = __ldcs(Un + T * k);
            acc[k].x += w.x;
            acc[k].y += w.y;
        }
    }
    // ---- Horner epilogue
    C* on = out + n * D2 + be + tid;
    const C* rn = rho + n * D2 + be + tid;
#pragma unroll
    for (int k = 0; k < E; ++k) {
        C b;
        if (base_kind == kBaseSelf) b = sx[tid + T * k];
        else if (base_kind == kBaseRho) b = __ldcs(rn + T * k);
        else b = mk<R>(0, 0);
        __stcs(on + T * k, mk<R>(b.x + alpha * acc[k].x, b.y + alpha * acc[k].y));
    }
}

// Element (r, c) of a Hermitian-packed slab, any r, c (one load, no branch
// around it, so several lookups can be in flight at once).
template <typename C>
__device__ __forceinline__ C packed_at(const C* __restrict__ slab, int r, int c, int logd)
{
    const bool lower = r > c;
    const C v = __ldg(slab + herm_index(lower ? c : r, lower ? r : c, logd));
    C w;
    w.x = v.x;
    w.y = lower ? -v.y : v.y;
    return w;
}

// ---------------------------------------------------------------------------
// Band kernel on Hermitian-packed slabs (layout in hx_internal.h).  A band is
// G = 2048 / d packed rows: matrix rows s0 .. s0+G-1 and their mirror rows
// d-1-s0-G+1 .. d-1-s0, so 2G full rows (4096 elements, as a full-slab band)
// and G (d+1) packed outputs.  The CTA rebuilds those 2G rows in shared
// memory: the upper parts from the band's own packed rows, the lower parts as
// conjugates gathered from the other packed rows through L2.  Column flips
// and the row flips of the low log2 G bits then read shared memory (mirror
// rows flip with the same local index); flips of higher row bits read the
// packed slab through L2.  Neighbours, the Horner base, U and the output
// stream in packed order.  No device-side waits.
// Threads per band: complex64 bands hide their L2 gathers with 512 threads
// (5 elements each); double-precision ones need more registers: 384 (6 each).
template <typename R> struct BandThreads { static constexpr int T = 384; };
template <> struct BandThreads<float> { static constexpr int T = 512; };

template <typename R, int LOGD>
__global__ void __launch_bounds__(BandThreads<R>::T, 2)
    herm_band_kernel(LargeArgs<R> a, const C2<R>* __restrict__ u, const C2<R>* rho, C2<R>* out, double alpha_d,
                     int base_kind)
{
    using C = C2<R>;
    constexpr int D = 1 << LOGD, T = BandThreads<R>::T, G = 2048 / D, LOGG = 11 - LOGD;
    constexpr int NE = G * (D + 1);  // packed elements of a band
    constexpr int E = (NE + T - 1) / T;
    constexpr long long P = static_cast<long long>(D / 2) * (D + 1);
    constexpr int NB = (D / 2) / G;  // bands per slab
    extern __shared__ __align__(128) unsigned char smem[];
    C* sx = reinterpret_cast<C*>(smem);                                   // [2G][D] rebuilt rows
    double* sWc = reinterpret_cast<double*>(smem + 2 * G * D * sizeof(C));  // [2M]
    double* sWa = sWc + 2 * a.M;                                          // [2M]
    R* sV = reinterpret_cast<R*>(sWa + 2 * a.M);                          // [J][D]
    R* sH = sV + a.J * D;                                                 // [LOGD]
    int* sSlab = reinterpret_cast<int*>(sH + LOGD + 1);                   // [2M]
    int* sBath = sSlab + 2 * a.M;                                         // [2M]

    const int tid = threadIdx.x;
    const long long n = a.first_ado + static_cast<long long>(blockIdx.x) / NB;
    const int s0 = static_cast<int>(blockIdx.x % NB) * G;
    const int q0 = s0 * (D + 1);  // the band's first packed element
    const C* un = u + n * P;
    const int Q = a.ent_count[n];
    for (int i = tid; i < a.J * D; i += T) sV[i] = a.vdiag[i];
    if (tid < LOGD) sH[tid] = a.hflip[tid];
    for (int q = tid; q < Q; q += T) {
        const long long src = n * 2 * a.M + q;
        sSlab[q] = a.ent_slab[src];
        sBath[q] = a.ent_bath[src] & 0xffff;
        sWc[q] = a.ent_wc[src];
        sWa[q] = a.ent_wa[src];
    }
    const R g = static_cast<R>(a.gsum[n]);
    const int slot = a.slot ? a.slot[n] : -1;
    const R alpha = static_cast<R>(alpha_d);
    // local row of matrix row r of the band
    auto lrow = [&](int r) { return r < D / 2 ? r - s0 : G + (D - 1 - s0 - r); };

    // ---- rebuild the band's 2G rows: upper parts from the band ...
    int rc[E];
#pragma unroll
    for (int k = 0; k < E; ++k) {
        const int i = tid + T * k;
        int r = 0, c = 0;
        if (i < NE) {
            herm_coords(q0 + i, LOGD, r, c);
            sx[lrow(r) * D + c] = __ldg(un + q0 + i);
        }
        rc[k] = (r << 16) | c;
    }
    // ... lower parts (c < r) as conjugates of the elements (c, r) of other packed rows
#pragma unroll 4
    for (int t = tid; t < G * (D - 1); t += T) {
        const int j = t / (D - 1), w = t - j * (D - 1);
        const int ra = s0 + j;
        int lr, r, c;
        if (w < ra) {
            lr = j;
            r = ra;
            c = w;
        } else {
            lr = G + j;
            r = D - 1 - s0 - j;
            c = w - ra;
        }
        const C v = __ldg(un + herm_index(c, r, LOGD));
        sx[lr * D + c] = mk<R>(v.x, -v.y);
    }
    __syncthreads();

    // ---- diagonal table and transverse field
    C acc[E];
#pragma unroll
    for (int k = 0; k < E; ++k) {
        const int i = tid + T * k;
        acc[k] = mk<R>(0, 0);
        if (i >= NE) continue;
        const int r = rc[k] >> 16, c = rc[k] & 0xffff, lr = lrow(r);
        const C x = sx[lr * D + c];
        const C t = __ldg(a.diag + q0 + i);
        R hr = 0, hi = 0;
#pragma unroll
        for (int b = 0; b < LOGD; ++b) {
            C rowp;
            if (b < LOGG) rowp = sx[(lr ^ (1 << b)) * D + c];
            else rowp = packed_at(un, r ^ (1 << b), c, LOGD);
            const C colp = sx[lr * D + (c ^ (1 << b))];
            hr += sH[b] * (rowp.x - colp.x);
            hi += sH[b] * (rowp.y - colp.y);
        }
        const R tr = t.x - g;
        acc[k].x = tr * x.x - t.y * x.y + hi;
        acc[k].y = tr * x.y + t.y * x.x - hr;
    }
    // ---- neighbour entries, E loads in flight
    for (int q = 0; q < Q; ++q) {
        const int j = sBath[q];
        const R wc = static_cast<R>(sWc[q]), wa = static_cast<R>(sWa[q]);
        const C* src = u + static_cast<long long>(sSlab[q]) * P + q0 + tid;
        C y[E];
#pragma unroll
        for (int k = 0; k < E; ++k) {
            const int r = rc[k] >> 16, c = rc[k] & 0xffff;
            const R vr = sV[j * D + r], vc = sV[j * D + c];
            y[k] = mk<R>(0, 0);
            if (tid + T * k < NE && ((vr + vc) * wa != R(0) || (vr - vc) * wc != R(0))) y[k] = __ldg(src + T * k);
        }
#pragma unroll
        for (int k = 0; k < E; ++k) {
            const int r = rc[k] >> 16, c = rc[k] & 0xffff;
            const R vr = sV[j * D + r], vc = sV[j * D + c];
            const R ar = -(vr + vc) * wa, ai = -(vr - vc) * wc;
            acc[k].x += ar * y[k].x - ai * y[k].y;
            acc[k].y += ar * y[k].y + ai * y[k].x;
        }
    }
    // ---- up term of tier L-1, summed by large_upterm_kernel
    if (slot >= 0) {
        const C* Un = a.U + static_cast<long long>(slot) * P + q0 + tid;
#pragma unroll
        for (int k = 0; k < E; ++k) {
            if (tid + T * k >= NE) continue;
            const C w = __ldcs(Un + T * k);
            acc[k].x += w.x;
            acc[k].y += w.y;
        }
    }
    // ---- Horner epilogue
    C* on = out + n * P + q0 + tid;
    const C* rn = rho + n * P + q0 + tid;
#pragma unroll
    for (int k = 0; k < E; ++k) {
        if (tid + T * k >= NE) continue;
        C b;
        if (base_kind == kBaseSelf) {
            const int r = rc[k] >> 16, c = rc[k] & 0xffff;
            b = sx[lrow(r) * D + c];
        } else if (base_kind == kBaseRho) {
            b = __ldcs(rn + T * k);
        } else {
            b = mk<R>(0, 0);
        }
        __stcs(on + T * k, mk<R>(b.x + alpha * acc[k].x, b.y + alpha * acc[k].y));
    }
}

// Up term of tier L-1 in the working precision, tile-major so the top-tier
// data of the resident tiles stays in L2 (as upterm_kernel, hx_upterm.cu).
constexpr int kUpWarps = 8, kUpSlots = 4, kUpTile = 32;

template <typename R>
__global__ void __launch_bounds__(kUpWarps * 32)
    large_upterm_kernel(LargeUpArgs<R> a, const C2<R>* __restrict__ u, C2<R>* __restrict__ U)
{
    using C = C2<R>;
    const int D = 1 << a.logd;
    // elements per stored slab: d^2, or the packed upper triangle
    const long long D2 = a.herm ? herm_elems(a.logd) : static_cast<long long>(D) * D;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long e = static_cast<long long>(blockIdx.y) * kUpTile + lane;
    if (e >= D2) return;
    int r, c;
    if (a.herm) {
        herm_coords(static_cast<int>(e), a.logd, r, c);
    } else {
        r = static_cast<int>(e >> a.logd);
        c = static_cast<int>(e & (D - 1));
    }
    const C* ue = u + e;
    const int s0 = (blockIdx.x * kUpWarps + warp) * kUpSlots;
    for (int s = s0; s < s0 + kUpSlots && s < a.S; ++s) {
        const int32_t* slab = a.slab + static_cast<long long>(s) * a.M;
        R re = 0, im = 0;
        for (int j = 0; j < a.J; ++j) {
            const R del = __ldg(a.vdiag + j * D + r) - __ldg(a.vdiag + j * D + c);
            if (del == R(0)) continue;
            const int m1 = __ldg(a.bath_off + j + 1);
            R sr = 0, si = 0;
            for (int m = __ldg(a.bath_off + j); m < m1; ++m) {
                const C y = __ldg(ue + static_cast<long long>(__ldg(slab + m)) * D2);
                sr += y.x;
                si += y.y;
            }
            re += del * si;  // -i del S
            im -= del * sr;
        }
        U[static_cast<long long>(s) * D2 + e] = mk<R>(re, im);
    }
}

// Tier-0 ADO of the mixed-precision propagator in double precision: its own
// slab u0, H and diagonal terms in FP64; its (up) neighbours come from the
// complex64 hierarchy and are accumulated in FP64.  Writes the FP64 result
// and its complex64 copy (slot 0 of the complex64 output).
__global__ void __launch_bounds__(256)
    ado0_kernel(Ado0Args a, const double2* __restrict__ u0, const float2* __restrict__ u, const double2* rho0,
                double2* out0, float2* out32, double alpha, int base_kind)
{
    const int D = 1 << a.logd;
    const long long D2 = a.herm ? herm_elems(a.logd) : static_cast<long long>(D) * D;
    const long long ge = blockIdx.x * 256ll + threadIdx.x;
    if (ge >= D2) return;
    int r, c;
    if (a.herm) {
        herm_coords(static_cast<int>(ge), a.logd, r, c);
    } else {
        r = static_cast<int>(ge >> a.logd);
        c = static_cast<int>(ge & (D - 1));
    }
    const double2 x = u0[ge];
    const double2 t = a.diag[ge];
    double hr = 0.0, hi = 0.0;
    for (int i = 0; i < a.logd; ++i) {
        double2 p, q;
        if (a.herm) {
            p = packed_at(u0, r ^ (1 << i), c, a.logd);
            q = packed_at(u0, r, c ^ (1 << i), a.logd);
        } else {
            p = u0[ge ^ (static_cast<long long>(D) << i)];
            q = u0[ge ^ (1ll << i)];
        }
        hr += a.hflip[i] * (p.x - q.x);
        hi += a.hflip[i] * (p.y - q.y);
    }
    double ax = t.x * x.x - t.y * x.y + hi;
    double ay = t.x * x.y + t.y * x.x - hr;
    if (a.dense_z) {
        // -i [H_off, X] = -i (conj(Z_cr) - Z_rc) of ADO 0 from its FP64 product Z = X H_off (X, H Hermitian);
        // the diagonal terms -2 Im Z_rr sum to -2 Im Tr(X H_off) = 0, so the commutator stays traceless
        const double2 zrc = a.dense_z[ge], zcr = a.dense_z[(static_cast<long long>(c) << a.logd) + r];
        ax -= zrc.y + zcr.y;
        ay += zrc.x - zcr.x;
    }
    const int Q = a.ent_count[0];
    for (int q = 0; q < Q; ++q) {
        const int j = a.ent_bath[q] & 0xffff;
        const double vr = a.vdiag[j * D + r], vc = a.vdiag[j * D + c];
        const double ar = -(vr + vc) * a.ent_wa[q], ai = -(vr - vc) * a.ent_wc[q];
        if (ar == 0.0 && ai == 0.0) continue;
        const float2 yf = u[static_cast<long long>(a.ent_slab[q]) * D2 + ge];
        const double yx = yf.x, yy = yf.y;
        ax += ar * yx - ai * yy;
        ay += ar * yy + ai * yx;
    }
    double2 b;
    if (base_kind == kBaseSelf) b = x;
    else if (base_kind == kBaseRho) b = rho0[ge];
    else b = make_double2(0.0, 0.0);
    const double2 o = make_double2(b.x + alpha * ax, b.y + alpha * ay);
    out0[ge] = o;
    out32[ge] = make_float2(static_cast<float>(o.x), static_cast<float>(o.y));
}

// Z = X H, d x d complex FP64 (ADO 0 of a dense-H stage): 32 x 32 output
// tiles, K staged through shared memory 16 at a time; each thread keeps four
// outputs of one column.  d^3 complex multiply-adds, a few microseconds at
// d = 256.
__global__ void __launch_bounds__(256) zgemm_kernel(const double2* __restrict__ x, const double2* __restrict__ h,
                                                    double2* __restrict__ z, int logd)
{
    constexpr int TM = 32, TN = 32, TK = 16;
    __shared__ double2 sa[TM][TK + 1];
    __shared__ double2 sb[TK][TN + 1];
    const int D = 1 << logd;
    const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    double2 acc[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[j] = make_double2(0.0, 0.0);
    for (int k0 = 0; k0 < D; k0 += TK) {
        for (int i = threadIdx.x; i < TM * TK; i += 256) {
            const int rr = i / TK, kk = i - rr * TK;
            sa[rr][kk] = x[(static_cast<long long>(m0 + rr) << logd) + k0 + kk];
        }
        for (int i = threadIdx.x; i < TK * TN; i += 256) {
            const int kk = i / TN, cc = i - kk * TN;
            sb[kk][cc] = h[(static_cast<long long>(k0 + kk) << logd) + n0 + cc];
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < TK; ++kk) {
            const double2 b = sb[kk][tx];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const double2 av = sa[ty + 8 * j][kk];
                acc[j].x = fma(av.x, b.x, fma(-av.y, b.y, acc[j].x));
                acc[j].y = fma(av.x, b.y, fma(av.y, b.x, acc[j].y));
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) z[(static_cast<long long>(m0 + ty + 8 * j) << logd) + n0 + tx] = acc[j];
}

__global__ void d2f_kernel(const double2* __restrict__ in, float2* __restrict__ out, long long n)
{
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
        out[i] = make_float2(static_cast<float>(in[i].x), static_cast<float>(in[i].y));
}

__global__ void vec_d2f_kernel(const double* __restrict__ in, float* __restrict__ out, long long n)
{
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
        out[i] = static_cast<float>(in[i]);
}

template <typename R, int LOGD>
size_t large_smem(int M, int J, bool dense)
{
    const size_t strip = dense ? sizeof(C2<R>) * (1 << LOGD) * (4096 / (1 << LOGD) + 1) + 16 : 0;
    return 4096 * sizeof(C2<R>) + 16 + sizeof(double) * 4 * M + sizeof(R) * (J * (1 << LOGD) + LOGD + 1) +
           sizeof(int) * 4 * M + 16 + strip;
}

template <typename R, int LOGD>
bool launch_t(const LargeArgs<R>& a, const C2<R>* u, const C2<R>* rho, C2<R>* out, double alpha, int base,
              cudaStream_t s, bool launch)
{
    const size_t smem = large_smem<R, LOGD>(a.M, a.J, a.dense_y != nullptr);
    if (smem > 227 * 1024) return false;
    static size_t configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && configured[dev] < smem) {
        if (cudaFuncSetAttribute(large_kernel<R, LOGD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)) != cudaSuccess ||
            cudaFuncSetAttribute(herm_band_kernel<R, LOGD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)) != cudaSuccess)
            return false;
        configured[dev] = smem;
    }
    if (!launch) return true;
    // bands per slab: d^2 / 4096 full-slab bands, or (d / 2) / (2048 / d) = d^2 / 4096 packed bands
    const long long nb = (a.H - a.first_ado) * ((1ll << (2 * LOGD)) / 4096);
    if (nb <= 0) return true;
    if (a.herm)
        herm_band_kernel<R, LOGD><<<static_cast<unsigned>(nb), BandThreads<R>::T, smem, s>>>(a, u, rho, out, alpha, base);
    else large_kernel<R, LOGD><<<static_cast<unsigned>(nb), LargeThreads<R>::T, smem, s>>>(a, u, rho, out, alpha, base);
    return true;
}

template <typename R>
bool dispatch(const LargeArgs<R>& a, const C2<R>* u, const C2<R>* rho, C2<R>* out, double alpha, int base,
              cudaStream_t s, bool launch)
{
    switch (a.logd) {
    case 7: return launch_t<R, 7>(a, u, rho, out, alpha, base, s, launch);
    case 8: return launch_t<R, 8>(a, u, rho, out, alpha, base, s, launch);
    case 9: return launch_t<R, 9>(a, u, rho, out, alpha, base, s, launch);
    case 10: return launch_t<R, 10>(a, u, rho, out, alpha, base, s, launch);
    default: return false;
    }
}

}  // namespace

bool large_supported(int logd, int M, int J)
{
    if (logd < 7 || logd > 10) return false;
    const size_t need = 4096 * sizeof(double2) + 16 + sizeof(double) * 4 * M + sizeof(double) * (J * (1 << logd) + logd + 1) +
                        sizeof(int) * 4 * M + 16;
    return need <= 227 * 1024;
}

template <typename R>
bool prepare_large(const LargeArgs<R>& a)
{
    return dispatch<R>(a, nullptr, nullptr, nullptr, 0.0, 0, nullptr, false);
}

template <typename R>
bool launch_large(const LargeArgs<R>& a, const C2<R>* u, const C2<R>* rho, C2<R>* out, double alpha, int base_kind,
                  cudaStream_t s)
{
    return dispatch<R>(a, u, rho, out, alpha, base_kind, s, true);
}

template <typename R>
void launch_large_upterm(const LargeUpArgs<R>& a, const C2<R>* u, C2<R>* U, cudaStream_t s)
{
    if (a.S <= 0) return;
    const long long D2 = a.herm ? herm_elems(a.logd) : 1ll << (2 * a.logd);
    const int per = kUpWarps * kUpSlots;
    dim3 grid((a.S + per - 1) / per, static_cast<unsigned>((D2 + kUpTile - 1) / kUpTile));
    large_upterm_kernel<R><<<grid, kUpWarps * 32, 0, s>>>(a, u, U);
}

template bool prepare_large<double>(const LargeArgs<double>&);
template bool prepare_large<float>(const LargeArgs<float>&);
template bool launch_large<double>(const LargeArgs<double>&, const double2*, const double2*, double2*, double, int,
                                   cudaStream_t);
template bool launch_large<float>(const LargeArgs<float>&, const float2*, const float2*, float2*, double, int,
                                  cudaStream_t);
template void launch_large_upterm<double>(const LargeUpArgs<double>&, const double2*, double2*, cudaStream_t);
template void launch_large_upterm<float>(const LargeUpArgs<float>&, const float2*, float2*, cudaStream_t);

void launch_zgemm(const double2* x, const double2* h, double2* z, int logd, cudaStream_t s)
{
    const unsigned nt = 1u << (logd - 5);
    zgemm_kernel<<<dim3(nt, nt), 256, 0, s>>>(x, h, z, logd);
}

void launch_ado0(const Ado0Args& a, const double2* u0, const float2* u, const double2* rho0, double2* out0,
                 float2* out32, double alpha, int base_kind, cudaStream_t s)
{
    const long long D2 = a.herm ? herm_elems(a.logd) : 1ll << (2 * a.logd);
    ado0_kernel<<<static_cast<unsigned>((D2 + 255) / 256), 256, 0, s>>>(a, u0, u, rho0, out0, out32, alpha, base_kind);
}

void launch_d2f(const double2* in, float2* out, long long n, cudaStream_t s)
{
    d2f_kernel<<<148 * 8, 256, 0, s>>>(in, out, n);
}

void launch_vec_d2f(const double* in, float* out, long long n, cudaStream_t s)
{
    vec_d2f_kernel<<<static_cast<unsigned>(n < 148 * 256 ? (n + 255) / 256 : 148), 256, 0, s>>>(in, out, n);
}

}  // namespace hx
