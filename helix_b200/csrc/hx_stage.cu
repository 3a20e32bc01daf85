// Fused HEOM stage kernel (FP64) and small helper kernels.
//
// One launch of `stage_kernel` evaluates, for every ADO n of the hierarchy,
//
//     out_n = base_n + alpha * L(u)_n
//
// where L is the full HEOM right-hand side of the reference (getdRhoSparse,
// src/liouville.cu:749-869) for diagonal coupling operators V_j and
// H = diag(E) + sum_i h_i sigma_x(i).  For diagonal V_j every bath term is an
// elementwise product at the same (r, c) across neighbouring ADOs:
//
//   [V_j, X]_rc = (v_r - v_c) X_rc        {V_j, X}_rc = (v_r + v_c) X_rc
//
// so the reference's 8 SpMM + 8 transposes + 7 axpy + 1 diagonal kernel per
// ADO collapse into one pass over the ADO's slab.  The H term is
//   -i[(E_r - E_c) X_rc + sum_i h_i (X_{r^2^i, c} - X_{r, c^2^i})]
// evaluated from the slab staged in shared memory by one TMA bulk copy.
//
// Integrator: the reference's Taylor recurrence (develop(),
// src/liouville.cu:502-590) evaluates sum_{j<=m} (dt L)^j / j! rho.  The same
// polynomial in Horner form,
//   u_1 = rho + (dt/m) L rho,  u_s = rho + (dt/(m-s+1)) L u_{s-1},  rho' = u_m,
// needs one launch per stage with base = rho, and the last stage can write
// rho' in place (each element of rho is read and written by the same thread
// only, and neighbours are read from u).  That is 2m-1 state reads and m
// writes per step instead of the 2m-1 reads and 2m writes of the recurrence.

#include <cuda_runtime.h>

#include <cstdint>

#include "hx_internal.h"

namespace hx {

namespace {

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// 1-D TMA bulk copy global -> shared, completion signalled on `bar`.
// dst and src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Bounded wait: gives up after `limit` polls (each poll may itself block for
// a hardware-defined interval) and reports failure instead of hanging.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t limit)
{
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

constexpr uint32_t kWaitLimit = 1u << 20;

template <int LOGD>
__global__ void __launch_bounds__(256) stage_kernel(StageTables t, const double2* __restrict__ u,
                                                    const double2* rho, double2* out, double alpha,
                                                    int base_kind)
{
    constexpr int D = 1 << LOGD;
    constexpr int D2 = D * D;
    extern __shared__ __align__(128) unsigned char smem[];
    double2* su = reinterpret_cast<double2*>(smem);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + D2 * sizeof(double2));
    double* sE = reinterpret_cast<double*>(smem + D2 * sizeof(double2) + 16);
    const int M = t.M, J = t.J;
    double* sV = sE + D;
    double* sF = sV + J * D;
    double* sXi = sF + LOGD;
    double* sCt = sXi + J;
    double* sA = sCt + J;
    double* sB = sA + M;
    int* sUp = reinterpret_cast<int*>(sB + J);
    int* sDn = sUp + M;
    int* sOff = sDn + M;

    const long long n = t.order ? static_cast<long long>(t.order[blockIdx.x]) : static_cast<long long>(blockIdx.x);
    const long long H = t.H;
    // thread 0 alone owns the mbarrier (init, copy, wait); the others learn of
    // the slab's arrival from the block barrier that follows its wait
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_expect_tx(bar, D2 * sizeof(double2));
        bulk_load(su, u + n * D2, D2 * sizeof(double2), bar);
    }
    for (int i = threadIdx.x; i < D; i += blockDim.x) sE[i] = t.hdiag[i];
    for (int i = threadIdx.x; i < J * D; i += blockDim.x) sV[i] = t.vdiag[i];
    for (int i = threadIdx.x; i < LOGD; i += blockDim.x) sF[i] = t.hflip[i];
    for (int i = threadIdx.x; i < J; i += blockDim.x) {
        sXi[i] = t.xi[i];
        sCt[i] = t.counter[i];
        sB[i] = t.bcoef[n * J + i];
    }
    for (int i = threadIdx.x; i <= J; i += blockDim.x) sOff[i] = t.bath_off[i];
    for (int i = threadIdx.x; i < M; i += blockDim.x) {
        sA[i] = t.acoef[n * M + i];
        sUp[i] = t.edges[n * 2 * M + i];
        sDn[i] = t.edges[n * 2 * M + M + i];
    }
    const double g = t.gsum[n];
    // one barrier publishes the tables above and the arrival of the slab
    if (__syncthreads_or(threadIdx.x == 0 && !mbar_wait_bounded(bar, 0, kWaitLimit))) {
        if (threadIdx.x == 0) atomicExch(t.error_flag, 1);
        return;
    }

    const double2* rho_n = rho + n * D2;
    double2* out_n = out + n * D2;
    for (int e = threadIdx.x; e < D2; e += blockDim.x) {
        const int r = e >> LOGD;
        const int c = e & (D - 1);
        const double2 x = su[e];
        // sigma damping and -i(E_r - E_c)
        const double dre = -g;
        const double dim = -(sE[r] - sE[c]);
        double are = dre * x.x - dim * x.y;
        double aim = dre * x.y + dim * x.x;
        // transverse field: -i sum_i h_i (X_{r^2^i,c} - X_{r,c^2^i})
        double hre = 0.0, him = 0.0;
#pragma unroll
        for (int i = 0; i < LOGD; ++i) {
            const double h = sF[i];
            const double2 a = su[e ^ (1 << (i + LOGD))];
            const double2 b = su[e ^ (1 << i)];
            hre += h * (a.x - b.x);
            him += h * (a.y - b.y);
        }
        are += him;
        aim -= hre;
        for (int j = 0; j < J; ++j) {
            const double vr = sV[j * D + r];
            const double vc = sV[j * D + c];
            const double del = vr - vc;
            const double sig = vr + vc;
            // Xi: -KXi [V,[V,X]] and counter: -i kappa {V,[V,X]}
            const double cr = -sXi[j] * del * del;
            const double ci = -sCt[j] * del * sig;
            are += cr * x.x - ci * x.y;
            aim += cr * x.y + ci * x.x;
            if (del != 0.0) {
                // phi (up) + theta/psi (down): -i del sum_m (X_{n+e_m} + a_m X_{n-e_m})
                double sre = 0.0, sim = 0.0;
                for (int m = sOff[j]; m < sOff[j + 1]; ++m) {
                    const int up = sUp[m];
                    if (up < H) {
                        const double2 w = __ldg(u + static_cast<long long>(up) * D2 + e);
                        sre += w.x;
                        sim += w.y;
                    }
                    const int dn = sDn[m];
                    if (dn < H) {
                        const double2 w = __ldg(u + static_cast<long long>(dn) * D2 + e);
                        const double a = sA[m];
                        sre += a * w.x;
                        sim += a * w.y;
                    }
                }
                are += del * sim;
                aim -= del * sre;
            }
            if (sig != 0.0) {
                // theta2: -b_j {V, X_{n-e_0}}
                const int dn0 = sDn[sOff[j]];
                if (dn0 < H) {
                    const double2 w = __ldg(u + static_cast<long long>(dn0) * D2 + e);
                    const double bs = sB[j] * sig;
                    are -= bs * w.x;
                    aim -= bs * w.y;
                }
            }
        }
        double2 base;
        if (base_kind == kBaseSelf) base = x;
        else if (base_kind == kBaseRho) base = __ldcs(rho_n + e);
        else base = make_double2(0.0, 0.0);
        __stcs(out_n + e, make_double2(base.x + alpha * are, base.y + alpha * aim));
    }
}

size_t stage_smem_bytes(int logd, int M, int J)
{
    const size_t D = size_t(1) << logd;
    return D * D * 16 + 16 + 8 * (D + J * D + logd + 3 * J + M) + 4 * (2 * M + J + 1);
}

template <int LOGD>
void launch_stage_t(const StageTables& t, const double2* u, const double2* rho, double2* out, double alpha,
                    int base_kind, cudaStream_t s)
{
    const int D2 = 1 << (2 * LOGD);
    int threads = D2 < 256 ? D2 : 256;
    if (threads < 32) threads = 32;
    const size_t smem = stage_smem_bytes(LOGD, t.M, t.J);
    // the dynamic shared-memory limit is a per-device function attribute
    static size_t configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && configured[dev] < smem) {
        cudaFuncSetAttribute(stage_kernel<LOGD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem));
        configured[dev] = smem;
    }
    stage_kernel<LOGD><<<static_cast<unsigned>(t.H), threads, smem, s>>>(t, u, rho, out, alpha, base_kind);
}

// Position of element (r, c) of rho0; in a packed slab the real part of
// (r, c) equals that of (c, r), which is all the energy needs.
__device__ __forceinline__ int obs_index(int r, int c, int logd, int herm)
{
    if (!herm) return (r << logd) + c;
    return r <= c ? herm_index(r, c, logd) : herm_index(c, r, logd);
}

__global__ void observables_kernel(const double2* __restrict__ rho0, int logd, int herm,
                                   const double* __restrict__ hdiag, const double* __restrict__ hflip,
                                   double2* rho0_copy, double* out)
{
    const int D = 1 << logd;
    const int n = herm ? herm_elems(logd) : D * D;
    double en = 0.0, tr = 0.0, ti = 0.0;
    for (int r = threadIdx.x; r < D; r += blockDim.x) {
        const double2 dgl = rho0[obs_index(r, r, logd, herm)];
        en += hdiag[r] * dgl.x;
        tr += dgl.x;
        ti += dgl.y;
        for (int i = 0; i < logd; ++i) en += hflip[i] * rho0[obs_index(r ^ (1 << i), r, logd, herm)].x;
    }
    if (rho0_copy)
        for (int e = threadIdx.x; e < n; e += blockDim.x) rho0_copy[e] = rho0[e];
    __shared__ double red[3][32];
    for (int off = 16; off > 0; off >>= 1) {
        en += __shfl_down_sync(0xffffffffu, en, off);
        tr += __shfl_down_sync(0xffffffffu, tr, off);
        ti += __shfl_down_sync(0xffffffffu, ti, off);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { red[0][w] = en; red[1][w] = tr; red[2][w] = ti; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0, c = 0;
        for (int k = 0; k < static_cast<int>(blockDim.x >> 5); ++k) { a += red[0][k]; b += red[1][k]; c += red[2][k]; }
        out[0] = a;
        out[1] = b;
        out[2] = c;
    }
}

__global__ void finite_kernel(const double2* __restrict__ x, long long n, int* flag)
{
    int bad = 0;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const double2 v = x[i];
        if (!isfinite(v.x) || !isfinite(v.y)) bad = 1;
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 1);
}

__global__ void init_state_kernel(double2* rho, long long n, long long one)
{
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
        rho[i] = make_double2(i == one ? 1.0 : 0.0, 0.0);
}

__global__ void pack_herm_kernel(const double2* __restrict__ full, int logd, double2* __restrict__ packed)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= herm_elems(logd)) return;
    int r, c;
    herm_coords(i, logd, r, c);
    packed[i] = full[(r << logd) + c];
}

// scale2[k] = max |x|^2 over full slab k (one block per slab).
__global__ void slab_max_kernel(const double2* __restrict__ full, long long slab, double* __restrict__ scale2)
{
    __shared__ double red[256];
    const double2* x = full + blockIdx.x * slab;
    double m = 0.0;
    for (long long e = threadIdx.x; e < slab; e += blockDim.x) {
        const double2 v = x[e];
        m = fmax(m, v.x * v.x + v.y * v.y);
    }
    red[threadIdx.x] = m;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) scale2[blockIdx.x] = red[0];
}

// Check (packed == nullptr) or pack `count` full slabs into Hermitian-packed
// slabs first .. first + count - 1 of `packed`.  The check lowers *bad to the
// index of an ADO whose (c, r) differs from conj (r, c) by more than
// sqrt(rel_tol2 * scale2).
__global__ void pack_check_kernel(const double2* __restrict__ full, long long count, int logd, double rel_tol2,
                                  const double* __restrict__ scale2, long long first, double2* __restrict__ packed,
                                  int* bad)
{
    const int D = 1 << logd;
    const long long P = herm_elems(logd);
    const long long total = count * P;
    for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
         t += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long k = t / P;
        const int i = static_cast<int>(t - k * P);
        int r, c;
        herm_coords(i, logd, r, c);
        const double2* x = full + k * static_cast<long long>(D) * D;
        const double2 up = x[static_cast<long long>(r) * D + c];
        if (!packed) {
            if (r != c) {
                const double2 lo = x[static_cast<long long>(c) * D + r];
                const double dr = up.x - lo.x, di = up.y + lo.y;
                if (dr * dr + di * di > rel_tol2 * scale2[k]) atomicMin(bad, static_cast<int>(first + k));
            }
        } else {
            packed[(first + k) * P + i] = up;
        }
    }
}

}  // namespace

void launch_herm_check(const double2* full, long long count, int logd, double rel_tol, double* scale2,
                       long long first, int* bad, cudaStream_t s)
{
    if (count <= 0) return;
    slab_max_kernel<<<static_cast<unsigned>(count), 256, 0, s>>>(full, 1LL << (2 * logd), scale2);
    pack_check_kernel<<<148 * 8, 256, 0, s>>>(full, count, logd, rel_tol * rel_tol, scale2, first, nullptr, bad);
}

// Packed complex64 copy of `count` full FP64 slabs (the mixed-precision hierarchy's upload).
__global__ void pack_f32_kernel(const double2* __restrict__ full, long long count, int logd, long long first,
                                float2* __restrict__ packed)
{
    const int D = 1 << logd;
    const long long P = herm_elems(logd);
    const long long total = count * P;
    for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
         t += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long k = t / P;
        const int i = static_cast<int>(t - k * P);
        int r, c;
        herm_coords(i, logd, r, c);
        const double2 up = full[k * static_cast<long long>(D) * D + static_cast<long long>(r) * D + c];
        packed[(first + k) * P + i] = make_float2(static_cast<float>(up.x), static_cast<float>(up.y));
    }
}

void launch_herm_pack_f32(const double2* full, long long count, int logd, long long first, float2* packed,
                          cudaStream_t s)
{
    if (count <= 0) return;
    pack_f32_kernel<<<148 * 8, 256, 0, s>>>(full, count, logd, first, packed);
}

void launch_herm_pack(const double2* full, long long count, int logd, long long first, double2* packed,
                      cudaStream_t s)
{
    if (count <= 0) return;
    pack_check_kernel<<<148 * 8, 256, 0, s>>>(full, count, logd, 0.0, nullptr, first, packed, nullptr);
}

void launch_stage(const StageTables& t, const double2* u, const double2* rho, double2* out, double alpha,
                  int base_kind, cudaStream_t s)
{
    switch (t.logd) {
    case 1: launch_stage_t<1>(t, u, rho, out, alpha, base_kind, s); break;
    case 2: launch_stage_t<2>(t, u, rho, out, alpha, base_kind, s); break;
    case 3: launch_stage_t<3>(t, u, rho, out, alpha, base_kind, s); break;
    case 4: launch_stage_t<4>(t, u, rho, out, alpha, base_kind, s); break;
    case 5: launch_stage_t<5>(t, u, rho, out, alpha, base_kind, s); break;
    case 6: launch_stage_t<6>(t, u, rho, out, alpha, base_kind, s); break;
    default: break;
    }
}

void launch_observables(const double2* rho0, int logd, int herm, const double* hdiag, const double* hflip,
                        double2* rho0_copy, double* out, cudaStream_t s)
{
    observables_kernel<<<1, 256, 0, s>>>(rho0, logd, herm, hdiag, hflip, rho0_copy, out);
}

void launch_pack_herm(const double2* full, int logd, double2* packed, cudaStream_t s)
{
    const int n = herm_elems(logd);
    pack_herm_kernel<<<(n + 255) / 256, 256, 0, s>>>(full, logd, packed);
}

void launch_finite_check(const double2* x, long long n, int* flag, cudaStream_t s)
{
    finite_kernel<<<148 * 4, 256, 0, s>>>(x, n, flag);
}

void launch_init_state(double2* rho, long long n, long long one, cudaStream_t s)
{
    init_state_kernel<<<148 * 4, 256, 0, s>>>(rho, n, one);
}

}  // namespace hx
