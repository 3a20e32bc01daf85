// Persistent fused stage kernel for d = 32 and d = 64 (FP64).
//
// Same mathematics as stage_kernel in hx_stage.cu (the reference RHS of
// getdRhoSparse, src/liouville.cu:749-869, for diagonal couplings), laid
// out for throughput:
//
//  * one persistent CTA per SM walks the ADOs; the slab of the next ADO is
//    prefetched by a TMA bulk copy into the second of two shared-memory
//    buffers while the current one is computed;
//  * thread t owns the elements e_k = t + 256 k (k < D^2/256): row r =
//    (t >> logd) + (256 >> logd) k, column c = t & (D-1).  Flips of the row
//    bits held in k are register moves; the other flips read shared memory;
//  * the ADO-independent part of the diagonal, -sum_j Xi_j (v_r - v_c)^2
//    - i[(E_r - E_c) + sum_j kappa_j (v_r^2 - v_c^2)], is a d x d table in
//    shared memory;
//  * neighbour terms come from a per-ADO list of present neighbours
//    (slab, bath, w_comm, w_anti): out += (-i delta w_comm - sigma w_anti) X_nbr
//    with delta = v_j(r) - v_j(c), sigma = v_j(r) + v_j(c); each entry issues
//    its 16 (or 4) element loads back to back, skipping elements whose weight
//    is zero;
//  * rho (Horner base) is read and the result written with streaming hints so
//    they do not displace neighbour slabs from L2.

#include <cuda_runtime.h>

#include <cstdint>

#include "hx_internal.h"

namespace hx {

namespace {

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void bar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void bar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void bar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void tma_load_1d(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool bar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

constexpr uint32_t kPollLimit = 1u << 20;

__device__ __forceinline__ double2 ld_stream(const double2* p)
{
    double2 v;
    asm volatile("ld.global.cs.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
    return v;
}

__device__ __forceinline__ void st_stream(double2* p, double2 v)
{
    asm volatile("st.global.cs.v2.f64 [%0], {%1, %2};" ::"l"(p), "d"(v.x), "d"(v.y) : "memory");
}

template <int LOGD>
struct Shape {
    static constexpr int D = 1 << LOGD;
    static constexpr int D2 = D * D;
    static constexpr int THREADS = 256;
    static constexpr int ELEMS = D2 / THREADS;               // elements per thread
    static constexpr int RSTEP_BITS = 8 - LOGD;              // k advances r by 2^RSTEP_BITS
};

template <int LOGD>
__global__ void __launch_bounds__(256, 1)
    stage2_kernel(Stage2Args a, const double2* __restrict__ u, const double2* rho, double2* out, double alpha,
                  int base_kind)
{
    using S = Shape<LOGD>;
    constexpr int D = S::D, D2 = S::D2, E = S::ELEMS;
    extern __shared__ __align__(1024) unsigned char smem[];
    double2* slab0 = reinterpret_cast<double2*>(smem);
    double2* slab1 = slab0 + D2;
    double2* sT = slab1 + D2;                                 // diagonal table
    uint64_t* bars = reinterpret_cast<uint64_t*>(sT + D2);    // 2 barriers
    double* sV = reinterpret_cast<double*>(bars + 2);         // [J][D]
    double* sH = sV + a.J * D;                                // [LOGD] transverse field
    double* sWc = sH + LOGD;                                  // [2M]
    double* sWa = sWc + 2 * a.M;                              // [2M]
    int* sSlab = reinterpret_cast<int*>(sWa + 2 * a.M);       // [2M]
    int* sBath = sSlab + 2 * a.M;                             // [2M]

    const int tid = threadIdx.x;
    const long long H = a.H;
    const int G = gridDim.x;

    if (tid == 0) {
        bar_init(&bars[0], 1);
        bar_init(&bars[1], 1);
        bar_fence_init();
    }
    for (int i = tid; i < D2; i += S::THREADS) sT[i] = a.diag[i];
    for (int i = tid; i < a.J * D; i += S::THREADS) sV[i] = a.vdiag[i];
    if (tid < LOGD) sH[tid] = a.hflip[tid];
    __syncthreads();

    auto ado_of = [&](long long it) -> long long { return a.order ? a.order[it] : it; };
    long long first = blockIdx.x;
    if (first < H && tid == 0) {
        bar_expect_tx(&bars[0], D2 * sizeof(double2));
        tma_load_1d(slab0, u + ado_of(first) * D2, D2 * sizeof(double2), &bars[0]);
    }

    const int c = tid & (D - 1);
    const int r0 = tid >> LOGD;
    int iter = 0;
    for (long long it = first; it < H; it += G, ++iter) {
        const int buf = iter & 1;
        const long long n = ado_of(it);
        double2* slab = buf ? slab1 : slab0;
        // prefetch the next slab into the other buffer (freed by the barrier at the end of the last iteration)
        const long long nx = it + G;
        if (nx < H && tid == 0) {
            double2* other = buf ? slab0 : slab1;
            bar_expect_tx(&bars[buf ^ 1], D2 * sizeof(double2));
            tma_load_1d(other, u + ado_of(nx) * D2, D2 * sizeof(double2), &bars[buf ^ 1]);
        }
        // neighbour entries of this ADO
        const int Q = a.ent_count[n];
        for (int q = tid; q < Q; q += S::THREADS) {
            const long long src = n * 2 * a.M + q;
            sSlab[q] = a.ent_slab[src];
            sBath[q] = a.ent_bath[src];
            sWc[q] = a.ent_wc[src];
            sWa[q] = a.ent_wa[src];
        }
        const double g = a.gsum[n];
        __syncthreads();
        {
            bool ok = false;
            for (uint32_t p = 0; p < kPollLimit && !ok; ++p) ok = bar_try_wait(&bars[buf], (iter >> 1) & 1);
            if (__syncthreads_or(!ok)) {  // uniform exit: every thread leaves together
                if (tid == 0) atomicExch(a.error_flag, 1);
                return;
            }
        }

        // ---- diagonal + transverse field from shared memory ----------------
        double2 acc[E];
        double2 x[E];
#pragma unroll
        for (int k = 0; k < E; ++k) x[k] = slab[tid + S::THREADS * k];
#pragma unroll
        for (int k = 0; k < E; ++k) {
            const int e = tid + S::THREADS * k;
            const double2 t = sT[e];
            const double tr = t.x - g;
            acc[k].x = tr * x[k].x - t.y * x[k].y;
            acc[k].y = tr * x[k].y + t.y * x[k].x;
            double hr = 0.0, hi = 0.0;
#pragma unroll
            for (int i = 0; i < LOGD; ++i) {
                const double h = sH[i];
                double2 rowp;
                if (i >= S::RSTEP_BITS) rowp = x[k ^ (1 << (i - S::RSTEP_BITS))];
                else rowp = slab[e ^ (D << i)];
                const double2 colp = slab[e ^ (1 << i)];
                hr += h * (rowp.x - colp.x);
                hi += h * (rowp.y - colp.y);
            }
            acc[k].x += hi;
            acc[k].y -= hr;
        }

        // ---- neighbour terms -------------------------------------------------
        const double2* ubase = u + tid;
        for (int q = 0; q < Q; ++q) {
            const int j = sBath[q];
            const double wc = sWc[q];
            const double wa = sWa[q];
            const double2* p = ubase + static_cast<long long>(sSlab[q]) * D2;
            const double vc = sV[j * D + c];
            const double* vrow = sV + j * D + r0;
            double2 y[E];
            // issue every load of this entry first (independent, predicated on a nonzero weight) ...
#pragma unroll
            for (int k = 0; k < E; ++k) {
                const double vr = vrow[k << S::RSTEP_BITS];
                const double wre = -(vr + vc) * wa;
                const double wim = -(vr - vc) * wc;
                y[k] = make_double2(0.0, 0.0);
                if (wre != 0.0 || wim != 0.0) y[k] = __ldg(p + S::THREADS * k);
            }
            // ... then accumulate (weights recomputed from the broadcast row values)
#pragma unroll
            for (int k = 0; k < E; ++k) {
                const double vr = vrow[k << S::RSTEP_BITS];
                const double wre = -(vr + vc) * wa;
                const double wim = -(vr - vc) * wc;
                acc[k].x += wre * y[k].x - wim * y[k].y;
                acc[k].y += wre * y[k].y + wim * y[k].x;
            }
        }

        // ---- Horner epilogue ----------------------------------------------------
        const double2* rho_n = rho + n * D2 + tid;
        double2* out_n = out + n * D2 + tid;
        if (base_kind == kBaseRho) {
            double2 b[E];
#pragma unroll
            for (int k = 0; k < E; ++k) b[k] = ld_stream(rho_n + S::THREADS * k);
#pragma unroll
            for (int k = 0; k < E; ++k)
                st_stream(out_n + S::THREADS * k, make_double2(b[k].x + alpha * acc[k].x, b[k].y + alpha * acc[k].y));
        } else if (base_kind == kBaseSelf) {
#pragma unroll
            for (int k = 0; k < E; ++k) {
                const double2 b = slab[tid + S::THREADS * k];
                st_stream(out_n + S::THREADS * k, make_double2(b.x + alpha * acc[k].x, b.y + alpha * acc[k].y));
            }
        } else {
#pragma unroll
            for (int k = 0; k < E; ++k)
                st_stream(out_n + S::THREADS * k, make_double2(alpha * acc[k].x, alpha * acc[k].y));
        }
        __syncthreads();  // slab buffer and entry lists are reused next iteration
    }
}

template <int LOGD>
size_t stage2_smem(int M, int J)
{
    using S = Shape<LOGD>;
    return 3 * S::D2 * sizeof(double2) + 16 + sizeof(double) * (J * S::D + LOGD + 4 * M) + sizeof(int) * 4 * M;
}

template <int LOGD>
bool launch_stage2_t(const Stage2Args& a, const double2* u, const double2* rho, double2* out, double alpha,
                     int base_kind, cudaStream_t s)
{
    const size_t smem = stage2_smem<LOGD>(a.M, a.J);
    if (smem > 227 * 1024) return false;
    static size_t configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && configured[dev] < smem) {
        if (cudaFuncSetAttribute(stage2_kernel<LOGD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)) != cudaSuccess)
            return false;
        configured[dev] = smem;
    }
    long long grid = a.ctas;
    if (grid > a.H) grid = a.H;
    stage2_kernel<LOGD><<<static_cast<unsigned>(grid), 256, smem, s>>>(a, u, rho, out, alpha, base_kind);
    return true;
}

// Per-ADO neighbour entries, grouped by bath: for each mode m of bath j,
//   up present:   (slab n+e_m, j, w_comm = 1,        w_anti = 0)
//   down present: (slab n-e_m, j, w_comm = a_{n,m},  w_anti = b_{n,j} if m is the Drude mode else 0)
__global__ void entries_kernel(const int32_t* edges, const double* acoef, const double* bcoef,
                               const int32_t* bath_off, long long H, int M, int J, int* count, int32_t* slab,
                               int32_t* bath, double* wc, double* wa)
{
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= H) return;
    int q = 0;
    const long long o = i * 2 * M;
    for (int j = 0; j < J; ++j) {
        for (int m = bath_off[j]; m < bath_off[j + 1]; ++m) {
            const int up = edges[i * 2 * M + m];
            if (up < H) {
                slab[o + q] = up;
                bath[o + q] = j;
                wc[o + q] = 1.0;
                wa[o + q] = 0.0;
                ++q;
            }
            const int dn = edges[i * 2 * M + M + m];
            if (dn < H) {
                slab[o + q] = dn;
                bath[o + q] = j;
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

bool launch_stage2(const Stage2Args& a, const double2* u, const double2* rho, double2* out, double alpha,
                   int base_kind, cudaStream_t s)
{
    switch (a.logd) {
    case 5: return launch_stage2_t<5>(a, u, rho, out, alpha, base_kind, s);
    case 6: return launch_stage2_t<6>(a, u, rho, out, alpha, base_kind, s);
    default: return false;
    }
}

bool stage2_supported(int logd, int M, int J)
{
    if (logd == 5) return stage2_smem<5>(M, J) <= 227 * 1024;
    if (logd == 6) return stage2_smem<6>(M, J) <= 227 * 1024;
    return false;
}

void launch_entries(const int32_t* edges, const double* acoef, const double* bcoef, const int32_t* bath_off,
                    long long H, int M, int J, int* count, int32_t* slab, int32_t* bath, double* wc, double* wa,
                    cudaStream_t s)
{
    if (H <= 0) return;
    const int block = 128;
    entries_kernel<<<static_cast<unsigned>((H + block - 1) / block), block, 0, s>>>(edges, acoef, bcoef, bath_off, H,
                                                                                   M, J, count, slab, bath, wc, wa);
}

void launch_diag_table(const double* hdiag, const double* vdiag, const double* xi, const double* kappa, int D, int J,
                       double2* T, cudaStream_t s)
{
    const int n = D * D;
    diag_table_kernel<<<(n + 255) / 256, 256, 0, s>>>(hdiag, vdiag, xi, kappa, D, J, T);
}

}  // namespace hx
