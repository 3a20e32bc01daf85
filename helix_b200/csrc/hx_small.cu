// Stage kernel for small slabs (d = 8, 16) with sigma_z couplings: the C1
// workload's path.
//
// Same mathematics as stage_kernel (hx_stage.cu): one launch evaluates
// out_n = base_n + alpha L(u)_n for every ADO n, L being the reference
// right-hand side (getdRhoSparse, src/liouville.cu:749-869).  At d = 16 a
// slab is 256 elements (4 KB), so a stage is bound by the latency of its
// gathers, not by bandwidth.  The generic kernel walks baths and modes and
// waits on each neighbour read in turn; here every ADO carries the compacted
// neighbour entry list of the fused kernels (slab, spin bit, commutator and
// anti-commutator weight; up neighbours of every tier included), and each
// thread issues the reads of kBatch entries before it consumes any, so a
// stage costs a few L2 round trips instead of one per entry.
//
//  * one CTA per ADO, one thread per element (d^2 threads, at least a warp);
//  * the slab goes to shared memory once for the transverse-field flips;
//  * diagonal term from two d-entry tables: Re T = -4 sum_j xi_j
//    [bit_j(r) != bit_j(c)] (over r ^ c) and Im T = -(E_r - E_c);
//  * sigma_z weights from the index bits, as in the fused kernels.

#include <cuda_runtime.h>

#include <cstdint>

#include "hx_internal.h"

namespace hx {

namespace {

constexpr int kBatch = 8;  // neighbour reads in flight per thread

template <int LOGD>
__global__ void __launch_bounds__((1 << (2 * LOGD)) < 32 ? 32 : (1 << (2 * LOGD)))
    small_kernel(FusedArgs a, const double2* __restrict__ u, const double2* rho, double2* out, double alpha,
                 int base_kind)
{
    constexpr int D = 1 << LOGD, D2 = D * D;
    extern __shared__ __align__(16) unsigned char smem[];
    double2* sx = reinterpret_cast<double2*>(smem);  // [D2]
    double* sE = reinterpret_cast<double*>(sx + D2);  // [D]
    double* sX = sE + D;                              // [D]
    double* sH = sX + D;                              // [LOGD]
    double* sWc = sH + LOGD;                          // [2M]
    double* sWa = sWc + 2 * a.M;                      // [2M]
    int* sSlab = reinterpret_cast<int*>(sWa + 2 * a.M);
    int* sBit = sSlab + 2 * a.M;

    const int tid = threadIdx.x;
    const long long n = a.order ? static_cast<long long>(a.order[blockIdx.x]) : static_cast<long long>(blockIdx.x);
    const bool active = tid < D2;
    const int e = active ? tid : 0;
    const int r = e >> LOGD, c = e & (D - 1);
    const double2 x = active ? __ldg(u + n * D2 + e) : make_double2(0.0, 0.0);
    if (active) sx[e] = x;
    const int Q = a.ent_count[n];
    for (int q = tid; q < Q; q += blockDim.x) {
        const long long src = n * 2 * a.M + q;
        sSlab[q] = a.ent_slab[src];
        sBit[q] = a.vbit[a.ent_bath[src] & 0xffff];
        sWc[q] = a.ent_wc[src];
        sWa[q] = a.ent_wa[src];
    }
    if (tid < D) {
        sE[tid] = a.hdiag[tid];
        double s = 0.0;
        for (int j = 0; j < a.J; ++j)
            if ((tid >> a.vbit[j]) & 1) s += a.xi[j];
        sX[tid] = 4.0 * s;
    }
    if (tid < LOGD) sH[tid] = a.hflip[tid];
    const double g = a.gsum[n];
    __syncthreads();
    if (!active) return;

    // diagonal and transverse field
    double hr = 0.0, hi = 0.0;
#pragma unroll
    for (int b = 0; b < LOGD; ++b) {
        const double2 rp = sx[e ^ (D << b)];
        const double2 cp = sx[e ^ (1 << b)];
        hr += sH[b] * (rp.x - cp.x);
        hi += sH[b] * (rp.y - cp.y);
    }
    const double tr = -sX[r ^ c] - g;
    const double ti = sE[c] - sE[r];
    double2 acc = make_double2(tr * x.x - ti * x.y + hi, tr * x.y + ti * x.x - hr);

    // neighbour entries, kBatch reads in flight
    const double2* ue = u + e;
    for (int q0 = 0; q0 < Q; q0 += kBatch) {
        double2 y[kBatch];
#pragma unroll
        for (int i = 0; i < kBatch; ++i) {
            const int q = q0 + i;
            y[i] = make_double2(0.0, 0.0);
            if (q < Q) {
                const int bit = sBit[q];
                const bool same = ((r >> bit) & 1) == ((c >> bit) & 1);
                if (same ? sWa[q] != 0.0 : sWc[q] != 0.0) y[i] = __ldg(ue + static_cast<long long>(sSlab[q]) * D2);
            }
        }
#pragma unroll
        for (int i = 0; i < kBatch; ++i) {
            const int q = q0 + i;
            if (q < Q) {
                const int bit = sBit[q];
                const int br = (r >> bit) & 1;
                const bool same = br == ((c >> bit) & 1);
                const double w2 = 2.0 * (same ? sWa[q] : sWc[q]);
                const double w = br ? -w2 : w2;
                acc.x += w * (same ? y[i].x : -y[i].y);
                acc.y += w * (same ? y[i].y : y[i].x);
            }
        }
    }

    double2 base = make_double2(0.0, 0.0);
    if (base_kind == kBaseSelf) base = x;
    else if (base_kind == kBaseRho) base = __ldcs(rho + n * D2 + e);
    __stcs(out + n * D2 + e, make_double2(base.x + alpha * acc.x, base.y + alpha * acc.y));
}

template <int LOGD>
void launch_small_t(const FusedArgs& a, const double2* u, const double2* rho, double2* out, double alpha, int base,
                    cudaStream_t s)
{
    constexpr int D = 1 << LOGD, D2 = D * D;
    const int threads = D2 < 32 ? 32 : D2;
    const size_t smem = small_smem(LOGD, a.M);
    small_kernel<LOGD><<<static_cast<unsigned>(a.H), threads, smem, s>>>(a, u, rho, out, alpha, base);
}

// Grid barrier of small_step_kernel: every CTA is resident (cooperative
// launch).  One arrival counter, zero when a launch begins: barrier k of the
// launch waits until it reaches (k + 1) G.  The block's writes are ordered
// before thread 0's arrival by the block barrier and a GPU-scope fence; the
// wait polls the counter with acquire loads, bounded.  After its last stage
// every CTA arrives once more and the last to do so puts the counter back to
// zero, so no host-side count is involved (a captured launch replays
// correctly).  Returns false when the wait ran out.
__device__ __forceinline__ bool grid_barrier(unsigned* count, unsigned target, unsigned max_polls)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        __threadfence();
        atomicAdd(count, 1u);
        uint32_t it = 0;
        while (true) {
            unsigned v;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(count) : "memory");
            if (static_cast<int>(v - target) >= 0) break;
            if (++it > max_polls) {
                ok = 0;
                break;
            }
            __nanosleep(20);
        }
    }
    __syncthreads();
    return ok != 0;
}

// One whole integrator step (all m Horner stages) for small slabs in one
// cooperative launch: the CTAs stay resident across the stages, each owning
// up to kStepPer ADOs, and a grid barrier separates the stages.  Per stage and
// owned ADO the arithmetic is small_kernel's, in the same order, so the
// results are the same bits; what goes away is a launch per stage, the
// reloading of the per-ADO tables, and the reloading of the own slab: a
// thread keeps its element of rho (the Horner base) and of the stage input in
// registers.  Neighbour elements are read through L2 (ld.global.cg: the
// buffers change between stages inside the launch).
constexpr int kStepPer = 4;

// MAXPER = 1: one ADO per CTA, registers capped so that four 256-thread CTAs
// fit on an SM; MAXPER = kStepPer: up to four ADOs per CTA, two CTAs per SM.
template <int LOGD, int MAXPER>
__global__ void __launch_bounds__((1 << (2 * LOGD)) < 32 ? 32 : (1 << (2 * LOGD)), MAXPER == 1 ? 4 : 2)
    small_step_kernel(FusedArgs a, double2* rho, double2* ua, double2* ub, double dt, int order, int per,
                      unsigned* gcount, StepWait w)
{
    constexpr int D = 1 << LOGD, D2 = D * D;
    extern __shared__ __align__(16) unsigned char smem[];
    double2* sx = reinterpret_cast<double2*>(smem);  // [D2] the slab of the ADO in hand
    double* sE = reinterpret_cast<double*>(sx + D2);  // [D]
    double* sX = sE + D;                              // [D]
    double* sH = sX + D;                              // [LOGD]
    double* sWc = sH + LOGD;                          // [per][2M]
    double* sWa = sWc + per * 2 * a.M;                // [per][2M]
    int* sSlab = reinterpret_cast<int*>(sWa + per * 2 * a.M);
    int* sBit = sSlab + per * 2 * a.M;
    int* sQ = sBit + per * 2 * a.M;                   // [per]

    const int tid = threadIdx.x;
    const bool active = tid < D2;
    const int e = active ? tid : 0;
    const int r = e >> LOGD, c = e & (D - 1);
    const unsigned G = gridDim.x;
    long long nn[MAXPER];
    double g[MAXPER];
    double2 base[MAXPER], x[MAXPER];
#pragma unroll
    for (int j = 0; j < MAXPER; ++j) {
        const long long n = static_cast<long long>(blockIdx.x) + static_cast<long long>(j) * G;
        nn[j] = (j < per && n < a.H) ? n : -1;
        g[j] = 0.0;
        base[j] = x[j] = make_double2(0.0, 0.0);
        if (nn[j] >= 0) {
            if (active) base[j] = x[j] = __ldcg(rho + nn[j] * D2 + e);
            g[j] = a.gsum[nn[j]];
            const int Q = a.ent_count[nn[j]];
            if (tid == 0) sQ[j] = Q;
            for (int q = tid; q < Q; q += blockDim.x) {
                const long long src = nn[j] * 2 * a.M + q;
                sSlab[j * 2 * a.M + q] = a.ent_slab[src];
                sBit[j * 2 * a.M + q] = a.vbit[a.ent_bath[src] & 0xffff];
                sWc[j * 2 * a.M + q] = a.ent_wc[src];
                sWa[j * 2 * a.M + q] = a.ent_wa[src];
            }
        }
    }
    if (tid < D) {
        sE[tid] = a.hdiag[tid];
        double sxs = 0.0;
        for (int j = 0; j < a.J; ++j)
            if ((tid >> a.vbit[j]) & 1) sxs += a.xi[j];
        sX[tid] = 4.0 * sxs;
    }
    if (tid < LOGD) sH[tid] = a.hflip[tid];

    double2* bufs[2] = {ua, ub};
    const double2* in = rho;
    for (int st = 1; st <= order; ++st) {
        const double alpha = dt / static_cast<double>(order - st + 1);
        double2* out = (st == order) ? rho : bufs[(st - 1) & 1];
#pragma unroll
        for (int j = 0; j < MAXPER; ++j) {
            if (nn[j] < 0) continue;  // uniform across the CTA
            __syncthreads();          // the previous ADO's flips are read; tables are in place
            if (active) sx[e] = x[j];
            __syncthreads();
            if (!active) continue;
            double hr = 0.0, hi = 0.0;
#pragma unroll
            for (int b = 0; b < LOGD; ++b) {
                const double2 rp = sx[e ^ (D << b)];
                const double2 cp = sx[e ^ (1 << b)];
                hr += sH[b] * (rp.x - cp.x);
                hi += sH[b] * (rp.y - cp.y);
            }
            const double tr = -sX[r ^ c] - g[j];
            const double ti = sE[c] - sE[r];
            double2 acc = make_double2(tr * x[j].x - ti * x[j].y + hi, tr * x[j].y + ti * x[j].x - hr);
            const int Q = sQ[j];
            const int* slab = sSlab + j * 2 * a.M;
            const int* bits = sBit + j * 2 * a.M;
            const double* wcs = sWc + j * 2 * a.M;
            const double* was = sWa + j * 2 * a.M;
            const double2* ue = in + e;
            for (int q0 = 0; q0 < Q; q0 += kBatch) {
                double2 y[kBatch];
#pragma unroll
                for (int i = 0; i < kBatch; ++i) {
                    const int q = q0 + i;
                    y[i] = make_double2(0.0, 0.0);
                    if (q < Q) {
                        const int bit = bits[q];
                        const bool same = ((r >> bit) & 1) == ((c >> bit) & 1);
                        if (same ? was[q] != 0.0 : wcs[q] != 0.0) y[i] = __ldcg(ue + static_cast<long long>(slab[q]) * D2);
                    }
                }
#pragma unroll
                for (int i = 0; i < kBatch; ++i) {
                    const int q = q0 + i;
                    if (q < Q) {
                        const int bit = bits[q];
                        const int br = (r >> bit) & 1;
                        const bool same = br == ((c >> bit) & 1);
                        const double w2 = 2.0 * (same ? was[q] : wcs[q]);
                        const double w = br ? -w2 : w2;
                        acc.x += w * (same ? y[i].x : -y[i].y);
                        acc.y += w * (same ? y[i].y : y[i].x);
                    }
                }
            }
            const double2 o = make_double2(base[j].x + alpha * acc.x, base[j].y + alpha * acc.y);
            out[nn[j] * D2 + e] = o;
            x[j] = o;
        }
        if (st < order && !grid_barrier(gcount, static_cast<unsigned>(st) * G + w.skew, w.max_polls)) {
            if (tid == 0) atomicExch(a.error_flag, 1);
            return;
        }
        in = out;
    }
    // every CTA has passed every barrier: the last one to get here resets the counter for the next launch
    if (tid == 0 && atomicAdd(gcount, 1u) == static_cast<unsigned>(order) * G - 1u) atomicExch(gcount, 0u);
}

template <int LOGD, int MAXPER>
int launch_small_step_v(const FusedArgs& a, double2* rho, double2* ua, double2* ub, double dt, int order,
                        unsigned* gcount, cudaStream_t s, bool dry, StepWait w)
{
    // 1 launched (or would launch, dry), 0 the ADOs do not fit (try the next form), -1 refused
    constexpr int D2 = 1 << (2 * LOGD);
    const int threads = D2 < 32 ? 32 : D2;
    static int capacity[64][MAXPER + 1] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return -1;
    for (int per = (MAXPER == 1 ? 1 : 2); per <= MAXPER; ++per) {
        const size_t smem = small_step_smem(LOGD, a.M, per);
        if (smem > 48 * 1024) return -1;
        if (capacity[dev][per] == 0) {
            int blocks = 0, sms = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, small_step_kernel<LOGD, MAXPER>, threads,
                                                              smem) != cudaSuccess ||
                cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
                return -1;
            capacity[dev][per] = blocks * sms > 0 ? blocks * sms : -1;
        }
        if (capacity[dev][per] < 0) return -1;
        const long long grid = (a.H + per - 1) / per;
        if (grid > capacity[dev][per]) continue;
        if (dry) return 1;
        FusedArgs args = a;
        int per_arg = per;
        StepWait wait = w;
        void* params[] = {&args, &rho, &ua, &ub, &dt, &order, &per_arg, &gcount, &wait};
        return cudaLaunchCooperativeKernel(reinterpret_cast<void*>(small_step_kernel<LOGD, MAXPER>),
                                           dim3(static_cast<unsigned>(grid)), dim3(threads), params, smem,
                                           s) == cudaSuccess
                   ? 1
                   : -1;
    }
    return 0;
}

template <int LOGD>
int launch_small_step_t(const FusedArgs& a, double2* rho, double2* ua, double2* ub, double dt, int order,
                        unsigned* gcount, cudaStream_t s, bool dry, StepWait w)
{
    const int r1 = launch_small_step_v<LOGD, 1>(a, rho, ua, ub, dt, order, gcount, s, dry, w);
    if (r1 != 0) return r1;
    return launch_small_step_v<LOGD, kStepPer>(a, rho, ua, ub, dt, order, gcount, s, dry, w);
}

}  // namespace

size_t small_smem(int logd, int M)
{
    const size_t D = size_t(1) << logd;
    return D * D * sizeof(double2) + sizeof(double) * (2 * D + logd + 4 * M) + sizeof(int) * 4 * M;
}

bool small_supported(int logd, int M, int pauli) { return pauli && logd >= 1 && logd <= 4 && small_smem(logd, M) <= 48 * 1024; }

size_t small_step_smem(int logd, int M, int per)
{
    const size_t D = size_t(1) << logd;
    return D * D * sizeof(double2) + sizeof(double) * (2 * D + logd + 4 * M * per) + sizeof(int) * (4 * M * per + per);
}

int launch_small_step(const FusedArgs& a, double2* rho, double2* ua, double2* ub, double dt, int order,
                      unsigned* gcount, cudaStream_t s, bool dry, StepWait w)
{
    if (order < 2) return 0;  // order 1 writes rho while neighbours read it
    switch (a.logd) {
    case 1: return launch_small_step_t<1>(a, rho, ua, ub, dt, order, gcount, s, dry, w);
    case 2: return launch_small_step_t<2>(a, rho, ua, ub, dt, order, gcount, s, dry, w);
    case 3: return launch_small_step_t<3>(a, rho, ua, ub, dt, order, gcount, s, dry, w);
    case 4: return launch_small_step_t<4>(a, rho, ua, ub, dt, order, gcount, s, dry, w);
    default: return 0;
    }
}

bool launch_small(const FusedArgs& a, const double2* u, const double2* rho, double2* out, double alpha, int base_kind,
                  cudaStream_t s)
{
    switch (a.logd) {
    case 1: launch_small_t<1>(a, u, rho, out, alpha, base_kind, s); return true;
    case 2: launch_small_t<2>(a, u, rho, out, alpha, base_kind, s); return true;
    case 3: launch_small_t<3>(a, u, rho, out, alpha, base_kind, s); return true;
    case 4: launch_small_t<4>(a, u, rho, out, alpha, base_kind, s); return true;
    default: return false;
    }
}

}  // namespace hx
