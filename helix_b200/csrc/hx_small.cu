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

}  // namespace

size_t small_smem(int logd, int M)
{
    const size_t D = size_t(1) << logd;
    return D * D * sizeof(double2) + sizeof(double) * (2 * D + logd + 4 * M) + sizeof(int) * 4 * M;
}

bool small_supported(int logd, int M, int pauli) { return pauli && logd >= 1 && logd <= 4 && small_smem(logd, M) <= 48 * 1024; }

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
