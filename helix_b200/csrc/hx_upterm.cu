// Up-coupling term of the tier just below the truncation, element-tiled.
//
// For an ADO n in tier L-1 (L = top tier), the up term of the right-hand side
// is  U_n = -i sum_{m : n+e_m in tier L} delta_{j(m)} X_{n+e_m}  (phi term of
// getdRhoSparse, src/liouville.cu:819-823, for diagonal couplings).  Its 16-
// 18 source slabs lie scattered through the top tier, so gathering them ADO
// by ADO misses L2.  This kernel walks the state tile by tile instead, so
// each top-tier element is fetched from DRAM about once per stage, and the
// stage kernel adds U_n from this buffer instead of gathering the up
// neighbours.

#include <cuda_runtime.h>

#include <cstdint>

#include "hx_internal.h"

namespace hx {

namespace {

constexpr int kWarps = 8;          // warps per CTA
constexpr int kSlotsPerWarp = 4;   // tier L-1 ADOs summed by one warp, one after the other
constexpr int kTile = 32;          // elements per tile (one per lane)

// Launch order is tile-major (blockIdx.y = tile), so the resident CTAs work on
// a narrow band of 32-element tiles and the top-tier data of that band
// (top-tier count x 512 B per tile) stays in L2.  Every mode of a tier L-1
// ADO has its up neighbour in the top tier and the up weight -i delta_j is
// the same for all modes of bath j, so each bath's neighbour slabs are summed
// unweighted and -i delta_j is applied once.  A warp sums its slots side by
// side, so each mode issues kSlotsPerWarp independent loads.
__device__ __forceinline__ void upterm_block(const UpTermArgs& a, int bx, int by, const double2* __restrict__ u,
                                             double2* __restrict__ U)
{
    const int D = 1 << a.logd;
    // elements per stored slab: d^2, or the packed upper triangle
    const long long D2 = a.herm ? herm_elems(a.logd) : static_cast<long long>(D) * D;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const long long e = static_cast<long long>(by) * kTile + lane;
    if (e >= D2) return;
    int r, c;
    if (a.herm) {
        herm_coords(static_cast<int>(e), a.logd, r, c);
    } else {
        r = static_cast<int>(e >> a.logd);
        c = static_cast<int>(e & (D - 1));
    }
    const double2* ue = u + e;
    const int s0 = (bx * kWarps + warp) * kSlotsPerWarp;
    int ns = a.S - s0;
    if (ns <= 0) return;
    ns = ns < kSlotsPerWarp ? ns : kSlotsPerWarp;
    const int32_t* slab[kSlotsPerWarp];
#pragma unroll
    for (int t = 0; t < kSlotsPerWarp; ++t) slab[t] = a.slab + static_cast<long long>(s0 + (t < ns ? t : 0)) * a.M;
    double re[kSlotsPerWarp], im[kSlotsPerWarp];
#pragma unroll
    for (int t = 0; t < kSlotsPerWarp; ++t) re[t] = im[t] = 0.0;
    for (int j = 0; j < a.J; ++j) {
        const double del = __ldg(a.vdiag + j * D + r) - __ldg(a.vdiag + j * D + c);
        if (del == 0.0) continue;
        const int m1 = __ldg(a.bath_off + j + 1);
        double sr[kSlotsPerWarp], si[kSlotsPerWarp];
#pragma unroll
        for (int t = 0; t < kSlotsPerWarp; ++t) sr[t] = si[t] = 0.0;
        for (int m = __ldg(a.bath_off + j); m < m1; ++m) {
            double2 y[kSlotsPerWarp];
#pragma unroll
            for (int t = 0; t < kSlotsPerWarp; ++t)
                y[t] = t < ns ? __ldg(ue + static_cast<long long>(__ldg(slab[t] + m)) * D2) : make_double2(0.0, 0.0);
#pragma unroll
            for (int t = 0; t < kSlotsPerWarp; ++t) {
                sr[t] += y[t].x;
                si[t] += y[t].y;
            }
        }
#pragma unroll
        for (int t = 0; t < kSlotsPerWarp; ++t) {
            re[t] += del * si[t];  // -i del S
            im[t] -= del * sr[t];
        }
    }
#pragma unroll
    for (int t = 0; t < kSlotsPerWarp; ++t)
        if (t < ns) U[static_cast<long long>(s0 + t) * D2 + e] = make_double2(re[t], im[t]);
}

__global__ void __launch_bounds__(kWarps * 32)
    upterm_kernel(UpTermArgs a, const double2* __restrict__ u, double2* __restrict__ U)
{
    upterm_block(a, blockIdx.x, blockIdx.y, u, U);
}

// slot[i] = rank of ADO i among tier L-1 ADOs (or -1); per slot, its up
// entries whose target lies in tier L.  Single CTA, runs once at set-up.
__global__ void upterm_tables_kernel(const int32_t* rows, const int32_t* edges, const int32_t* mode_bath, long long H,
                                     int M, int top, int32_t* slot, int* S_out, int32_t* ado, int* cnt, int32_t* slab,
                                     int32_t* bath)
{
    __shared__ int base;
    __shared__ int warp_sums[32];
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    for (long long i0 = 0; i0 < H; i0 += blockDim.x) {
        const long long i = i0 + threadIdx.x;
        int t = 0;
        if (i < H)
            for (int m = 0; m < M; ++m) t += rows[i * M + m];
        const int flag = (i < H && t == top - 1) ? 1 : 0;
        // block exclusive scan of flag
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        int v = flag;
        for (int o = 1; o < 32; o <<= 1) {
            const int n = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += n;
        }
        if (lane == 31) warp_sums[w] = v;
        __syncthreads();
        if (w == 0) {
            int x = (lane < static_cast<int>(blockDim.x >> 5)) ? warp_sums[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const int n = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += n;
            }
            warp_sums[lane] = x;
        }
        __syncthreads();
        const int excl = base + (w ? warp_sums[w - 1] : 0) + v - flag;
        if (i < H) {
            slot[i] = flag ? excl : -1;
            if (flag) {
                ado[excl] = static_cast<int32_t>(i);
                // a tier L-1 ADO has an up neighbour for every mode (tier L exists)
                for (int m = 0; m < M; ++m) {
                    slab[static_cast<long long>(excl) * M + m] = edges[i * 2 * M + m];
                    bath[static_cast<long long>(excl) * M + m] = mode_bath[m];
                }
                cnt[excl] = M;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) base += warp_sums[(blockDim.x >> 5) - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) *S_out = base;
}

}  // namespace

void launch_upterm(const UpTermArgs& a, const double2* u, double2* U, cudaStream_t s)
{
    if (a.S <= 0) return;
    const long long D2 = a.herm ? herm_elems(a.logd) : 1ll << (2 * a.logd);
    const int per_cta = kWarps * kSlotsPerWarp;
    dim3 grid((a.S + per_cta - 1) / per_cta, static_cast<unsigned>((D2 + kTile - 1) / kTile));
    upterm_kernel<<<grid, kWarps * 32, 0, s>>>(a, u, U);
}

void launch_upterm_tables(const int32_t* rows, const int32_t* edges, const int32_t* mode_bath, long long H, int M,
                          int top, int32_t* slot, int* S_out, int32_t* ado, int* cnt, int32_t* slab, int32_t* bath,
                          cudaStream_t s)
{
    upterm_tables_kernel<<<1, 1024, 0, s>>>(rows, edges, mode_bath, H, M, top, slot, S_out, ado, cnt, slab, bath);
}

}  // namespace hx
