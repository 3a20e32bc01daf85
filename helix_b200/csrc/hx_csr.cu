// Stage kernels for general sparse Hermitian operators (H and every V_j in
// compressed rows), any Hilbert dimension up to 4096, double precision.
//
// The reference validates System::from_sparse but executes only its compiled
// model (src/helix.cpp:166-258,335-347); its right-hand side
// (getdRhoSparse, src/liouville.cu:778-860) applies V through SpMM and
// transposes.  Here the operator products are gathers along CSR rows: for a
// Hermitian operator A,
//   (A X)_rc = sum_{p in row r} A_p X_{col p, c}
//   (X A)_rc = sum_k X_rk A_kc = sum_{p in row c} X_{r, col p} conj(A_p)
// so both sides of a commutator use the rows of A.  As in the flip path
// (hx_flip.cu) each stage runs in two passes:
//   csr_comm_kernel:    B_{j,n} = [V_j, u_n] and A_{j,n} = {V_j, u_n} for
//                       every bath j and ADO n (B for all (j, n), then A)
//   csr_combine_kernel: out_n = base_n + alpha * ( -i[H,u_n] - g_n u_n
//                         - i sum_{m up} B_{j(m), n+e_m}
//                         - i sum_{m down} a_{n,m} B_{j(m), n-e_m}
//                         - sum_j b_{n,j} A_{j, n-e_j0}
//                         + sum_j ((-Xi_j - i kappa_j) V_j B_{j,n} + (Xi_j - i kappa_j) B_{j,n} V_j) )
// the last line being -Xi [V, B] - i kappa {V, B}.  One thread per element;
// the gathered rows and columns of a slab are read through L1/L2.

#include <cuda_runtime.h>

#include <cstdint>

#include "hx_internal.h"

namespace hx {

namespace {

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// a * conj(b)
__device__ __forceinline__ double2 cmulc(double2 a, double2 b)
{
    return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// (A X)_rc and (X A)_rc of operator k for slab X (row-major, d = 2^logd).
struct Sides {
    double2 left, right;
};

__device__ __forceinline__ Sides sides(const CsrArgs& a, int k, const double2* __restrict__ X, int r, int c)
{
    const int D = 1 << a.logd;
    const int32_t* ptr = a.ptr + static_cast<long long>(k) * (D + 1);
    double2 L = make_double2(0.0, 0.0), R = make_double2(0.0, 0.0);
    for (int p = __ldg(ptr + r); p < __ldg(ptr + r + 1); ++p) {
        const double2 v = __ldg(a.val + p);
        const double2 x = __ldg(X + (static_cast<long long>(__ldg(a.col + p)) << a.logd) + c);
        const double2 t = cmul(v, x);
        L.x += t.x;
        L.y += t.y;
    }
    for (int p = __ldg(ptr + c); p < __ldg(ptr + c + 1); ++p) {
        const double2 v = __ldg(a.val + p);
        const double2 x = __ldg(X + (static_cast<long long>(r) << a.logd) + __ldg(a.col + p));
        const double2 t = cmulc(x, v);
        R.x += t.x;
        R.y += t.y;
    }
    return Sides{L, R};
}

__global__ void __launch_bounds__(256) csr_comm_kernel(CsrArgs a, const double2* __restrict__ u, double2* __restrict__ B)
{
    const int D = 1 << a.logd;
    const long long D2 = static_cast<long long>(D) * D;
    const long long HD2 = a.H * D2;
    const long long total = static_cast<long long>(a.J) * HD2;
    for (long long ne = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; ne < HD2;
         ne += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long n = ne >> (2 * a.logd);
        const long long e = ne & (D2 - 1);
        const int r = static_cast<int>(e >> a.logd), c = static_cast<int>(e & (D - 1));
        for (int j = 0; j < a.J; ++j) {
            const Sides s = sides(a, 1 + j, u + n * D2, r, c);
            const long long idx = static_cast<long long>(j) * HD2 + ne;
            B[idx] = make_double2(s.left.x - s.right.x, s.left.y - s.right.y);
            B[total + idx] = make_double2(s.left.x + s.right.x, s.left.y + s.right.y);
        }
    }
}

__global__ void __launch_bounds__(256)
    csr_combine_kernel(CsrArgs a, const double2* __restrict__ u, const double2* __restrict__ B, const double2* rho,
                       double2* out, double alpha, int base_kind)
{
    const int D = 1 << a.logd;
    const long long D2 = static_cast<long long>(D) * D;
    const long long total = a.H * D2;
    const long long HD2 = a.H * D2;
    for (long long idx = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long n = idx >> (2 * a.logd);
        const long long e = idx & (D2 - 1);
        const int r = static_cast<int>(e >> a.logd), c = static_cast<int>(e & (D - 1));
        const double2* un = u + n * D2;
        const double2 x = un[e];
        // -g u - i [H, u]
        const double g = a.gsum[n];
        const Sides h = sides(a, 0, un, r, c);
        const double cr = h.left.x - h.right.x, ci = h.left.y - h.right.y;
        double re = -g * x.x + ci;
        double im = -g * x.y - cr;
        const int32_t* edges = a.edges + n * 2 * a.M;
        for (int j = 0; j < a.J; ++j) {
            const double2* Bj = B + static_cast<long long>(j) * HD2;
            // up and down neighbours: -i B_up, -i a B_down
            double sr = 0.0, si = 0.0;
            for (int m = a.bath_off[j]; m < a.bath_off[j + 1]; ++m) {
                const int up = edges[m];
                if (up < a.H) {
                    const double2 y = __ldg(Bj + static_cast<long long>(up) * D2 + e);
                    sr += y.x;
                    si += y.y;
                }
                const int dn = edges[a.M + m];
                if (dn < a.H) {
                    const double w = a.acoef[n * a.M + m];
                    const double2 y = __ldg(Bj + static_cast<long long>(dn) * D2 + e);
                    sr += w * y.x;
                    si += w * y.y;
                }
            }
            re += si;
            im -= sr;
            // theta2: -b {V_j, u_{n-e_j0}} = -b A_{j, n-e_j0}
            const int dn0 = edges[a.M + a.bath_off[j]];
            if (dn0 < a.H) {
                const double b = a.bcoef[n * a.J + j];
                const double2 y = __ldg(Bj + static_cast<long long>(a.J) * HD2 + static_cast<long long>(dn0) * D2 + e);
                re -= b * y.x;
                im -= b * y.y;
            }
            // -Xi [V, B_n] - i kappa {V, B_n} = (-Xi - i kappa) V B + (Xi - i kappa) B V
            const double xi = a.xi[j], ka = a.counter[j];
            const Sides s = sides(a, 1 + j, Bj + n * D2, r, c);
            re += -xi * s.left.x + ka * s.left.y + xi * s.right.x + ka * s.right.y;
            im += -xi * s.left.y - ka * s.left.x + xi * s.right.y - ka * s.right.x;
        }
        double2 base;
        if (base_kind == kBaseSelf) base = x;
        else if (base_kind == kBaseRho) base = rho[idx];
        else base = make_double2(0.0, 0.0);
        out[idx] = make_double2(base.x + alpha * re, base.y + alpha * im);
    }
}

// out[0] = Re Tr(H rho_0) = Re sum_r sum_{p in row r} H_p rho0_{col p, r}, out[1..2] = Tr rho_0.
__global__ void csr_observables_kernel(const double2* __restrict__ rho0, int logd, const int32_t* __restrict__ ptr,
                                       const int32_t* __restrict__ col, const double2* __restrict__ val, double* out)
{
    const int D = 1 << logd;
    double en = 0.0, tr = 0.0, ti = 0.0;
    for (int r = threadIdx.x; r < D; r += blockDim.x) {
        const double2 dg = rho0[(static_cast<long long>(r) << logd) + r];
        tr += dg.x;
        ti += dg.y;
        for (int p = ptr[r]; p < ptr[r + 1]; ++p) {
            const double2 y = rho0[(static_cast<long long>(col[p]) << logd) + r];
            en += val[p].x * y.x - val[p].y * y.y;
        }
    }
    __shared__ double red[3][256];
    red[0][threadIdx.x] = en;
    red[1][threadIdx.x] = tr;
    red[2][threadIdx.x] = ti;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int q = 0; q < 3; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < 3; ++q) out[q] = red[q][0];
}

unsigned grid_for(long long n)
{
    const long long g = (n + 255) / 256;
    return static_cast<unsigned>(g < 148ll * 64 ? g : 148ll * 64);
}

}  // namespace

void launch_csr_stage(const CsrArgs& a, const double2* u, double2* B, const double2* rho, double2* out, double alpha,
                      int base_kind, cudaStream_t s)
{
    const long long D2 = 1ll << (2 * a.logd);
    csr_comm_kernel<<<grid_for(a.H * D2), 256, 0, s>>>(a, u, B);
    csr_combine_kernel<<<grid_for(a.H * D2), 256, 0, s>>>(a, u, B, rho, out, alpha, base_kind);
}

void launch_observables_csr(const double2* rho0, int logd, const int32_t* ptr, const int32_t* col,
                            const double2* val, double* out, cudaStream_t s)
{
    csr_observables_kernel<<<1, 256, 0, s>>>(rho0, logd, ptr, col, val, out);
}

}  // namespace hx
