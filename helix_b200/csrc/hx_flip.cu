// Stage kernels for coupling operators with transverse (spin-flip) parts and
// for any Hilbert dimension up to 4096.
//
// Coupling operators V_j = diag(v_j) + sum_i w_ji sigma_x(i) (the reference's
// compiled model has one collective V = Dlong sum s_z + Dtrans sum_i sigma_x(i),
// src/initialize.cu:95-147).  Commutators then mix elements within a slab:
//
//   [V,X]_rc = (v_r - v_c) X_rc + sum_i w_i (X_{r^2^i,c} - X_{r,c^2^i})
//   {V,X}_rc = (v_r + v_c) X_rc + sum_i w_i (X_{r^2^i,c} + X_{r,c^2^i})
//
// so, as in the reference (getdRhoSparse, src/liouville.cu:778-860), each
// stage runs in two passes:
//   comm_kernel:     B_{j,n} = [V_j, u_n] and A_{j,n} = {V_j, u_n} for every
//                    bath j and ADO n (both from the same flip loads)
//   combine_kernel:  out_n = base_n + alpha * ( -i[H,u_n] - g_n u_n
//                      - i sum_{m up} B_{j(m), n+e_m}
//                      - i sum_{m down} a_{n,m} B_{j(m), n-e_m}
//                      - sum_j b_{n,j} A_{j, n-e_j0}
//                      - sum_j (Xi_j [V_j, B_{j,n}] + i kappa_j {V_j, B_{j,n}}) )
// The buffer holds B for all (j, n), then A for all (j, n).
// One thread per element, flip partners read through L1/L2 (a slab of
// d = 1024 is 16 MB and stays in L2 while its rows are processed).

#include <cuda_runtime.h>

#include <cstdint>

#include "hx_internal.h"

namespace hx {

namespace {

__global__ void __launch_bounds__(256)
    comm_kernel(FlipArgs a, const double2* __restrict__ u, double2* __restrict__ B)
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
        const double2* un = u + n * D2;
        const double2 x = un[e];
        for (int j = 0; j < a.J; ++j) {
            const double vr = a.vdiag[j * D + r], vc = a.vdiag[j * D + c];
            const double del = vr - vc, sum = vr + vc;
            double re = del * x.x, im = del * x.y;
            double ar = sum * x.x, ai = sum * x.y;
            for (int i = 0; i < a.logd; ++i) {
                const double w = a.vflip[j * a.logd + i];
                if (w == 0.0) continue;
                const double2 pr = __ldg(un + (e ^ (static_cast<long long>(1) << (i + a.logd))));
                const double2 pc = __ldg(un + (e ^ (static_cast<long long>(1) << i)));
                re += w * (pr.x - pc.x);
                im += w * (pr.y - pc.y);
                ar += w * (pr.x + pc.x);
                ai += w * (pr.y + pc.y);
            }
            const long long idx = static_cast<long long>(j) * HD2 + ne;
            B[idx] = make_double2(re, im);
            B[total + idx] = make_double2(ar, ai);
        }
    }
}

__global__ void __launch_bounds__(256)
    combine_kernel(FlipArgs a, const double2* __restrict__ u, const double2* __restrict__ B, const double2* rho,
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
        // -g u - i (E_r - E_c) u - i sum_i h_i (u_{r^i,c} - u_{r,c^i})
        const double g = a.gsum[n];
        const double dE = a.hdiag[r] - a.hdiag[c];
        double re = -g * x.x + dE * x.y;
        double im = -g * x.y - dE * x.x;
        {
            double hr = 0.0, hi = 0.0;
            for (int i = 0; i < a.logd; ++i) {
                const double h = a.hflip[i];
                if (h == 0.0) continue;
                const double2 pr = __ldg(un + (e ^ (static_cast<long long>(1) << (i + a.logd))));
                const double2 pc = __ldg(un + (e ^ (static_cast<long long>(1) << i)));
                hr += h * (pr.x - pc.x);
                hi += h * (pr.y - pc.y);
            }
            re += hi;
            im -= hr;
        }
        const int32_t* edges = a.edges + n * 2 * a.M;
        for (int j = 0; j < a.J; ++j) {
            const double2* Bj = B + static_cast<long long>(j) * HD2;
            const double vr = a.vdiag[j * D + r], vc = a.vdiag[j * D + c];
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
            // Xi and counter: -Xi [V, B_n] - i kappa {V, B_n}
            const double xi = a.xi[j], ka = a.counter[j];
            const double2* Bn = Bj + n * D2;
            const double2 y = Bn[e];
            const double cr = -xi * (vr - vc), ci = -ka * (vr + vc);  // coefficient cr + i ci
            re += cr * y.x - ci * y.y;
            im += cr * y.y + ci * y.x;
            for (int i = 0; i < a.logd; ++i) {
                const double w = a.vflip[j * a.logd + i];
                if (w == 0.0) continue;
                const double2 pr = __ldg(Bn + (e ^ (static_cast<long long>(1) << (i + a.logd))));
                const double2 pc = __ldg(Bn + (e ^ (static_cast<long long>(1) << i)));
                // w [(-xi - i ka) B_row + (xi - i ka) B_col]
                re += w * (-xi * pr.x + ka * pr.y + xi * pc.x + ka * pc.y);
                im += w * (-xi * pr.y - ka * pr.x + xi * pc.y - ka * pc.x);
            }
        }
        double2 base;
        if (base_kind == kBaseSelf) base = x;
        else if (base_kind == kBaseRho) base = rho[idx];
        else base = make_double2(0.0, 0.0);
        out[idx] = make_double2(base.x + alpha * re, base.y + alpha * im);
    }
}

}  // namespace

void launch_flip_stage(const FlipArgs& a, const double2* u, double2* B, const double2* rho, double2* out,
                       double alpha, int base_kind, cudaStream_t s)
{
    const long long D2 = 1ll << (2 * a.logd);
    const long long nc = a.H * D2;
    auto grid_for = [](long long n) {
        long long g = (n + 255) / 256;
        return static_cast<unsigned>(g < 148ll * 64 ? g : 148ll * 64);
    };
    comm_kernel<<<grid_for(nc), 256, 0, s>>>(a, u, B);
    combine_kernel<<<grid_for(nc), 256, 0, s>>>(a, u, B, rho, out, alpha, base_kind);
}

}  // namespace hx
