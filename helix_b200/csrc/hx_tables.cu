// Hierarchy index and neighbour tables, built on the device.
//
// The reference builds them on the host: rows by recursion in lexicographic
// order with mode 0 most significant and sum(n) < maxLevel
// (appendHierarchyRows, src/initialize_detail.h:174-214), edges by an
// O(H^2 M) search (buildHierarchyEdges, src/initialize_detail.h:234-269).
// Here one thread per ADO unranks its index vector from its position and
// finds its neighbours by ranking n +- e_k, both by counting lattice points:
// cnt(m, s) = number of length-m vectors with sum < s = C(m + s - 1, m).
// The output is bit-identical to the reference tables (same order, same
// sentinel H).

#include <cuda_runtime.h>

#include <vector>

#include "hx_internal.h"

namespace hx {

namespace {

constexpr int kMaxBinomN = 192;

// binomial table in global memory: binom[n * (kMaxK + 1) + k], n <= M + D, k <= M
struct Binom {
    const unsigned long long* t;
    int kcols;
    __device__ unsigned long long operator()(int n, int k) const
    {
        if (k < 0 || n < 0 || k > n) return 0ull;
        return t[n * kcols + k];
    }
};

// number of length-m non-negative vectors with sum < s
__device__ inline unsigned long long lattice_count(const Binom& C, int m, int s)
{
    if (s <= 0) return 0ull;
    if (m == 0) return 1ull;
    return C(m + s - 1, m);
}

__global__ void tables_kernel(Binom C, int M, int D, long long H, int32_t* rows, int32_t* edges)
{
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= H) return;
    int n[kMaxModes];
    // unrank
    unsigned long long rem = static_cast<unsigned long long>(i);
    int budget = D;
    int total = 0;
    for (int p = 0; p < M; ++p) {
        int v = 0;
        for (;;) {
            const unsigned long long blk = lattice_count(C, M - p - 1, budget - v);
            if (rem < blk || blk == 0ull) break;
            rem -= blk;
            ++v;
        }
        n[p] = v;
        budget -= v;
        total += v;
    }
    for (int p = 0; p < M; ++p) rows[i * M + p] = n[p];

    // rank of n with mode k shifted by delta (+1 / -1)
    auto rank_shifted = [&](int k, int delta) -> long long {
        unsigned long long r = 0ull;
        int s = D;
        for (int p = 0; p < M; ++p) {
            const int np = n[p] + (p == k ? delta : 0);
            for (int v = 0; v < np; ++v) r += lattice_count(C, M - p - 1, s - v);
            s -= np;
        }
        return static_cast<long long>(r);
    };
    for (int k = 0; k < M; ++k) {
        long long up = H, dn = H;
        if (total + 1 < D) up = rank_shifted(k, +1);
        if (n[k] > 0) dn = rank_shifted(k, -1);
        edges[i * 2 * M + k] = static_cast<int32_t>(up);
        edges[i * 2 * M + M + k] = static_cast<int32_t>(dn);
    }
}

// Per-ADO weights of the fused right-hand side.  With one bath they equal the
// reference coefficient table of initSparse (src/liouville.cu:723-743):
//   a_{n,m} (k = 0) = (nu_0 n_0) * theta_c      [theta, KThetaCommutate]
//   a_{n,m} (k >= 1) = (nu_k n_k) * phi_k       [psi, KPhi]
//   b_{n,j}          = (nu_0 n_0) * theta_a     [theta2, KThetaAntiCommutate]
//   g_n              = sum_m nu_m n_m           [sigma]
__global__ void coefficients_kernel(const int32_t* rows, long long H, int M, int J,
                                    const int32_t* mode_bath, const int32_t* mode_k,
                                    const double* nu, const double* theta_c, const double* theta_a,
                                    const double* phi, const int32_t* bath_off, double* acoef,
                                    double* bcoef, double* gsum)
{
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= H) return;
    const int32_t* n = rows + i * M;
    double g = 0.0;
    for (int j = 0; j < J; ++j) {
        double s = 0.0;
        for (int m = bath_off[j]; m < bath_off[j + 1]; ++m) s += nu[m] * n[m];
        g += s;
    }
    gsum[i] = g;
    for (int m = 0; m < M; ++m) {
        const int j = mode_bath[m];
        const int k = mode_k[m];
        const double w = nu[m] * n[m];
        acoef[i * M + m] = (k == 0) ? w * theta_c[j] : w * phi[m];
    }
    for (int j = 0; j < J; ++j) {
        const int m0 = bath_off[j];
        bcoef[i * J + j] = (nu[m0] * n[m0]) * theta_a[j];
    }
}

}  // namespace

int build_tables_device(int M, int D, long long H, int32_t* d_rows, int32_t* d_edges, cudaStream_t s)
{
    if (M > kMaxModes) return fail(HX_ERR_UNSUPPORTED_HIERARCHY, "too many modes for the device table builder");
    const int nmax = M + D + 1;
    if (nmax > kMaxBinomN) return fail(HX_ERR_UNSUPPORTED_HIERARCHY, "hierarchy too deep for the table builder");
    const int kcols = M + 1;
    std::vector<unsigned long long> host(static_cast<size_t>(nmax) * kcols, 0ull);
    for (int n = 0; n < nmax; ++n)
        for (int k = 0; k <= M && k <= n; ++k) host[n * kcols + k] = binom_u64(n, k);
    unsigned long long* dev = nullptr;
    HX_CUDA_TRY(cudaMallocAsync(&dev, host.size() * sizeof(unsigned long long), s));
    cudaError_t e = cudaMemcpyAsync(dev, host.data(), host.size() * sizeof(unsigned long long),
                                    cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && H > 0) {
        const int block = 128;
        const long long grid = (H + block - 1) / block;
        tables_kernel<<<static_cast<unsigned>(grid), block, 0, s>>>(Binom{dev, kcols}, M, D, H, d_rows, d_edges);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // host vector must outlive the copy
    cudaFreeAsync(dev, s);
    if (e != cudaSuccess) return cuda_fail(e, "hierarchy table kernel");
    return HX_OK;
}

void launch_tables_with_binomials(const unsigned long long* d_binom, int kcols, int M, int D, long long H,
                                  int32_t* d_rows, int32_t* d_edges, cudaStream_t s)
{
    if (H <= 0) return;
    const int block = 128;
    const long long grid = (H + block - 1) / block;
    tables_kernel<<<static_cast<unsigned>(grid), block, 0, s>>>(Binom{d_binom, kcols}, M, D, H, d_rows, d_edges);
}

void launch_coefficients(const int32_t* rows, long long H, int M, int J, const int32_t* mode_bath,
                         const int32_t* mode_k, const double* nu, const double* theta_c,
                         const double* theta_a, const double* phi, const int32_t* bath_off,
                         double* acoef, double* bcoef, double* gsum, cudaStream_t s)
{
    if (H <= 0) return;
    const int block = 128;
    const long long grid = (H + block - 1) / block;
    coefficients_kernel<<<static_cast<unsigned>(grid), block, 0, s>>>(
        rows, H, M, J, mode_bath, mode_k, nu, theta_c, theta_a, phi, bath_off, acoef, bcoef, gsum);
}

}  // namespace hx
