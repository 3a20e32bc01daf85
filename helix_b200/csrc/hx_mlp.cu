// Learned closure of the hierarchy: a small MLP in BF16 with FP32
// accumulation, its training kernels, and its use inside the propagator.
//
// Network: x (the 2 d^2 reals of an ADO of the top tier, scaled, and a
// one-hot mode index) -> Linear(in, hidden) -> GELU -> Linear(hidden, hidden)
// -> GELU -> Linear(hidden, 2 d^2) = the scaled prediction of its up
// neighbour in the next tier, which the truncated hierarchy drops.  Weights
// are kept in FP32 (Adam master copy) and used in BF16 by the GEMMs.
//
// GEMM: C = op(A) op(B), BF16 operands, FP32 accumulation on the tensor cores
// (WMMA 16x16x16 fragments), 64x64 tiles staged in shared memory, fused
// epilogues (bias + GELU keeping the pre-activation, bias, plain, GELU
// backward).  Training: MSE loss, backward pass, Adam, all on the device.
// The training set lives on the device: harvest kernels copy, from a deep
// (fine) hierarchy's state, the top-tier ADOs of the truncated (coarse)
// hierarchy and their up neighbours.
//
// No counterpart in the reference, which truncates the hierarchy at
// Param::JMax (src/parameters.cu:31, src/initialize_detail.h:196-213).

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <mma.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <new>
#include <vector>

#include "hx_internal.h"

using hx::fail;
using bf16 = __nv_bfloat16;

namespace hx {

namespace {

constexpr int BM = 64, BN = 64, BK = 32, GT = 128;

enum Epi : int { kEpiBiasGelu = 0, kEpiBias = 1, kEpiStore = 2, kEpiGeluBack = 3 };

struct GemmOut {
    const float* bias;   // [N]
    float* outf;         // FP32 result (pre-activation for kEpiBiasGelu)
    bf16* outh;          // BF16 result (GELU output, or dZ for kEpiGeluBack)
    const float* aux;    // pre-activation Z for kEpiGeluBack
    int ldo;
};

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }

__device__ __forceinline__ float gelu_grad(float z)
{
    const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
    return cdf + z * pdf;
}

// C[M x N] = op(A) op(B); op(A) = A (row-major M x K, lda) or A^T (A stored K x M);
// op(B) = B (row-major K x N, ldb) or B^T (B stored N x K).  Four warps, each a 32 x 32 block.
template <bool TA, bool TB, int EPI>
__global__ void __launch_bounds__(GT)
    gemm_kernel(int M, int N, int K, const bf16* __restrict__ A, int lda, const bf16* __restrict__ B, int ldb,
                GemmOut o)
{
    using namespace nvcuda;
    __shared__ __align__(32) bf16 sA[BM][BK + 8];
    __shared__ __align__(32) bf16 sB[BK][BN + 8];
    __shared__ __align__(32) float sC[BM][BN + 4];
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int warp = threadIdx.x >> 5;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[2][2];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) wmma::fill_fragment(acc[i][j], 0.0f);
    const bf16 zero = __float2bfloat16(0.0f);
    for (int k0 = 0; k0 < K; k0 += BK) {
        for (int idx = threadIdx.x; idx < BM * BK; idx += GT) {
            int mm, kk;
            if (!TA) {
                mm = idx / BK;
                kk = idx % BK;
            } else {
                kk = idx / BM;
                mm = idx % BM;
            }
            const int gm = m0 + mm, gk = k0 + kk;
            bf16 v = zero;
            if (gm < M && gk < K)
                v = TA ? A[static_cast<long long>(gk) * lda + gm] : A[static_cast<long long>(gm) * lda + gk];
            sA[mm][kk] = v;
        }
        for (int idx = threadIdx.x; idx < BK * BN; idx += GT) {
            int kk, nn;
            if (!TB) {
                kk = idx / BN;
                nn = idx % BN;
            } else {
                nn = idx / BK;
                kk = idx % BK;
            }
            const int gn = n0 + nn, gk = k0 + kk;
            bf16 v = zero;
            if (gn < N && gk < K)
                v = TB ? B[static_cast<long long>(gn) * ldb + gk] : B[static_cast<long long>(gk) * ldb + gn];
            sB[kk][nn] = v;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; kk += 16) {
            wmma::fragment<wmma::matrix_a, 16, 16, 16, bf16, wmma::row_major> fa[2];
            wmma::fragment<wmma::matrix_b, 16, 16, 16, bf16, wmma::row_major> fb[2];
#pragma unroll
            for (int i = 0; i < 2; ++i) wmma::load_matrix_sync(fa[i], &sA[wm + 16 * i][kk], BK + 8);
#pragma unroll
            for (int j = 0; j < 2; ++j) wmma::load_matrix_sync(fb[j], &sB[kk][wn + 16 * j], BN + 8);
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j) wmma::mma_sync(acc[i][j], fa[i], fb[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
            wmma::store_matrix_sync(&sC[wm + 16 * i][wn + 16 * j], acc[i][j], BN + 4, wmma::mem_row_major);
    __syncthreads();
    for (int idx = threadIdx.x; idx < BM * BN; idx += GT) {
        const int mm = idx / BN, nn = idx % BN;
        const int gm = m0 + mm, gn = n0 + nn;
        if (gm >= M || gn >= N) continue;
        const float v = sC[mm][nn];
        const long long off = static_cast<long long>(gm) * o.ldo + gn;
        if (EPI == kEpiBiasGelu) {
            const float z = v + o.bias[gn];
            o.outf[off] = z;
            o.outh[off] = __float2bfloat16(gelu(z));
        } else if (EPI == kEpiBias) {
            o.outf[off] = v + o.bias[gn];
        } else if (EPI == kEpiStore) {
            o.outf[off] = v;
        } else {
            o.outh[off] = __float2bfloat16(v * gelu_grad(o.aux[off]));
            if (o.outf) o.outf[off] = v * gelu_grad(o.aux[off]);
        }
    }
}

// Scratch of the tensor-core path: K-major copies of operands stored the other
// way round (hx_tcgemm.cu computes A B^T with both K-major), and its error word.
struct TcScratch {
    bf16* a = nullptr;
    bf16* b = nullptr;
    size_t a_elems = 0, b_elems = 0;
    int* err = nullptr;
};

bool tc_enabled()
{
    static const bool v = [] {
        const char* e = std::getenv("HX_TC_GEMM");
        return !(e && e[0] == '0');
    }();
    return v;
}

inline int round8(int x) { return (x + 7) & ~7; }

// C[M x N] = op(A) op(B): on the tensor cores (tcgen05, hx_tcgemm.cu) when the
// operands allow it, the transposed layouts first copied K-major into the
// scratch; otherwise the WMMA kernel above.
template <bool TA, bool TB, int EPI>
void gemm(int M, int N, int K, const bf16* A, int lda, const bf16* B, int ldb, const GemmOut& o, cudaStream_t s,
          TcScratch* ts = nullptr)
{
    if (ts && tc_enabled()) {
        const bf16* a = A;
        const bf16* b = B;
        int la = lda, lb = ldb;
        bool ok = true;
        if (TA) {  // A stored K x M
            la = round8(K);
            ok = ok && static_cast<size_t>(M) * la <= ts->a_elems;
            if (ok) launch_transpose_bf16(A, K, M, lda, ts->a, la, s);
            a = ts->a;
        }
        if (!TB) {  // B stored K x N
            lb = round8(K);
            ok = ok && static_cast<size_t>(N) * lb <= ts->b_elems;
            if (ok) launch_transpose_bf16(B, K, N, ldb, ts->b, lb, s);
            b = ts->b;
        }
        const TcGemmOut to{EPI, o.bias, o.outf, o.outh, o.aux, o.ldo};
        if (ok && tc_gemm(M, N, K, a, la, b, lb, to, ts->err, s)) return;
    }
    dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
    gemm_kernel<TA, TB, EPI><<<grid, GT, 0, s>>>(M, N, K, A, lda, B, ldb, o);
}

// column sums of an FP32 matrix [rows x cols] (bias gradients) in a fixed
// order: block (32, 8) per 32 columns, thread (tx, ty) sums rows ty, ty + 8,
// ... of column tx (coalesced), then the 8 partial sums are added in order
__global__ void colsum_kernel(const float* __restrict__ x, int rows, int cols, int ld, float* out)
{
    __shared__ float part[8][33];
    const int c = blockIdx.x * 32 + threadIdx.x;
    float s = 0.f;
    if (c < cols)
        for (int r = threadIdx.y; r < rows; r += 8) s += x[static_cast<long long>(r) * ld + c];
    part[threadIdx.y][threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.y == 0 && c < cols) {
        float t = 0.f;
        for (int k = 0; k < 8; ++k) t += part[k][threadIdx.x];
        out[c] = t;
    }
}

void colsum(const float* x, int rows, int cols, int ld, float* out, cudaStream_t s)
{
    colsum_kernel<<<(cols + 31) / 32, dim3(32, 8), 0, s>>>(x, rows, cols, ld, out);
}

// residual R = Y - T, dY = 2 R / (rows cols) (FP32 and BF16); per-block partial sums of R^2
__global__ void mse_kernel(const float* __restrict__ y, const float* __restrict__ t, long long n, float scale,
                           float* dyf, bf16* dyh, float* partial)
{
    float s = 0.f;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const float r = y[i] - t[i];
        s += r * r;
        const float g = scale * r;
        dyf[i] = g;
        dyh[i] = __float2bfloat16(g);
    }
    __shared__ float red[256];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

__global__ void adam_kernel(float* w, const float* g, float* m, float* v, bf16* wh, long long n, float lr, float b1,
                            float b2, float c1, float c2, float eps)
{
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        wh[i] = __float2bfloat16(wi);
    }
}

__global__ void f2h_kernel(const float* __restrict__ x, bf16* y, long long n)
{
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
        y[i] = __float2bfloat16(x[i]);
}

// rows of X (BF16, ld = in_ld) from FP32 host-provided inputs [rows x in_dim]
__global__ void pack_rows_kernel(const float* __restrict__ x, int rows, int in_dim, int in_ld, bf16* X)
{
    const long long n = static_cast<long long>(rows) * in_ld;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int r = static_cast<int>(i / in_ld), c = static_cast<int>(i % in_ld);
        X[i] = __float2bfloat16(c < in_dim ? x[static_cast<long long>(r) * in_dim + c] : 0.f);
    }
}

__device__ __forceinline__ uint64_t mix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Minibatch from a host-style dataset on the device: sample b = uniform row of (x, t).
__global__ void gather_rows_kernel(const float* __restrict__ x, const float* __restrict__ t, int n, int in_dim,
                                   int out_dim, int in_ld, int batch, uint64_t seed, bf16* X, float* T)
{
    const int b = blockIdx.x;
    if (b >= batch) return;
    const int row = static_cast<int>(mix64(seed ^ (0x5851F42D4C957F2Dull * (b + 1))) % static_cast<uint64_t>(n));
    for (int c = threadIdx.x; c < in_ld; c += blockDim.x)
        X[static_cast<long long>(b) * in_ld + c] =
            __float2bfloat16(c < in_dim ? x[static_cast<long long>(row) * in_dim + c] : 0.f);
    for (int c = threadIdx.x; c < out_dim; c += blockDim.x)
        T[static_cast<long long>(b) * out_dim + c] = t[static_cast<long long>(row) * out_dim + c];
}

// Features of closure element (mode k, occupation n_k of the top-tier ADO,
// matrix element r, c) in one BF16 row: one-hot k, v_j(r), v_j(c) (j = bath
// of k), (E_r - E_c) / e_scale, one-hot n_k, zero padding to in_ld.
__device__ __forceinline__ void closure_features(bf16* X, int in_ld, int M, int maxd, int k, int nk, int r, int c,
                                                 const int* mode_bath, const double* vdiag, const double* hdiag,
                                                 int D, double inv_e)
{
    const int j = mode_bath[k];
    for (int q = 0; q < in_ld; ++q) X[q] = __float2bfloat16(0.f);
    X[k] = __float2bfloat16(1.f);
    X[M] = __float2bfloat16(static_cast<float>(vdiag[j * D + r]));
    X[M + 1] = __float2bfloat16(static_cast<float>(vdiag[j * D + c]));
    X[M + 2] = __float2bfloat16(static_cast<float>((hdiag[r] - hdiag[c]) * inv_e));
    X[M + 3 + (nk < maxd ? nk : maxd - 1)] = __float2bfloat16(1.f);
}

// Minibatch of closure samples, one thread per row: sample b = (snapshot, top-tier
// ADO i, mode k, element r, c with v_j(r) != v_j(c), up to eight draws), its
// features in X, the scaled element of ADO i in xin and of its up neighbour
// n_i + e_k in tgt.
__global__ void gather_closure_kernel(const float2* __restrict__ din, const float2* __restrict__ dout,
                                      const int* __restrict__ up_local, const int8_t* __restrict__ top_occ,
                                      const int* __restrict__ mode_bath, const double* __restrict__ vdiag,
                                      const double* __restrict__ hdiag, double inv_e, int n_snap, int n_top,
                                      int n_up, int M, int maxd, int logd, float inv_in, float inv_out, int in_ld,
                                      int batch, uint64_t seed, bf16* X, float2* xin, float2* tgt)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= batch) return;
    const int D = 1 << logd, d2 = D * D;
    uint64_t z = mix64(seed ^ (0x2545F4914F6CDD1Dull * (b + 1)));
    const long long pairs = static_cast<long long>(n_snap) * n_top * M;
    const long long pidx = static_cast<long long>(z % static_cast<uint64_t>(pairs));
    const int snap = static_cast<int>(pidx / (static_cast<long long>(n_top) * M));
    const int i = static_cast<int>((pidx / M) % n_top);
    const int k = static_cast<int>(pidx % M);
    const int j = mode_bath[k];
    int e = 0;
    for (int tries = 0; tries < 8; ++tries) {
        z = mix64(z);
        e = static_cast<int>(z % static_cast<uint64_t>(d2));
        if (vdiag[j * D + (e >> logd)] != vdiag[j * D + (e & (D - 1))]) break;
    }
    const int r = e >> logd, c = e & (D - 1);
    closure_features(X + static_cast<long long>(b) * in_ld, in_ld, M, maxd, k, top_occ[i * M + k], r, c, mode_bath,
                     vdiag, hdiag, D, inv_e);
    const float2 x = din[(static_cast<long long>(snap) * n_top + i) * d2 + e];
    const float2 t = dout[(static_cast<long long>(snap) * n_up + up_local[i * M + k]) * d2 + e];
    xin[b] = make_float2(x.x * inv_in, x.y * inv_in);
    tgt[b] = make_float2(t.x * inv_out, t.y * inv_out);
}

// Loss of the linear closure: the network's two outputs (a, b) are the
// complex coefficient A of pred = A x; loss = mean |pred - t|^2, and
// dL/da = 2 Re(conj(err) x) / B, dL/db = 2 Im(conj(x) err) / B (FP32 and BF16).
__global__ void closure_loss_kernel(const float* __restrict__ Y, const float2* __restrict__ xin,
                                    const float2* __restrict__ tgt, int B, float* dyf, bf16* dyh, float* partial)
{
    float s = 0.f;
    const float g = 2.0f / static_cast<float>(B);
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < B; b += gridDim.x * blockDim.x) {
        const float a = Y[2 * b], bb = Y[2 * b + 1];
        const float2 x = xin[b], t = tgt[b];
        const float er = a * x.x - bb * x.y - t.x, ei = a * x.y + bb * x.x - t.y;
        s += er * er + ei * ei;
        const float da = g * (er * x.x + ei * x.y), db = g * (ei * x.x - er * x.y);
        dyf[2 * b] = da;
        dyf[2 * b + 1] = db;
        dyh[2 * b] = __float2bfloat16(da);
        dyh[2 * b + 1] = __float2bfloat16(db);
    }
    __shared__ float red[256];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// Feature rows [row0, row0 + n) of the coefficient table; row = (k maxd + n_k) d^2 + r d + c.
__global__ void table_features_kernel(const int* __restrict__ mode_bath, const double* __restrict__ vdiag,
                                      const double* __restrict__ hdiag, double inv_e, int M, int maxd, int logd,
                                      int in_ld, long long row0, int n, bf16* X)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const long long row = row0 + q;
    const int D = 1 << logd, d2 = D * D;
    const int e = static_cast<int>(row % d2);
    const long long kn = row / d2;
    const int k = static_cast<int>(kn / maxd), nk = static_cast<int>(kn % maxd);
    closure_features(X + static_cast<long long>(q) * in_ld, in_ld, M, maxd, k, nk, e >> logd, e & (D - 1), mode_bath,
                     vdiag, hdiag, D, inv_e);
}

// coef(row) = ratio (A(r, c) + conj A(c, r)) / 2: the Hermitian part of the
// predicted up neighbour, so the closure term keeps the state Hermitian.
__global__ void table_kernel(const float2* __restrict__ raw, long long rows, int logd, double ratio, double2* coef)
{
    const long long row = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (row >= rows) return;
    const int D = 1 << logd, d2 = D * D;
    const int e = static_cast<int>(row % d2);
    const long long base = row - e;
    const int r = e >> logd, c = e & (D - 1);
    const float2 a = raw[row], b = raw[base + (c << logd) + r];
    coef[row] = make_double2(0.5 * ratio * (static_cast<double>(a.x) + b.x),
                             0.5 * ratio * (static_cast<double>(a.y) - b.y));
}

// Element e = r d + c of a stored slab: full, or Hermitian-packed (lower
// triangle read as the conjugate of the upper one).
__device__ __forceinline__ double2 slab_elem(const double2* slab, int e, int logd, int herm)
{
    if (!herm) return slab[e];
    const int r = e >> logd, c = e & ((1 << logd) - 1);
    if (r <= c) return slab[herm_index(r, c, logd)];
    const double2 v = slab[herm_index(c, r, logd)];
    return make_double2(v.x, -v.y);
}

// Copy, from a fine hierarchy's state, the coarse top-tier ADOs and their up
// neighbours (FP32, full d x d); stride = stored elements per slab.
__global__ void harvest_kernel(const double2* __restrict__ fine, const int* __restrict__ top_fine,
                               const int* __restrict__ up_fine, int n_top, int n_up, int d2, int logd, int herm,
                               long long stride, float2* din, float2* dout)
{
    const int s = blockIdx.y;  // slab number: [0, n_top) top tier, then [0, n_up) up neighbours
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= d2) return;
    if (s < n_top) {
        const double2 v = slab_elem(fine + top_fine[s] * stride, e, logd, herm);
        din[static_cast<long long>(s) * d2 + e] = make_float2(static_cast<float>(v.x), static_cast<float>(v.y));
    } else {
        const int t = s - n_top;
        const double2 v = slab_elem(fine + up_fine[t] * stride, e, logd, herm);
        dout[static_cast<long long>(t) * d2 + e] = make_float2(static_cast<float>(v.x), static_cast<float>(v.y));
    }
}

// Closure term of a stage: out_{top i}(r, c) += alpha sum_k -i (v_j(r) - v_j(c))
// coef[k][n_{i,k}](r, c) u_{top i}(r, c)   (the dropped up coupling, with the
// up neighbour predicted elementwise).  Full or Hermitian-packed slabs.
__global__ void closure_lin_kernel(const double2* __restrict__ u, const int* __restrict__ top,
                                   const int8_t* __restrict__ top_occ, const int* __restrict__ mode_bath,
                                   const double* __restrict__ vdiag, const double2* __restrict__ coef, int n_top,
                                   int M, int maxd, int logd, int herm, long long stride, double alpha,
                                   double2* out)
{
    const int D = 1 << logd, d2 = D * D;
    const int nel = herm ? herm_elems(logd) : d2;
    const int i = blockIdx.y;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nel || i >= n_top) return;
    int r, c;
    if (herm) {
        herm_coords(q, logd, r, c);
    } else {
        r = q >> logd;
        c = q & (D - 1);
    }
    const int e = (r << logd) + c;
    const double2 x = u[top[i] * stride + q];
    double sr = 0.0, si = 0.0;
    for (int k = 0; k < M; ++k) {
        const int j = mode_bath[k];
        const double del = vdiag[j * D + r] - vdiag[j * D + c];
        if (del == 0.0) continue;
        const double2 a = coef[(static_cast<long long>(k) * maxd + top_occ[i * M + k]) * d2 + e];
        // -i del (a x)
        sr += del * (a.x * x.y + a.y * x.x);
        si -= del * (a.x * x.x - a.y * x.y);
    }
    double2* o = out + top[i] * stride + q;
    o->x += alpha * sr;
    o->y += alpha * si;
}

// sum of squares of FP32 complex data (deterministic two-level sum)
__global__ void sumsq_kernel(const float2* __restrict__ x, long long n, double* partial)
{
    double s = 0.0;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
        s += static_cast<double>(x[i].x) * x[i].x + static_cast<double>(x[i].y) * x[i].y;
    __shared__ double red[256];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

}  // namespace

}  // namespace hx

// ---------------------------------------------------------------------------
// MLP object
// ---------------------------------------------------------------------------

struct hx_mlp {
    int in_dim = 0, in_ld = 0, hidden = 0, out_dim = 0;
    long long n_params = 0;
    cudaStream_t stream = nullptr;
    // FP32 parameters (W1 b1 W2 b2 W3 b3, contiguous), gradients, Adam moments, BF16 copy
    float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
    bf16* wh = nullptr;
    long long adam_t = 0;
    uint64_t version = 0;  // bumped whenever the parameters change
    // activations for one batch
    int cap = 0;
    bf16 *X = nullptr, *H1 = nullptr, *H2 = nullptr, *dYh = nullptr, *dZ2h = nullptr, *dZ1h = nullptr;
    float *Z1 = nullptr, *Z2 = nullptr, *Y = nullptr, *T = nullptr, *dYf = nullptr, *dZ2f = nullptr, *dZ1f = nullptr;
    float* partial = nullptr;
    float* pinned = nullptr;
    // parameter offsets
    long long oW1 = 0, ob1 = 0, oW2 = 0, ob2 = 0, oW3 = 0, ob3 = 0;
    // tensor-core GEMM scratch (transposed operands) and error word
    hx::TcScratch tc;
};

namespace {

void mlp_free_batch(hx_mlp* n)
{
    void* p[] = {n->X, n->H1, n->H2, n->dYh, n->dZ2h, n->dZ1h, n->Z1, n->Z2, n->Y, n->T, n->dYf, n->dZ2f, n->dZ1f,
                 n->tc.a, n->tc.b};
    for (void* q : p)
        if (q) cudaFree(q);
    n->tc.a = n->tc.b = nullptr;
    n->tc.a_elems = n->tc.b_elems = 0;
    n->X = n->H1 = n->H2 = n->dYh = n->dZ2h = n->dZ1h = nullptr;
    n->Z1 = n->Z2 = n->Y = n->T = n->dYf = n->dZ2f = n->dZ1f = nullptr;
    n->cap = 0;
}

int mlp_reserve(hx_mlp* n, int batch)
{
    if (batch <= n->cap) return HX_OK;
    mlp_free_batch(n);
    const size_t B = static_cast<size_t>(batch);
    cudaError_t e = cudaMalloc(&n->X, B * n->in_ld * sizeof(bf16));
    if (e == cudaSuccess) e = cudaMalloc(&n->H1, B * n->hidden * sizeof(bf16));
    if (e == cudaSuccess) e = cudaMalloc(&n->H2, B * n->hidden * sizeof(bf16));
    if (e == cudaSuccess) e = cudaMalloc(&n->dYh, B * n->out_dim * sizeof(bf16));
    if (e == cudaSuccess) e = cudaMalloc(&n->dZ2h, B * n->hidden * sizeof(bf16));
    if (e == cudaSuccess) e = cudaMalloc(&n->dZ1h, B * n->hidden * sizeof(bf16));
    if (e == cudaSuccess) e = cudaMalloc(&n->Z1, B * n->hidden * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&n->Z2, B * n->hidden * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&n->Y, B * n->out_dim * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&n->T, B * n->out_dim * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&n->dYf, B * n->out_dim * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&n->dZ2f, B * n->hidden * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&n->dZ1f, B * n->hidden * sizeof(float));
    // transposed operands: rows up to max(hidden, out, in), leading dimension up to max(batch, hidden, out) rounded to 8
    const size_t rows = static_cast<size_t>(std::max(n->hidden, std::max(n->out_dim, n->in_ld)));
    const size_t cols = static_cast<size_t>((std::max(batch, std::max(n->hidden, n->out_dim)) + 7) & ~7);
    if (e == cudaSuccess) e = cudaMalloc(&n->tc.a, rows * cols * sizeof(bf16));
    if (e == cudaSuccess) e = cudaMalloc(&n->tc.b, rows * cols * sizeof(bf16));
    if (e == cudaSuccess) n->tc.a_elems = n->tc.b_elems = rows * cols;
    if (e != cudaSuccess) {
        mlp_free_batch(n);
        return hx::cuda_fail(e, "cudaMalloc (MLP activations)");
    }
    n->cap = batch;
    return HX_OK;
}

// Forward pass of rows X[0..B) (BF16, already in n->X): Z1, H1, Z2, H2, Y.
void mlp_forward(hx_mlp* n, int B, cudaStream_t s)
{
    using namespace hx;
    const bf16* W = n->wh;
    gemm<false, true, kEpiBiasGelu>(B, n->hidden, n->in_dim, n->X, n->in_ld, W + n->oW1, n->in_dim,
                                    GemmOut{n->w + n->ob1, n->Z1, n->H1, nullptr, n->hidden}, s, &n->tc);
    gemm<false, true, kEpiBiasGelu>(B, n->hidden, n->hidden, n->H1, n->hidden, W + n->oW2, n->hidden,
                                    GemmOut{n->w + n->ob2, n->Z2, n->H2, nullptr, n->hidden}, s, &n->tc);
    gemm<false, true, kEpiBias>(B, n->out_dim, n->hidden, n->H2, n->hidden, W + n->oW3, n->hidden,
                                GemmOut{n->w + n->ob3, n->Y, nullptr, nullptr, n->out_dim}, s, &n->tc);
}

// Gradient of every parameter into n->g from dL/dY already in n->dYf / n->dYh.
void mlp_backward_dy(hx_mlp* n, int B, cudaStream_t s)
{
    using namespace hx;
    const bf16* W = n->wh;
    // layer 3
    gemm<true, false, kEpiStore>(n->out_dim, n->hidden, B, n->dYh, n->out_dim, n->H2, n->hidden,
                                 GemmOut{nullptr, n->g + n->oW3, nullptr, nullptr, n->hidden}, s, &n->tc);
    colsum(n->dYf, B, n->out_dim, n->out_dim, n->g + n->ob3, s);
    gemm<false, false, kEpiGeluBack>(B, n->hidden, n->out_dim, n->dYh, n->out_dim, W + n->oW3, n->hidden,
                                     GemmOut{nullptr, n->dZ2f, n->dZ2h, n->Z2, n->hidden}, s, &n->tc);
    // layer 2
    gemm<true, false, kEpiStore>(n->hidden, n->hidden, B, n->dZ2h, n->hidden, n->H1, n->hidden,
                                 GemmOut{nullptr, n->g + n->oW2, nullptr, nullptr, n->hidden}, s, &n->tc);
    colsum(n->dZ2f, B, n->hidden, n->hidden, n->g + n->ob2, s);
    gemm<false, false, kEpiGeluBack>(B, n->hidden, n->hidden, n->dZ2h, n->hidden, W + n->oW2, n->hidden,
                                     GemmOut{nullptr, n->dZ1f, n->dZ1h, n->Z1, n->hidden}, s, &n->tc);
    // layer 1
    gemm<true, false, kEpiStore>(n->hidden, n->in_dim, B, n->dZ1h, n->hidden, n->X, n->in_ld,
                                 GemmOut{nullptr, n->g + n->oW1, nullptr, nullptr, n->in_dim}, s, &n->tc);
    colsum(n->dZ1f, B, n->hidden, n->hidden, n->g + n->ob1, s);
}

// Sum of the per-block loss partials (148 blocks) divided by count.
// Error word of the tensor-core GEMMs (a wait that ran out of its budget); cleared when read.
int mlp_tc_status(hx_mlp* n, cudaStream_t s)
{
    int flag = 0;
    HX_CUDA_TRY(cudaMemcpyAsync(&flag, n->tc.err, sizeof(int), cudaMemcpyDeviceToHost, s));
    HX_CUDA_TRY(cudaStreamSynchronize(s));
    if (flag != 0) {
        cudaMemsetAsync(n->tc.err, 0, sizeof(int), s);
        return fail(HX_ERR_DEVICE_TIMEOUT, "a tensor-core GEMM wait ran out of its iteration budget");
    }
    return HX_OK;
}

int mlp_loss_of_partials(hx_mlp* n, double count, float* loss, cudaStream_t s)
{
    HX_CUDA_TRY(cudaMemcpyAsync(n->pinned, n->partial, 148 * sizeof(float), cudaMemcpyDeviceToHost, s));
    HX_CUDA_TRY(cudaStreamSynchronize(s));
    if (int rc = mlp_tc_status(n, s)) return rc;
    double acc = 0.0;
    for (int i = 0; i < 148; ++i) acc += n->pinned[i];
    *loss = static_cast<float>(acc / count);
    return HX_OK;
}

// MSE loss against n->T and the gradient of every parameter into n->g; returns the loss.
int mlp_backward(hx_mlp* n, int B, float* loss, cudaStream_t s)
{
    const long long ny = static_cast<long long>(B) * n->out_dim;
    hx::mse_kernel<<<148, 256, 0, s>>>(n->Y, n->T, ny, 2.0f / static_cast<float>(ny), n->dYf, n->dYh, n->partial);
    mlp_backward_dy(n, B, s);
    return loss ? mlp_loss_of_partials(n, static_cast<double>(ny), loss, s) : HX_OK;
}

void mlp_adam(hx_mlp* n, float lr, cudaStream_t s)
{
    n->adam_t += 1;
    n->version += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, static_cast<float>(n->adam_t));
    const float c2 = 1.f - std::pow(b2, static_cast<float>(n->adam_t));
    hx::adam_kernel<<<148 * 4, 256, 0, s>>>(n->w, n->g, n->m, n->v, n->wh, n->n_params, lr, b1, b2, c1, c2, 1e-8f);
}

void mlp_release(hx_mlp* n)
{
    if (!n) return;
    if (n->stream) cudaStreamSynchronize(n->stream);
    mlp_free_batch(n);
    void* p[] = {n->w, n->g, n->m, n->v, n->wh, n->partial, n->tc.err};
    for (void* q : p)
        if (q) cudaFree(q);
    if (n->pinned) cudaFreeHost(n->pinned);
    if (n->stream) cudaStreamDestroy(n->stream);
    delete n;
}

}  // namespace

// ---------------------------------------------------------------------------
// Closure object: index maps, device training set, the MLP
// ---------------------------------------------------------------------------

// The closure predicts the dropped up neighbour of a top-tier ADO n
// elementwise: rho_{n+e_k}(r, c) ~ A(k, n_k, r, c) rho_n(r, c), the complex
// coefficient A coming from the MLP on the features of (k, n_k, r, c)
// (closure_features).  The equations are linear, and so is this prediction
// in rho_n.  After training, A is evaluated once for every (k, n_k, r, c) into
// a coefficient table, so a stage costs one elementwise kernel.
struct hx_closure {
    hx_mlp* net = nullptr;
    int d = 0, logd = 0, d2 = 0, M = 0, J = 0;
    uint32_t coarse_depth = 0, fine_depth = 0;
    int maxd = 0;                // n_k of a top-tier ADO is in [0, maxd)
    int n_top = 0, n_up = 0;
    std::vector<int> mode_bath;
    int* top_coarse = nullptr;   // [n_top] coarse index of each top-tier ADO
    int* top_fine = nullptr;     // [n_top] its index in the fine hierarchy
    int8_t* top_occ = nullptr;   // [n_top][M] occupation n_k of each top-tier ADO
    int* up_fine = nullptr;      // [n_up] fine index of each distinct up neighbour
    int* up_local = nullptr;     // [n_top][M] which of them is n_top[i] + e_k
    int* mode_bath_d = nullptr;  // [M]
    double* vdiag = nullptr;     // [J][d] coupling diagonals
    double* hdiag = nullptr;     // [d] diagonal of H
    double inv_e = 1.0;          // 1 / (max E - min E)
    float2* din = nullptr;       // [cap][n_top][d2]
    float2* dout = nullptr;      // [cap][n_up][d2]
    float2* xin = nullptr;       // [batch] training inputs (scaled elements)
    float2* tgt = nullptr;       // [batch] training targets
    int sample_cap = 0;
    float2* raw = nullptr;       // [M][maxd][d2] network output A
    double2* coef = nullptr;     // [M][maxd][d2] Hermitian part of A times s_out / s_in
    uint64_t table_version = ~0ull;  // network version the table was built from
    int cap = 0, n_snap = 0;
    double s_in = 1.0, s_out = 1.0;  // RMS scales of inputs and targets
    bool scaled = false;
    cudaStream_t stream = nullptr;
};

namespace {

void closure_release(hx_closure* c)
{
    if (!c) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    void* p[] = {c->top_coarse, c->top_fine, c->up_fine, c->up_local, c->mode_bath_d, c->din, c->dout,
                 c->top_occ, c->vdiag, c->hdiag, c->xin, c->tgt, c->raw, c->coef};
    for (void* q : p)
        if (q) cudaFree(q);
    if (c->net) mlp_release(c->net);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

double rms_of(const float2* x, long long n, cudaStream_t s)
{
    double* partial = nullptr;
    if (cudaMalloc(&partial, 148 * sizeof(double)) != cudaSuccess) return -1.0;
    hx::sumsq_kernel<<<148, 256, 0, s>>>(x, n, partial);
    double h[148];
    cudaMemcpyAsync(h, partial, sizeof(h), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    cudaFree(partial);
    double acc = 0.0;
    for (double v : h) acc += v;
    return std::sqrt(acc / (2.0 * static_cast<double>(n)));
}

}  // namespace

// closure hook used by the context's stages (hx_ctx.cu)
bool hx::closure_matches_hierarchy(const hx_closure* cl, int d, int M, long long H)
{
    uint64_t Hc = 0;
    hx_hierarchy_size(static_cast<uint32_t>(cl->M), cl->coarse_depth, &Hc);
    return cl->d == d && cl->M == M && static_cast<long long>(Hc) == H;
}

namespace {

// Evaluate the network on every (k, n_k, r, c) and store the Hermitian part
// of A, times s_out / s_in, in the coefficient table.
int build_table(hx_closure* cl, cudaStream_t s)
{
    hx_mlp* n = cl->net;
    const long long rows = static_cast<long long>(cl->M) * cl->maxd * cl->d2;
    const int chunk = 8192;
    int rc = mlp_reserve(n, chunk);
    if (rc != HX_OK) return rc;
    for (long long r0 = 0; r0 < rows; r0 += chunk) {
        const int cnt = static_cast<int>(std::min<long long>(chunk, rows - r0));
        hx::table_features_kernel<<<(cnt + 127) / 128, 128, 0, s>>>(cl->mode_bath_d, cl->vdiag, cl->hdiag, cl->inv_e,
                                                                   cl->M, cl->maxd, cl->logd, n->in_ld, r0, cnt, n->X);
        mlp_forward(n, cnt, s);
        HX_CUDA_TRY(cudaMemcpyAsync(cl->raw + r0, n->Y, cnt * sizeof(float2), cudaMemcpyDeviceToDevice, s));
    }
    hx::table_kernel<<<static_cast<unsigned>((rows + 255) / 256), 256, 0, s>>>(cl->raw, rows, cl->logd,
                                                                               cl->s_out / cl->s_in, cl->coef);
    HX_CUDA_TRY(cudaGetLastError());
    cl->table_version = n->version;
    return HX_OK;
}

}  // namespace

namespace hx {
int closure_stage(hx_closure* cl, const ::hx_ctx* c, const double2* u, double2* out, double alpha, cudaStream_t s)
{
    if (!cl || !cl->scaled) return HX_OK;
    if (cl->table_version != cl->net->version) {
        const int rc = build_table(cl, s);
        if (rc != HX_OK) return rc;
    }
    const int herm = c->herm ? 1 : 0;
    const long long stride = static_cast<long long>(c->slab_store);
    const int nel = herm ? herm_elems(cl->logd) : cl->d2;
    dim3 grid((nel + 255) / 256, cl->n_top);
    closure_lin_kernel<<<grid, 256, 0, s>>>(u, cl->top_coarse, cl->top_occ, cl->mode_bath_d, cl->vdiag, cl->coef,
                                           cl->n_top, cl->M, cl->maxd, cl->logd, herm, stride, alpha, out);
    return HX_OK;
}
}  // namespace hx


extern "C" {

int hx_mlp_create(uint32_t in_dim, uint32_t hidden, uint32_t out_dim, uint64_t seed, hx_mlp** out)
{
    if (!out) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL MLP output");
    *out = nullptr;
    if (in_dim == 0 || hidden == 0 || out_dim == 0 || in_dim > 65536 || hidden > 8192 || out_dim > 65536)
        return fail(HX_ERR_INVALID_RUNTIME_OPTION, "MLP dimensions out of range");
    hx_mlp* n = new (std::nothrow) hx_mlp();
    if (!n) return fail(HX_ERR_OUT_OF_MEMORY, "host allocation failed");
    n->in_dim = static_cast<int>(in_dim);
    n->in_ld = (n->in_dim + 7) & ~7;
    n->hidden = static_cast<int>(hidden);
    n->out_dim = static_cast<int>(out_dim);
    n->oW1 = 0;
    n->ob1 = n->oW1 + static_cast<long long>(hidden) * in_dim;
    n->oW2 = n->ob1 + hidden;
    n->ob2 = n->oW2 + static_cast<long long>(hidden) * hidden;
    n->oW3 = n->ob2 + hidden;
    n->ob3 = n->oW3 + static_cast<long long>(out_dim) * hidden;
    n->n_params = n->ob3 + out_dim;
    // the BF16 copies of W2, W3 start at offsets oW2, oW3: keep them 16-byte aligned
    auto bail = [&](int rc) {
        mlp_release(n);
        return rc;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking);
    const size_t np = static_cast<size_t>(n->n_params);
    if (e == cudaSuccess) e = cudaMalloc(&n->w, np * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&n->g, np * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&n->m, np * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&n->v, np * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&n->wh, np * sizeof(bf16));
    if (e == cudaSuccess) e = cudaMalloc(&n->partial, 256 * sizeof(float));
    if (e == cudaSuccess) e = cudaMallocHost(&n->pinned, 256 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&n->tc.err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(n->tc.err, 0, sizeof(int));
    if (e != cudaSuccess) return bail(hx::cuda_fail(e, "cudaMalloc (MLP)"));
    // He-style uniform init from splitmix64(seed), biases zero
    std::vector<float> w(np, 0.f);
    uint64_t st = seed;
    auto uni = [&]() {
        st += 0x9E3779B97F4A7C15ull;
        uint64_t z = st;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return static_cast<double>(z >> 11) * (1.0 / 9007199254740992.0);
    };
    auto fill = [&](long long off, long long count, int fan_in) {
        const double a = std::sqrt(6.0 / fan_in);
        for (long long i = 0; i < count; ++i) w[off + i] = static_cast<float>((2.0 * uni() - 1.0) * a);
    };
    fill(n->oW1, static_cast<long long>(hidden) * in_dim, static_cast<int>(in_dim));
    fill(n->oW2, static_cast<long long>(hidden) * hidden, static_cast<int>(hidden));
    fill(n->oW3, static_cast<long long>(out_dim) * hidden, static_cast<int>(hidden));
    const int rc = hx_mlp_set_params(n, w.data(), np);
    if (rc != HX_OK) return bail(rc);
    *out = n;
    return HX_OK;
}

void hx_mlp_destroy(hx_mlp* n) { mlp_release(n); }

int hx_mlp_num_params(const hx_mlp* n, uint64_t* count)
{
    if (!n || !count) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL argument");
    *count = static_cast<uint64_t>(n->n_params);
    return HX_OK;
}

int hx_mlp_set_params(hx_mlp* n, const float* params, uint64_t count)
{
    if (!n || !params) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL argument");
    if (count != static_cast<uint64_t>(n->n_params)) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "parameter count mismatch");
    const size_t np = static_cast<size_t>(n->n_params);
    HX_CUDA_TRY(cudaMemcpyAsync(n->w, params, np * sizeof(float), cudaMemcpyHostToDevice, n->stream));
    HX_CUDA_TRY(cudaMemsetAsync(n->m, 0, np * sizeof(float), n->stream));
    HX_CUDA_TRY(cudaMemsetAsync(n->v, 0, np * sizeof(float), n->stream));
    hx::f2h_kernel<<<148 * 4, 256, 0, n->stream>>>(n->w, n->wh, n->n_params);
    HX_CUDA_TRY(cudaGetLastError());
    HX_CUDA_TRY(cudaStreamSynchronize(n->stream));
    n->adam_t = 0;
    n->version += 1;
    return HX_OK;
}

int hx_mlp_get_params(hx_mlp* n, float* params, uint64_t count)
{
    if (!n || !params) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL argument");
    if (count != static_cast<uint64_t>(n->n_params)) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "parameter count mismatch");
    HX_CUDA_TRY(cudaMemcpyAsync(params, n->w, n->n_params * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
    HX_CUDA_TRY(cudaStreamSynchronize(n->stream));
    return HX_OK;
}

int hx_mlp_forward(hx_mlp* n, const float* x, uint32_t rows, float* y)
{
    if (!n || !x || !y) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL argument");
    if (rows == 0) return HX_OK;
    int rc = mlp_reserve(n, static_cast<int>(rows));
    if (rc != HX_OK) return rc;
    float* dx = nullptr;
    const size_t nx = static_cast<size_t>(rows) * n->in_dim;
    HX_CUDA_TRY(cudaMalloc(&dx, nx * sizeof(float)));
    cudaError_t e = cudaMemcpyAsync(dx, x, nx * sizeof(float), cudaMemcpyHostToDevice, n->stream);
    if (e == cudaSuccess) {
        hx::pack_rows_kernel<<<148 * 4, 256, 0, n->stream>>>(dx, static_cast<int>(rows), n->in_dim, n->in_ld, n->X);
        mlp_forward(n, static_cast<int>(rows), n->stream);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(y, n->Y, static_cast<size_t>(rows) * n->out_dim * sizeof(float), cudaMemcpyDeviceToHost,
                            n->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(n->stream);
    cudaFree(dx);
    if (e != cudaSuccess) return hx::cuda_fail(e, "MLP forward");
    return mlp_tc_status(n, n->stream);
}

int hx_mlp_gradients(hx_mlp* n, const float* x, const float* t, uint32_t rows, float* loss, float* grads,
                     uint64_t count)
{
    if (!n || !x || !t || !grads) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL argument");
    if (count != static_cast<uint64_t>(n->n_params)) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "parameter count mismatch");
    if (rows == 0) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "empty batch");
    int rc = mlp_reserve(n, static_cast<int>(rows));
    if (rc != HX_OK) return rc;
    float* dx = nullptr;
    const size_t nx = static_cast<size_t>(rows) * n->in_dim, nt = static_cast<size_t>(rows) * n->out_dim;
    HX_CUDA_TRY(cudaMalloc(&dx, nx * sizeof(float)));
    cudaError_t e = cudaMemcpyAsync(dx, x, nx * sizeof(float), cudaMemcpyHostToDevice, n->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(n->T, t, nt * sizeof(float), cudaMemcpyHostToDevice, n->stream);
    if (e == cudaSuccess) {
        hx::pack_rows_kernel<<<148 * 4, 256, 0, n->stream>>>(dx, static_cast<int>(rows), n->in_dim, n->in_ld, n->X);
        mlp_forward(n, static_cast<int>(rows), n->stream);
        rc = mlp_backward(n, static_cast<int>(rows), loss, n->stream);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && rc == HX_OK)
        e = cudaMemcpyAsync(grads, n->g, n->n_params * sizeof(float), cudaMemcpyDeviceToHost, n->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(n->stream);
    cudaFree(dx);
    if (rc != HX_OK) return rc;
    if (e != cudaSuccess) return hx::cuda_fail(e, "MLP gradients");
    return HX_OK;
}

int hx_mlp_train(hx_mlp* n, const float* x, const float* t, uint32_t rows, uint32_t batch, uint32_t iters, float lr,
                 uint64_t seed, float* loss_trace)
{
    if (!n || !x || !t) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL argument");
    if (rows == 0 || batch == 0) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "empty data or batch");
    int rc = mlp_reserve(n, static_cast<int>(batch));
    if (rc != HX_OK) return rc;
    float *dx = nullptr, *dt = nullptr;
    const size_t nx = static_cast<size_t>(rows) * n->in_dim, nt = static_cast<size_t>(rows) * n->out_dim;
    HX_CUDA_TRY(cudaMalloc(&dx, nx * sizeof(float)));
    cudaError_t e = cudaMalloc(&dt, nt * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpyAsync(dx, x, nx * sizeof(float), cudaMemcpyHostToDevice, n->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dt, t, nt * sizeof(float), cudaMemcpyHostToDevice, n->stream);
    for (uint32_t it = 0; it < iters && e == cudaSuccess && rc == HX_OK; ++it) {
        hx::gather_rows_kernel<<<batch, 256, 0, n->stream>>>(dx, dt, static_cast<int>(rows), n->in_dim, n->out_dim,
                                                            n->in_ld, static_cast<int>(batch), seed + it, n->X, n->T);
        mlp_forward(n, static_cast<int>(batch), n->stream);
        float l = 0.f;
        rc = mlp_backward(n, static_cast<int>(batch), loss_trace ? &l : nullptr, n->stream);
        if (loss_trace) loss_trace[it] = l;
        mlp_adam(n, lr, n->stream);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(n->stream);
    cudaFree(dx);
    cudaFree(dt);
    if (rc != HX_OK) return rc;
    if (e != cudaSuccess) return hx::cuda_fail(e, "MLP training");
    return HX_OK;
}

int hx_closure_create(const hx_problem* coarse, uint32_t fine_max_depth, uint32_t hidden, uint32_t capacity,
                      uint64_t seed, hx_closure** out)
{
    if (!out) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL closure output");
    *out = nullptr;
    if (!coarse || !coarse->baths || coarse->n_baths == 0 || !coarse->h_diag)
        return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL problem");
    if (coarse->h_csr) return fail(HX_ERR_UNSUPPORTED_EXECUTION, "closures need diagonal plus flip Hamiltonians");
    for (uint32_t j = 0; j < coarse->n_baths; ++j)
        if (coarse->baths[j].coupling_csr)
            return fail(HX_ERR_UNSUPPORTED_EXECUTION, "closures need diagonal coupling operators");
    const uint32_t d = coarse->dim;
    if (d < 2 || d > 64 || (d & (d - 1)) != 0) return fail(HX_ERR_INVALID_DIMENSION, "closures need 2 <= dim <= 64");
    if (coarse->max_depth < 2 || fine_max_depth <= coarse->max_depth)
        return fail(HX_ERR_UNSUPPORTED_HIERARCHY, "the fine hierarchy must be deeper than the coarse one (coarse max_depth >= 2)");
    if (capacity == 0) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "capacity must be positive");
    int M = 0;
    std::vector<int> mb;
    for (uint32_t j = 0; j < coarse->n_baths; ++j)
        for (uint32_t k = 0; k <= coarse->baths[j].pade_terms; ++k, ++M) mb.push_back(static_cast<int>(j));
    if (M > 128) return fail(HX_ERR_UNSUPPORTED_HIERARCHY, "too many modes");
    uint64_t Hc = 0, Hf = 0;
    int rc = hx_hierarchy_size(M, coarse->max_depth, &Hc);
    if (rc == HX_OK) rc = hx_hierarchy_size(M, fine_max_depth, &Hf);
    if (rc != HX_OK) return rc;
    if (Hf >= (1ull << 31)) return fail(HX_ERR_UNSUPPORTED_HIERARCHY, "fine hierarchy too large");
    std::vector<int32_t> rc_rows(Hc * M), rc_edges(Hc * 2 * M), rf_rows(Hf * M), rf_edges(Hf * 2 * M);
    if ((rc = hx_hierarchy_tables(M, coarse->max_depth, rc_rows.data(), rc_edges.data(), Hc)) != HX_OK) return rc;
    if ((rc = hx_hierarchy_tables(M, fine_max_depth, rf_rows.data(), rf_edges.data(), Hf)) != HX_OK) return rc;
    // fine index of every index vector
    std::map<std::vector<int32_t>, int> fine_of;
    for (uint64_t i = 0; i < Hf; ++i)
        fine_of[std::vector<int32_t>(rf_rows.begin() + i * M, rf_rows.begin() + (i + 1) * M)] = static_cast<int>(i);
    hx_closure* c = new (std::nothrow) hx_closure();
    if (!c) return fail(HX_ERR_OUT_OF_MEMORY, "host allocation failed");
    auto bail = [&](int code) {
        closure_release(c);
        return code;
    };
    c->d = static_cast<int>(d);
    while ((1 << c->logd) < c->d) ++c->logd;
    c->d2 = c->d * c->d;
    c->M = M;
    c->J = static_cast<int>(coarse->n_baths);
    c->coarse_depth = coarse->max_depth;
    c->fine_depth = fine_max_depth;
    c->maxd = static_cast<int>(coarse->max_depth);
    c->mode_bath = mb;
    // operators for the features: coupling diagonals and the diagonal of H
    std::vector<double> vd(static_cast<size_t>(c->J) * d), hd(coarse->h_diag, coarse->h_diag + d);
    for (int j = 0; j < c->J; ++j) {
        if (!coarse->baths[j].coupling_diag) return bail(fail(HX_ERR_UNSUPPORTED_BATH, "coupling operator is NULL"));
        if (coarse->baths[j].coupling_flip)
            for (int b = 0; (1u << b) < d; ++b)
                if (coarse->baths[j].coupling_flip[b] != 0.0)
                    return bail(fail(HX_ERR_UNSUPPORTED_EXECUTION, "closures need diagonal coupling operators"));
        std::copy(coarse->baths[j].coupling_diag, coarse->baths[j].coupling_diag + d,
                  vd.begin() + static_cast<size_t>(j) * d);
    }
    const double emax = *std::max_element(hd.begin(), hd.end()), emin = *std::min_element(hd.begin(), hd.end());
    c->inv_e = emax > emin ? 1.0 / (emax - emin) : 1.0;
    // top tier of the coarse hierarchy and the fine indices of its up neighbours
    std::vector<int> top_c, top_f, up_f, up_loc;
    std::vector<int8_t> occ;
    std::map<int, int> up_index;
    for (uint64_t i = 0; i < Hc; ++i) {
        std::vector<int32_t> v(rc_rows.begin() + i * M, rc_rows.begin() + (i + 1) * M);
        int tier = 0;
        for (int x : v) tier += x;
        if (tier != static_cast<int>(coarse->max_depth) - 1) continue;
        top_c.push_back(static_cast<int>(i));
        top_f.push_back(fine_of.at(v));
        for (int k = 0; k < M; ++k) occ.push_back(static_cast<int8_t>(v[k]));
        for (int k = 0; k < M; ++k) {
            std::vector<int32_t> w = v;
            w[k] += 1;
            const int fi = fine_of.at(w);
            auto it = up_index.find(fi);
            if (it == up_index.end()) {
                it = up_index.emplace(fi, static_cast<int>(up_f.size())).first;
                up_f.push_back(fi);
            }
            up_loc.push_back(it->second);
        }
    }
    c->n_top = static_cast<int>(top_c.size());
    c->n_up = static_cast<int>(up_f.size());
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    auto dalloc = [&](auto** p, size_t n) { return cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(**p)); };
    if (e == cudaSuccess) e = dalloc(&c->top_coarse, top_c.size());
    if (e == cudaSuccess) e = dalloc(&c->top_fine, top_f.size());
    if (e == cudaSuccess) e = dalloc(&c->up_fine, up_f.size());
    if (e == cudaSuccess) e = dalloc(&c->up_local, up_loc.size());
    if (e == cudaSuccess) e = dalloc(&c->mode_bath_d, mb.size());
    if (e == cudaSuccess) e = dalloc(&c->din, static_cast<size_t>(capacity) * c->n_top * c->d2);
    if (e == cudaSuccess) e = dalloc(&c->dout, static_cast<size_t>(capacity) * c->n_up * c->d2);
    const size_t table = static_cast<size_t>(M) * c->maxd * c->d2;
    if (e == cudaSuccess) e = dalloc(&c->top_occ, occ.size());
    if (e == cudaSuccess) e = dalloc(&c->vdiag, vd.size());
    if (e == cudaSuccess) e = dalloc(&c->hdiag, hd.size());
    if (e == cudaSuccess) e = dalloc(&c->raw, table);
    if (e == cudaSuccess) e = dalloc(&c->coef, table);
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->top_occ, occ.data(), occ.size(), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(c->vdiag, vd.data(), vd.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(c->hdiag, hd.data(), hd.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->top_coarse, top_c.data(), top_c.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->top_fine, top_f.data(), top_f.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->up_fine, up_f.data(), up_f.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->up_local, up_loc.data(), up_loc.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->mode_bath_d, mb.data(), mb.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return bail(hx::cuda_fail(e, "closure set-up"));
    c->cap = static_cast<int>(capacity);
    if ((rc = hx_mlp_create(static_cast<uint32_t>(M + 3 + c->maxd), hidden, 2, seed, &c->net)) != HX_OK)
        return bail(rc);
    *out = c;
    return HX_OK;
}

void hx_closure_destroy(hx_closure* c) { closure_release(c); }

int hx_closure_mlp(hx_closure* c, hx_mlp** net)
{
    if (!c || !net) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL argument");
    *net = c->net;
    return HX_OK;
}

int hx_closure_info(const hx_closure* c, uint32_t* top_ados, uint32_t* up_ados, uint32_t* snapshots, double* s_in,
                    double* s_out)
{
    if (!c) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL closure");
    if (top_ados) *top_ados = static_cast<uint32_t>(c->n_top);
    if (up_ados) *up_ados = static_cast<uint32_t>(c->n_up);
    if (snapshots) *snapshots = static_cast<uint32_t>(c->n_snap);
    if (s_in) *s_in = c->s_in;
    if (s_out) *s_out = c->s_out;
    return HX_OK;
}

int hx_closure_harvest(hx_closure* c, hx_ctx* fine)
{
    if (!c || !fine) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL argument");
    if (c->n_snap >= c->cap) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "closure training set is full");
    hx_info info{};
    int rc = hx_ctx_info(fine, &info);
    if (rc != HX_OK) return rc;
    uint64_t Hf = 0;
    hx_hierarchy_size(c->M, c->fine_depth, &Hf);
    if (static_cast<int>(info.dim) != c->d || static_cast<int>(info.modes) != c->M || info.hierarchy_size != Hf)
        return fail(HX_ERR_INVALID_RUNTIME_OPTION, "the context is not the closure's fine hierarchy");
    void* state = nullptr;
    if ((rc = hx_ctx_state_device_ptr(fine, &state)) != HX_OK) return rc;
    void* fs = nullptr;
    if ((rc = hx_ctx_get_stream(fine, &fs)) != HX_OK) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(fs);
    const long long snap = c->n_snap;
    dim3 grid((c->d2 + 255) / 256, c->n_top + c->n_up);
    hx::harvest_kernel<<<grid, 256, 0, s>>>(static_cast<const double2*>(state), c->top_fine, c->up_fine, c->n_top,
                                           c->n_up, c->d2, c->logd, fine->herm ? 1 : 0,
                                           static_cast<long long>(fine->slab_store), c->din + snap * c->n_top * c->d2,
                                           c->dout + snap * c->n_up * c->d2);
    HX_CUDA_TRY(cudaGetLastError());
    HX_CUDA_TRY(cudaStreamSynchronize(s));
    c->n_snap += 1;
    c->scaled = false;
    return HX_OK;
}

int hx_closure_train(hx_closure* c, uint32_t iters, uint32_t batch, float lr, uint64_t seed, float* loss_trace)
{
    if (!c) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL closure");
    if (c->n_snap == 0) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "the closure training set is empty");
    if (batch == 0) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "empty batch");
    hx_mlp* n = c->net;
    if (!c->scaled) {
        const double si = rms_of(c->din, static_cast<long long>(c->n_snap) * c->n_top * c->d2, c->stream);
        const double so = rms_of(c->dout, static_cast<long long>(c->n_snap) * c->n_up * c->d2, c->stream);
        if (!(si > 0.0) || !(so > 0.0)) return fail(HX_ERR_NON_FINITE, "closure training data has no signal");
        c->s_in = si;
        c->s_out = so;
        c->scaled = true;
    }
    int rc = mlp_reserve(n, static_cast<int>(batch));
    if (rc != HX_OK) return rc;
    if (c->sample_cap < static_cast<int>(batch)) {
        cudaFree(c->xin);
        cudaFree(c->tgt);
        c->xin = c->tgt = nullptr;
        c->sample_cap = 0;
        HX_CUDA_TRY(cudaMalloc(&c->xin, batch * sizeof(float2)));
        HX_CUDA_TRY(cudaMalloc(&c->tgt, batch * sizeof(float2)));
        c->sample_cap = static_cast<int>(batch);
    }
    // cosine learning-rate decay over the call
    for (uint32_t it = 0; it < iters && rc == HX_OK; ++it) {
        hx::gather_closure_kernel<<<(batch + 127) / 128, 128, 0, n->stream>>>(
            c->din, c->dout, c->up_local, c->top_occ, c->mode_bath_d, c->vdiag, c->hdiag, c->inv_e, c->n_snap,
            c->n_top, c->n_up, c->M, c->maxd, c->logd, static_cast<float>(1.0 / c->s_in),
            static_cast<float>(1.0 / c->s_out), n->in_ld, static_cast<int>(batch), seed + it, n->X, c->xin, c->tgt);
        mlp_forward(n, static_cast<int>(batch), n->stream);
        hx::closure_loss_kernel<<<148, 256, 0, n->stream>>>(n->Y, c->xin, c->tgt, static_cast<int>(batch), n->dYf,
                                                            n->dYh, n->partial);
        mlp_backward_dy(n, static_cast<int>(batch), n->stream);
        float l = 0.f;
        if (loss_trace) rc = mlp_loss_of_partials(n, static_cast<double>(batch), &l, n->stream);
        if (loss_trace) loss_trace[it] = l;
        const float f = 0.5f * (1.f + std::cos(3.14159265358979f * static_cast<float>(it) / static_cast<float>(iters)));
        mlp_adam(n, lr * (0.05f + 0.95f * f), n->stream);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = hx::cuda_fail(e, "closure training");
    }
    if (rc != HX_OK) return rc;
    if ((rc = build_table(c, n->stream)) != HX_OK) return rc;
    HX_CUDA_TRY(cudaStreamSynchronize(n->stream));
    return HX_OK;
}

int hx_closure_set_scales(hx_closure* c, double s_in, double s_out)
{
    if (!c) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL closure");
    if (!(s_in > 0.0) || !(s_out > 0.0)) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "scales must be positive");
    c->s_in = s_in;
    c->s_out = s_out;
    c->scaled = true;
    c->table_version = ~0ull;  // rebuilt with the new scales before the next stage
    return HX_OK;
}

}  // extern "C"
