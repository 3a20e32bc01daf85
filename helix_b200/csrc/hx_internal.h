// Internal declarations of the helix_b200 CUDA library.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "helix_b200.h"

struct hx_ctx;

namespace hx {

// Thread-local last-error text behind hx_last_error().
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

#define HX_CUDA_TRY(expr)                                     \
    do {                                                      \
        cudaError_t hx_e_ = (expr);                           \
        if (hx_e_ != cudaSuccess) return ::hx::cuda_fail(hx_e_, #expr); \
    } while (0)

// ---------------------------------------------------------------------------
// Host math (hx_host.cpp)
// ---------------------------------------------------------------------------

// [K-1/K] Pade poles/residues of the Bose function (src/psd/psd.cu:12-113).
bool psd_bose(int K, double* poles, double* residues);

// Per-bath constants of the right-hand side, in the reference's form
// (src/initialize.cu:160-218, omega0 = 1):
//   nu[k]      nu_0 = gamma, nu_k = xi_k / beta
//   theta_c    Im KThetaCommutate   = (beta gamma/2) cot(beta gamma/2) zeta/beta
//   theta_a    KThetaAntiCommutate  = (beta gamma/2) zeta / beta
//   phi[k-1]   Im KPhi_k            = (zeta/beta) 2 eta_k gamma^2 / (nu_k^2 - gamma^2)
//   xi         KXi (real)           = sigma zeta / beta
//   counter    Im KXiCounter        = zeta (beta gamma/2) / beta
struct BathConst {
    int K = 0;
    int offset = 0;  // first mode index
    std::vector<double> nu, phi;
    double theta_c = 0, theta_a = 0, xi = 0, counter = 0;
};
bool bath_constants(double beta, double gamma, double zeta, int K, BathConst& out);

uint64_t binom_u64(int n, int k);

// Spin p when v (d values) is sigma_z of spin p, i.e. v[r] = +1 where bit p
// of r is set and -1 elsewhere; -1 for any other diagonal.
int pauli_spin(const double* v, int D);

// ---------------------------------------------------------------------------
// Device-side parameter blocks
// ---------------------------------------------------------------------------

constexpr int kMaxLogD = 6;       // slab-in-shared-memory stage kernels: d <= 64
constexpr int kMaxLogDFlip = 12;  // flip-path stage kernels (hx_flip.cu): d <= 4096
constexpr int kMaxModes = 128;
constexpr int kMaxBaths = 64;

// Read-only per-context tables used by the stage kernel.
struct StageTables {
    const int32_t* edges;    // [H][2M] reference layout, sentinel H
    const double* acoef;     // [H][M]  down-commutator weight a_{n,m}
    const double* bcoef;     // [H][J]  down anti-commutator weight b_{n,j} (Drude mode)
    const double* gsum;      // [H]     sum_m nu_m n_m
    const double* hdiag;     // [d]
    const double* hflip;     // [log2 d]
    const double* vdiag;     // [J][d]
    const double* xi;        // [J]
    const double* counter;   // [J]
    const int32_t* bath_off; // [J+1]  mode offsets
    const int32_t* order;    // [H] processing order (ADO index per CTA), or nullptr
    int* error_flag;         // device error word
    long long H;
    int M, J, logd;
};

enum BaseKind : int { kBaseSelf = 0, kBaseRho = 1, kBaseZero = 2 };

// Hermitian-packed slab.  Every ADO of this hierarchy stays Hermitian: H and
// the V_j are Hermitian, every commutator term carries a factor -i times a
// real weight and every anti-commutator term a real weight, so L maps
// Hermitian matrices to Hermitian matrices, and the initial state is
// Hermitian.  A packed slab keeps the upper triangle r <= c of a d x d
// Hermitian matrix (d = 2^logd >= 2) as d/2 packed rows of d + 1 elements:
// packed row s holds row s from the diagonal on (d - s elements), then row
// d-1-s from the diagonal on (s + 1 elements).  Consecutive packed elements
// are consecutive columns of at most two matrix rows, and d(d+1)/2 elements
// replace d^2.
__host__ __device__ inline int herm_elems(int logd) { return (1 << (logd - 1)) * ((1 << logd) + 1); }
// Packed position of element (r, c), r <= c.
__host__ __device__ inline int herm_index(int r, int c, int logd)
{
    const int D = 1 << logd;
    return r < (D >> 1) ? r * (D + 1) + (c - r) : (D - 1 - r) * (D + 1) + c + 1;
}
// Element (r, c), r <= c, at packed position i.
__host__ __device__ inline void herm_coords(int i, int logd, int& r, int& c)
{
    const int D = 1 << logd;
    const int s = i / (D + 1), t = i - s * (D + 1);
    if (t < D - s) {
        r = s;
        c = s + t;
    } else {
        r = D - 1 - s;
        c = t - 1;
    }
}
// Packed copy of a full d x d table (upper triangle).
void launch_pack_herm(const double2* full, int logd, double2* packed, cudaStream_t s);
// count full slabs: the Hermiticity check of the host packer (relative to each slab's largest element; *bad
// is lowered to the index first + k of a slab that fails it), then the packing into slabs first.. of `packed`
void launch_herm_check(const double2* full, long long count, int logd, double rel_tol, double* scale2,
                       long long first, int* bad, cudaStream_t s);
void launch_herm_pack(const double2* full, long long count, int logd, long long first, double2* packed,
                      cudaStream_t s);
// The same packing into complex64 slabs (mixed precision).
void launch_herm_pack_f32(const double2* full, long long count, int logd, long long first, float2* packed,
                          cudaStream_t s);
// Full row-major complex matrix (2 d^2 doubles) from a packed slab, on the host.
void unpack_herm_host(const double2* pk, int logd, double* out);

// out_n = base_n + alpha * L(u)_n for every ADO n
void launch_stage(const StageTables& t, const double2* u, const double2* rho, double2* out,
                  double alpha, int base_kind, cudaStream_t s);

// Fused multi-CTA stage kernel for d = 32, 64 (hx_fused.cu)
struct FusedArgs {
    const double2* diag;     // [d*d] ADO-independent diagonal coefficient table
    const double* vdiag;     // [J][d]
    const double* hflip;     // [log2 d]
    const double* gsum;      // [H]
    const int* ent_count;    // [H]
    const int32_t* ent_slab; // [H][2M] neighbour slab
    const int32_t* ent_bath; // [H][2M] bath | (keep-in-L2 flag << 16)
    const double* ent_wc;    // [H][2M] commutator weight
    const double* ent_wa;    // [H][2M] anti-commutator weight
    const int32_t* order;    // [H] or nullptr
    const int8_t* ado_keep;  // [H] 1 = slab below the top tier (evict_last in L2)
    const int32_t* slot;     // [H] slot of a tier L-1 ADO in U, else -1
    const double2* U;        // [S][d*d] up terms of tier L-1 (hx_upterm.cu)
    int* error_flag;
    long long H;
    int M, J, logd;
    int herm;                // 1: slabs Hermitian-packed (herm_elems(logd) elements), diag and U packed too
    const int* vbit;         // [J] spin of V_j = sigma_z(spin) for every bath (pauli = 1), else nullptr
    int pauli;
    const double* hdiag;     // [d] diagonal of H (E_r)
    const double* xi;        // [J] low-temperature correction coefficients
};
bool fused_supported(int logd, int M, int J, int herm);
// BF16 GEMM on the tensor cores (hx_tcgemm.cu): C = A B^T, A [M x K] and B [N x K] row-major, FP32
// accumulation, with the closure network's epilogues.  Returns false (nothing launched) when the operands
// do not suit the tensor loads (16-byte aligned bases, leading dimensions multiples of 8).
enum TcEpi : int { kTcEpiBiasGelu = 0, kTcEpiBias = 1, kTcEpiStore = 2, kTcEpiGeluBack = 3 };
struct TcGemmOut {
    int kind;           // TcEpi
    const float* bias;  // [N]
    float* outf;        // FP32 result (the pre-activation for kTcEpiBiasGelu)
    void* outh;         // BF16 result (the GELU output, or dZ for kTcEpiGeluBack)
    const float* aux;   // pre-activation Z for kTcEpiGeluBack
    int ldo;
};
bool tc_gemm_eligible(const void* A, int lda, const void* B, int ldb);
bool tc_gemm(int M, int N, int K, const void* A, int lda, const void* B, int ldb, const TcGemmOut& o, int* err,
             cudaStream_t s);
// Sum of up to three products A_p B_p^T in one accumulator, BF16 or FP32 operands (the latter on the TF32
// path): the terms of a split-precision product.  Leading dimensions multiples of 16 bytes.
struct TcPair {
    const void* A;
    int lda;
    const void* B;
    int ldb;
};
bool tc_gemm_sum(int M, int N, int K, int npairs, const TcPair* pairs, bool tf32, const TcGemmOut& o, int* err,
                 cudaStream_t s);
// The driver entry point and kernel attributes the tensor-core GEMM needs are available.
bool tc_gemm_ready(bool tf32);
// C [M x N] = A_hi B_hi^T + A_hi B_lo^T + A_lo B_hi^T with the TF32 split of the FP32 operand A done in
// shared memory (B_hi, B_lo exact TF32 values, N <= 256 per tile column); FP32 result, row length ldo.
bool tc_split_gemm(int M, int N, int K, const float* A, int lda, const float* Bhi, const float* Blo, int ldb,
                   float* out, int ldo, int* err, cudaStream_t s);
void launch_transpose_bf16(const void* in, int rows, int cols, int ld_in, void* out, int ld_out, cudaStream_t s);
// d <= 16, full slabs, sigma_z couplings, every up term in the entry lists: batched gathers (hx_small.cu)
size_t small_smem(int logd, int M);
bool small_supported(int logd, int M, int pauli);
// The same, one cooperative launch per integrator step (order >= 2), stages separated by grid barriers on
// an arrival counter (*gcount, zeroed by the caller once; every launch leaves it at zero).  Returns 1 when
// launched (with dry: when it would launch), 0 when the ADOs do not fit the resident CTAs (up to 4 per
// CTA), -1 when refused.
size_t small_step_smem(int logd, int M, int per);
// Grid-barrier waits of small_step_kernel: polls before giving up (and setting the error word), and an
// offset added to every barrier's arrival target (nonzero only to make the waits run out on purpose).
struct StepWait {
    unsigned skew = 0;
    unsigned max_polls = 1u << 24;
};
int launch_small_step(const FusedArgs& a, double2* rho, double2* ua, double2* ub, double dt, int order,
                      unsigned* gcount, cudaStream_t s, bool dry, StepWait w = StepWait{});
bool launch_small(const FusedArgs& a, const double2* u, const double2* rho, double2* out, double alpha,
                  int base_kind, cudaStream_t s);
bool prepare_fused(int logd, int M, int J, int herm);  // raises the shared-memory limit; call before stream capture
bool launch_fused(const FusedArgs& a, const double2* u, const double2* rho, double2* out, double alpha,
                  int base_kind, cudaStream_t s);
void launch_entries(const int32_t* rows, const int32_t* edges, const double* acoef, const double* bcoef,
                    const int32_t* bath_off, long long H, int M, int J, int max_depth, int* count, int32_t* slab,
                    int32_t* bath, double* wc, double* wa, int8_t* keep, cudaStream_t s);
void launch_diag_table(const double* hdiag, const double* vdiag, const double* xi, const double* kappa, int D, int J,
                       double2* T, cudaStream_t s);

// Up term of tier L-1, element-tiled (hx_upterm.cu)
struct UpTermArgs {
    const double* vdiag;    // [J][d]
    const int* cnt;         // [S]
    const int32_t* slab;    // [S][M] up neighbour per mode
    const int32_t* bath;    // [S][M]
    const int32_t* bath_off;// [J+1]
    int S, M, J, logd;
    int herm;               // 1: slabs and U Hermitian-packed
};
void launch_upterm(const UpTermArgs& a, const double2* u, double2* U, cudaStream_t s);

void launch_upterm_tables(const int32_t* rows, const int32_t* edges, const int32_t* mode_bath, long long H, int M,
                          int top, int32_t* slot, int* S_out, int32_t* ado, int* cnt, int32_t* slab, int32_t* bath,
                          cudaStream_t s);

// Stage kernels for 128 <= d <= 1024 with diagonal couplings, in double or
// in single precision with complex64 storage (hx_large.cu)
template <typename R> struct C2Of;
template <> struct C2Of<double> { using type = double2; };
template <> struct C2Of<float> { using type = float2; };
template <typename R> using C2 = typename C2Of<R>::type;

template <typename R>
struct LargeArgs {
    const C2<R>* diag;       // [d*d] ADO-independent diagonal coefficient table
    const R* vdiag;          // [J][d]
    const R* hflip;          // [log2 d]
    const double* gsum;      // [H]
    const int* ent_count;    // [H]
    const int32_t* ent_slab; // [H][2M]
    const int32_t* ent_bath; // [H][2M] bath (low 16 bits)
    const double* ent_wc;    // [H][2M]
    const double* ent_wa;    // [H][2M]
    const int32_t* slot;     // [H] slot of a tier L-1 ADO in U, else -1
    const C2<R>* U;          // [S][d*d], or [S][herm_elems] with herm
    int* error_flag;
    long long H;
    int M, J, logd;
    int first_ado;           // 1 when ADO 0 runs in double precision (ado0_kernel)
    int herm;                // 1: slabs, diag and U Hermitian-packed (herm_band_kernel)
    // dense H on the tensor cores (HX_FLAG_DENSE_H, full slabs): Y_n = X_n H_off for every ADO (H_off: H
    // without its diagonal), in the state layout; X_n is Hermitian, so H_off X_n = Y_n^dagger and
    // -i[H_off, X_n]_rc = -i(conj(Y_cr) - Y_rc)
    const C2<R>* dense_y;
};
template <typename R>
struct LargeUpArgs {
    const R* vdiag;          // [J][d]
    const int32_t* slab;     // [S][M]
    const int32_t* bath_off; // [J+1]
    int S, M, J, logd;
    int herm;                // 1: slabs and U Hermitian-packed
};
struct Ado0Args {
    const double2* diag;     // [d*d]
    const double* vdiag;     // [J][d]
    const double* hflip;     // [log2 d]
    const int* ent_count;    // entries of ADO 0 (first row of the context's tables)
    const int32_t* ent_slab;
    const int32_t* ent_bath;
    const double* ent_wc;
    const double* ent_wa;
    int M, J, logd;
    int herm;                // 1: the slabs (and diag) are Hermitian-packed
    const double2* dense_z;  // dense H: Z_0 = X_0 H_off in FP64 ([d][d], from zgemm_kernel), else nullptr
};
bool large_supported(int logd, int M, int J);
template <typename R> bool prepare_large(const LargeArgs<R>& a);  // shared-memory limit; call before capture
template <typename R>
bool launch_large(const LargeArgs<R>& a, const C2<R>* u, const C2<R>* rho, C2<R>* out, double alpha, int base_kind,
                  cudaStream_t s);
template <typename R> void launch_large_upterm(const LargeUpArgs<R>& a, const C2<R>* u, C2<R>* U, cudaStream_t s);
// Z = X H for one d x d complex pair in FP64, row-major (d = 2^logd >= 32): ADO 0 of a dense-H stage
void launch_zgemm(const double2* x, const double2* h, double2* z, int logd, cudaStream_t s);
void launch_ado0(const Ado0Args& a, const double2* u0, const float2* u, const double2* rho0, double2* out0,
                 float2* out32, double alpha, int base_kind, cudaStream_t s);
void launch_d2f(const double2* in, float2* out, long long n, cudaStream_t s);
void launch_vec_d2f(const double* in, float* out, long long n, cudaStream_t s);

// Whether a closure was made for a hierarchy of this dimension, mode count and size (hx_mlp.cu)
bool closure_matches_hierarchy(const ::hx_closure* cl, int d, int M, long long H);
// Learned closure term of a stage: out_top += alpha * (dropped up coupling) (hx_mlp.cu)
int closure_stage(::hx_closure* cl, const ::hx_ctx* c, const double2* u, double2* out, double alpha,
                  cudaStream_t s);

// Argument blocks of a context's fused and up-term kernels (hx_ctx.cu)
FusedArgs fused_args_of(const ::hx_ctx* c);
UpTermArgs upterm_args_of(const ::hx_ctx* c);

// Two-pass stage for coupling operators with spin-flip parts, any d (hx_flip.cu)
struct FlipArgs {
    const int32_t* edges;    // [H][2M]
    const double* acoef;     // [H][M]
    const double* bcoef;     // [H][J]
    const double* gsum;      // [H]
    const double* hdiag;     // [d]
    const double* hflip;     // [log2 d]
    const double* vdiag;     // [J][d]
    const double* vflip;     // [J][log2 d]
    const double* xi;        // [J]
    const double* counter;   // [J]
    const int32_t* bath_off; // [J+1]
    long long H;
    int M, J, logd;
};
// B (2 J H d*d complex) receives [V_j, u_n], then {V_j, u_n}; then out = base + alpha L(u).
void launch_flip_stage(const FlipArgs& a, const double2* u, double2* B, const double2* rho, double2* out,
                       double alpha, int base_kind, cudaStream_t s);

// Two-pass stage for general sparse Hermitian H and V_j (hx_csr.cu).
// Operator k (0 = H, 1 + j = V_j) has row pointers ptr[k (d+1) .. k (d+1) + d]
// (absolute offsets into col / val).
struct CsrArgs {
    const int32_t* ptr;      // [(J+1)(d+1)]
    const int32_t* col;
    const double2* val;
    const int32_t* edges;    // [H][2M]
    const double* acoef;     // [H][M]
    const double* bcoef;     // [H][J]
    const double* gsum;      // [H]
    const double* xi;        // [J]
    const double* counter;   // [J]
    const int32_t* bath_off; // [J+1]
    long long H;
    int M, J, logd;
};
void launch_csr_stage(const CsrArgs& a, const double2* u, double2* B, const double2* rho, double2* out, double alpha,
                      int base_kind, cudaStream_t s);
// out[0] = Re Tr(H rho_0) with H in CSR (operator 0), out[1..2] = Tr rho_0.
void launch_observables_csr(const double2* rho0, int logd, const int32_t* ptr, const int32_t* col,
                            const double2* val, double* out, cudaStream_t s);

// Tables on the device (hx_tables.cu)
int build_tables_device(int M, int D, long long H, int32_t* d_rows, int32_t* d_edges, cudaStream_t s);
// Same table kernel with a binomial table (rows n <= M + D, columns k <= M,
// kcols = M + 1) that the caller already placed in device memory.
void launch_tables_with_binomials(const unsigned long long* d_binom, int kcols, int M, int D, long long H,
                                  int32_t* d_rows, int32_t* d_edges, cudaStream_t s);
void launch_coefficients(const int32_t* rows, long long H, int M, int J, const int32_t* mode_bath,
                         const int32_t* mode_k, const double* nu, const double* theta_c,
                         const double* theta_a, const double* phi, const int32_t* bath_off,
                         double* acoef, double* bcoef, double* gsum, cudaStream_t s);

// Observables of rho_0: energy = Re Tr(H rho_0), trace.  Optionally copies
// rho_0 into rho0_copy.  out[0] = energy, out[1] = Re tr, out[2] = Im tr.
// herm = 1: rho0 is a Hermitian-packed slab.
void launch_observables(const double2* rho0, int logd, int herm, const double* hdiag, const double* hflip,
                        double2* rho0_copy, double* out, cudaStream_t s);

void launch_finite_check(const double2* x, long long n, int* flag, cudaStream_t s);
// Zero n elements, then rho[one] = 1 (the |d-1><d-1| element of ADO 0).
void launch_init_state(double2* rho, long long n, long long one, cudaStream_t s);

}  // namespace hx

struct hx_ctx {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    int d = 0, logd = 0, M = 0, J = 0, order = 4;
    long long H = 0;
    double dt = 0.0;
    uint64_t steps_done = 0;
    size_t slab = 0;   // d*d: elements of one slab as read and written through the C ABI
    bool herm = false; // state buffers hold Hermitian-packed slabs (fused path, d = 32, 64)
    size_t slab_store = 0; // elements of one slab in the device buffers (d*d, or herm_elems(logd))
    // device memory
    double2* rho = nullptr;
    double2* ua = nullptr;
    double2* ub = nullptr;
    int32_t* rows = nullptr;
    int32_t* edges = nullptr;
    double* acoef = nullptr;
    double* bcoef = nullptr;
    double* gsum = nullptr;
    double* hdiag = nullptr;
    double* hflip = nullptr;
    double* vdiag = nullptr;
    double* vflip = nullptr;      // [J][log2 d]
    bool use_flip = false;        // two-pass flip path (flips in V, or d > 1024)
    bool use_csr = false;         // two-pass path for general sparse H / V_j (hx_csr.cu)
    int32_t* csr_ptr = nullptr;   // [(J+1)(d+1)] operator 0 = H, 1 + j = V_j
    int32_t* csr_col = nullptr;
    double2* csr_val = nullptr;
    bool use_large = false;       // band kernels for 128 <= d <= 1024, diagonal V (hx_large.cu)
    bool mixed = false;           // complex64 hierarchy, ADO 0 in double precision
    hx_closure* closure = nullptr; // learned closure term added by every stage (hx_mlp.cu)
    float2* rho32 = nullptr;      // mixed: complex64 state buffers (rho, ua, ub mirror them)
    float2* ua32 = nullptr;
    float2* ub32 = nullptr;
    float2* U32 = nullptr;        // mixed: up terms of tier L-1
    float2* diag32 = nullptr;
    float* vdiag32 = nullptr;
    float* hflip32 = nullptr;
    double2* Bbuf = nullptr;      // [2][J][H][d*d] [V_j, u_n] then {V_j, u_n} (flip and CSR paths)
    double* xi = nullptr;
    double* counter = nullptr;
    int32_t* bath_off = nullptr;
    int* error_flag = nullptr;
    // fused stage-kernel tables (d = 32, 64)
    bool use_fused = false;
    bool use_small = false;       // d <= 16 sigma_z stage kernel (hx_small.cu)
    bool use_small_step = false;  // ... as one cooperative launch per step (small_step_kernel)
    unsigned* gbar = nullptr;     // grid-barrier arrival counter of small_step_kernel
    bool stall_next_step = false; // hx_ctx_inject_wait_timeout: the next step's barriers cannot complete
    int sm_count = 0;
    int up_slots = 0;             // ADOs in tier L-1
    int32_t* up_slot = nullptr;   // [H]
    int32_t* up_ado = nullptr;    // [S]
    int* up_cnt = nullptr;        // [S]
    int32_t* up_slab = nullptr;   // [S][M]
    int32_t* up_bath = nullptr;   // [S][M]
    double2* U = nullptr;         // [S][d*d]
    double2* diag_table = nullptr;
    double2* diag_herm = nullptr; // packed diagonal table (herm)
    int* vbit = nullptr;          // [J] sigma_z spin of each coupling operator, when every one is a sigma_z
    int* ent_count = nullptr;
    int32_t* ent_slab = nullptr;
    int32_t* ent_bath = nullptr;
    double* ent_wc = nullptr;
    double* ent_wa = nullptr;
    int32_t* order_perm = nullptr;
    int8_t* ado_keep = nullptr;
    double* obs = nullptr;        // [3] observables scratch
    double2* trace_buf = nullptr; // per-step rho_0 chunk
    double* energy_buf = nullptr;
    int trace_cap = 0;
    double* pinned = nullptr;     // pinned staging for traces
    size_t pinned_bytes = 0;
    double2* state_pinned = nullptr; // pinned staging for packed whole-state transfers
    double* pack_scale = nullptr;    // [H] per-slab scale of the device-side packer (first use)
    int* pack_bad = nullptr;         // first ADO that failed the packer's Hermiticity check
    // dense H (HX_FLAG_DENSE_H): Y = X H on the tensor cores before every stage
    bool dense = false;
    float* dense_hr = nullptr;    // [2d][2d] real form of H_off, K-major: row 2c = (Re H_kc, -Im H_kc)_k,
    float* dense_hr_lo = nullptr; //   row 2c+1 = (Im H_kc, Re H_kc)_k; and its TF32 residual
    float2* dense_y = nullptr;    // [H][d][d] Y_n = X_n H_off (H without its diagonal)
    double2* dense_h64 = nullptr; // [d][d] H_off in FP64 (ADO 0's product)
    double2* dense_z0 = nullptr;  // [d][d] Z_0 = X_0 H_off in FP64
    bool launch_failed = false;   // a stage could not be enqueued (reported by the next error check)
    size_t state_pinned_elems = 0;
    size_t device_bytes = 0;
    hx_counters counters{};
    std::vector<double> h_hdiag, h_hflip;
};
