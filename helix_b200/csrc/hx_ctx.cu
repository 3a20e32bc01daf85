// Context lifecycle and the C ABI entry points of helix_b200 that touch the
// device.  One context = one HEOM problem resident on one GPU: hierarchy
// tables, per-ADO weights, operator diagonals and three state buffers
// (rho and two stage buffers; the Horner form needs no separate sum buffer).
//
// Replaces the reference's process-global device state (src/matrix_storage.cu:4-23),
// its session lifecycle (src/library/legacy_runtime_session.cu:53-118) and
// develop() (src/liouville.cu:502-590).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "hx_internal.h"

using hx::fail;

namespace {

template <typename T>
int dev_alloc(hx_ctx* c, T** p, size_t count)
{
    *p = nullptr;
    if (count == 0) count = 1;
    const size_t bytes = count * sizeof(T);
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), bytes);
    if (e != cudaSuccess) return hx::cuda_fail(e, "cudaMalloc");
    c->device_bytes += bytes;
    return HX_OK;
}

template <typename T>
int upload(hx_ctx* c, T* dst, const std::vector<T>& src)
{
    if (src.empty()) return HX_OK;
    HX_CUDA_TRY(cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, c->stream));
    c->counters.h2d_bytes += src.size() * sizeof(T);
    return HX_OK;
}

void release(hx_ctx* c)
{
    if (!c) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    void* ptrs[] = {c->rho, c->ua, c->ub, c->rows, c->edges, c->acoef, c->bcoef, c->gsum, c->hdiag,
                    c->hflip, c->vdiag, c->xi, c->counter, c->bath_off, c->error_flag, c->obs,
                    c->trace_buf, c->energy_buf, c->diag_table, c->ent_count, c->ent_slab, c->ent_bath,
                    c->ent_wc, c->ent_wa, c->order_perm, c->ado_keep, c->up_slot, c->up_ado, c->up_cnt,
                    c->up_slab, c->up_bath, c->U, c->vflip, c->Bbuf, c->rho32, c->ua32, c->ub32,
                    c->U32, c->diag32, c->vdiag32, c->hflip32, c->diag_herm, c->vbit, c->csr_ptr, c->csr_col,
                    c->csr_val, c->pack_scale, c->pack_bad, c->dense_hr, c->dense_hr_lo, c->dense_y,
                    c->dense_h64, c->dense_z0, c->gbar};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (c->pinned) cudaFreeHost(c->pinned);
    if (c->state_pinned) cudaFreeHost(c->state_pinned);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
}

hx::StageTables tables_of(const hx_ctx* c)
{
    hx::StageTables t{};
    t.edges = c->edges;
    t.acoef = c->acoef;
    t.bcoef = c->bcoef;
    t.gsum = c->gsum;
    t.hdiag = c->hdiag;
    t.hflip = c->hflip;
    t.vdiag = c->vdiag;
    t.xi = c->xi;
    t.counter = c->counter;
    t.bath_off = c->bath_off;
    t.order = nullptr;
    t.error_flag = c->error_flag;
    t.H = c->H;
    t.M = c->M;
    t.J = c->J;
    t.logd = c->logd;
    return t;
}

}  // namespace

hx::FusedArgs hx::fused_args_of(const hx_ctx* c)
{
    hx::FusedArgs a{};
    a.diag = c->herm ? c->diag_herm : c->diag_table;
    a.vdiag = c->vdiag;
    a.hflip = c->hflip;
    a.gsum = c->gsum;
    a.ent_count = c->ent_count;
    a.ent_slab = c->ent_slab;
    a.ent_bath = c->ent_bath;
    a.ent_wc = c->ent_wc;
    a.ent_wa = c->ent_wa;
    a.order = c->order_perm;
    a.ado_keep = c->ado_keep;
    a.slot = c->up_slot;
    a.U = c->U;
    a.error_flag = c->error_flag;
    a.H = c->H;
    a.M = c->M;
    a.J = c->J;
    a.logd = c->logd;
    a.herm = c->herm ? 1 : 0;
    a.vbit = c->vbit;
    a.pauli = c->vbit ? 1 : 0;
    a.hdiag = c->hdiag;
    a.xi = c->xi;
    return a;
}

hx::UpTermArgs hx::upterm_args_of(const hx_ctx* c)
{
    return hx::UpTermArgs{c->vdiag, c->up_cnt, c->up_slab, c->up_bath, c->bath_off, c->up_slots,
                          c->M,     c->J,      c->logd,    c->herm ? 1 : 0};
}

void hx::unpack_herm_host(const double2* pk, int logd, double* out)
{
    const int D = 1 << logd, P = hx::herm_elems(logd);
    for (int i = 0; i < P; ++i) {
        int r, c;
        hx::herm_coords(i, logd, r, c);
        const double2 v = pk[i];
        out[2 * (static_cast<size_t>(r) * D + c)] = v.x;
        out[2 * (static_cast<size_t>(r) * D + c) + 1] = v.y;
        out[2 * (static_cast<size_t>(c) * D + r)] = v.x;
        out[2 * (static_cast<size_t>(c) * D + r) + 1] = r == c ? v.y : -v.y;
    }
}

namespace {

hx::FlipArgs flip_args_of(const hx_ctx* c)
{
    hx::FlipArgs a{};
    a.edges = c->edges;
    a.acoef = c->acoef;
    a.bcoef = c->bcoef;
    a.gsum = c->gsum;
    a.hdiag = c->hdiag;
    a.hflip = c->hflip;
    a.vdiag = c->vdiag;
    a.vflip = c->vflip;
    a.xi = c->xi;
    a.counter = c->counter;
    a.bath_off = c->bath_off;
    a.H = c->H;
    a.M = c->M;
    a.J = c->J;
    a.logd = c->logd;
    return a;
}

hx::LargeArgs<double> large_args64(const hx_ctx* c)
{
    hx::LargeArgs<double> a{};
    a.diag = c->herm ? c->diag_herm : c->diag_table;
    a.vdiag = c->vdiag;
    a.hflip = c->hflip;
    a.gsum = c->gsum;
    a.ent_count = c->ent_count;
    a.ent_slab = c->ent_slab;
    a.ent_bath = c->ent_bath;
    a.ent_wc = c->ent_wc;
    a.ent_wa = c->ent_wa;
    a.slot = c->up_slot;
    a.U = c->U;
    a.error_flag = c->error_flag;
    a.H = c->H;
    a.M = c->M;
    a.J = c->J;
    a.logd = c->logd;
    a.first_ado = 0;
    a.herm = c->herm ? 1 : 0;
    return a;
}

hx::LargeArgs<float> large_args32(const hx_ctx* c)
{
    hx::LargeArgs<float> a{};
    a.diag = c->diag32;
    a.vdiag = c->vdiag32;
    a.hflip = c->hflip32;
    a.gsum = c->gsum;
    a.ent_count = c->ent_count;
    a.ent_slab = c->ent_slab;
    a.ent_bath = c->ent_bath;
    a.ent_wc = c->ent_wc;
    a.ent_wa = c->ent_wa;
    a.slot = c->up_slot;
    a.U = c->U32;
    a.error_flag = c->error_flag;
    a.H = c->H;
    a.M = c->M;
    a.J = c->J;
    a.logd = c->logd;
    a.first_ado = 1;
    a.herm = c->herm ? 1 : 0;
    a.dense_y = c->dense ? c->dense_y : nullptr;
    return a;
}

template <typename R>
hx::LargeUpArgs<R> large_up_args(const hx_ctx* c, const R* vdiag)
{
    return hx::LargeUpArgs<R>{vdiag, c->up_slab, c->bath_off, c->up_slots, c->M, c->J, c->logd, c->herm ? 1 : 0};
}

hx::Ado0Args ado0_args(const hx_ctx* c)
{
    return hx::Ado0Args{c->herm ? c->diag_herm : c->diag_table, c->vdiag, c->hflip, c->ent_count, c->ent_slab, c->ent_bath,
                        c->ent_wc, c->ent_wa, c->M, c->J, c->logd, c->herm ? 1 : 0,
                        c->dense ? c->dense_z0 : nullptr};
}

// Index of a state buffer of the context: 0 = rho, 1 = ua, 2 = ub.
int buffer_id(const hx_ctx* c, const double2* p) { return p == c->rho ? 0 : (p == c->ua ? 1 : 2); }

// Dense H: Y_n = X_n H_off (H without its diagonal, which the band kernels
// apply exactly) for every ADO of the complex64 stage input u32, as the real
// product [H d x 2d] x [2d x 2d] (interleaved complex rows of X times the
// real form of H_off) in 3-term TF32 split form, X_hi H_hi + X_hi H_lo +
// X_lo H_hi with FP32 accumulation; the split of X happens in shared memory
// inside the GEMM (tc_split_gemm).  Returns kernels launched.
int launch_dense_product(hx_ctx* c, const float2* u32)
{
    const int d2 = 2 * c->d;
    if (!hx::tc_split_gemm(static_cast<int>(c->H * c->d), d2, d2, reinterpret_cast<const float*>(u32), d2,
                           c->dense_hr, c->dense_hr_lo, d2, reinterpret_cast<float*>(c->dense_y), d2, c->error_flag,
                           c->stream))
        c->launch_failed = true;
    return 1;
}

// One stage of the band kernels (hx_large.cu): the up-term kernel of tier
// L-1, the band kernel over the hierarchy and, in mixed precision, the
// double-precision kernel of ADO 0 (with a dense H, the tensor-core product
// first).  Returns kernels launched.
int launch_large_stage(hx_ctx* c, const double2* u, const double2* rho, double2* out, double alpha, int base)
{
    int k = 0;
    if (!c->mixed) {
        if (c->up_slots > 0) {
            hx::launch_large_upterm<double>(large_up_args<double>(c, c->vdiag), u, c->U, c->stream);
            ++k;
        }
        hx::launch_large<double>(large_args64(c), u, rho, out, alpha, base, c->stream);
        return k + 1;
    }
    float2* b32[3] = {c->rho32, c->ua32, c->ub32};
    const float2* u32 = b32[buffer_id(c, u)];
    float2* o32 = b32[buffer_id(c, out)];
    if (c->dense) {
        k += launch_dense_product(c, u32);
        hx::launch_zgemm(u, c->dense_h64, c->dense_z0, c->logd, c->stream);  // ADO 0 in FP64
        ++k;
    }
    if (c->up_slots > 0) {
        hx::launch_large_upterm<float>(large_up_args<float>(c, c->vdiag32), u32, c->U32, c->stream);
        ++k;
    }
    if (c->H > 1) {
        hx::launch_large<float>(large_args32(c), u32, c->rho32, o32, alpha, base, c->stream);
        ++k;
    }
    hx::launch_ado0(ado0_args(c), u, u32, rho, out, o32, alpha, base, c->stream);
    return k + 1;
}

int launch_stage_core(hx_ctx* c, const double2* u, const double2* rho, double2* out, double alpha, int base);

// One stage, then the learned closure term when one is attached.
int launch_stage_any(hx_ctx* c, const double2* u, const double2* rho, double2* out, double alpha, int base)
{
    int k = launch_stage_core(c, u, rho, out, alpha, base);
    if (c->closure) {
        hx::closure_stage(c->closure, c, u, out, alpha, c->stream);
        k += 1;  // the elementwise closure kernel (the coefficient table is rebuilt only after training)
    }
    return k;
}

// One stage: the two-pass flip path when V has spin-flip parts or d > 64; for
// d = 32, 64 the up-term kernel of tier L-1 followed by the fused multi-CTA
// kernel; the generic kernel otherwise.  Returns kernels launched.
int launch_stage_core(hx_ctx* c, const double2* u, const double2* rho, double2* out, double alpha, int base)
{
    if (c->use_large) return launch_large_stage(c, u, rho, out, alpha, base);
    if (c->use_csr) {
        const hx::CsrArgs a{c->csr_ptr, c->csr_col, c->csr_val, c->edges, c->acoef, c->bcoef, c->gsum,
                            c->xi,      c->counter, c->bath_off, c->H, c->M, c->J, c->logd};
        hx::launch_csr_stage(a, u, c->Bbuf, rho, out, alpha, base, c->stream);
        return 2;
    }
    if (c->use_flip) {
        hx::launch_flip_stage(flip_args_of(c), u, c->Bbuf, rho, out, alpha, base, c->stream);
        return 2;
    }
    if (c->use_small && hx::launch_small(hx::fused_args_of(c), u, rho, out, alpha, base, c->stream)) return 1;
    if (c->use_fused) {
        int k = 0;
        if (c->up_slots > 0) {
            hx::launch_upterm(hx::upterm_args_of(c), u, c->U, c->stream);
            ++k;
        }
        if (hx::launch_fused(hx::fused_args_of(c), u, rho, out, alpha, base, c->stream)) return k + 1;
    }
    hx::launch_stage(tables_of(c), u, rho, out, alpha, base, c->stream);
    return 1;
}

// Enqueue one integrator step (Horner form of the order-m Taylor polynomial).
int enqueue_step(hx_ctx* c)
{
    const int m = c->order;
    int launched = 0;
    if (c->use_small_step && !c->closure) {
        hx::StepWait w;
        if (c->stall_next_step) {  // test hook: one arrival more than the CTAs make, a short wait
            w.skew = 1;
            w.max_polls = 1u << 12;
            c->stall_next_step = false;
        }
        if (hx::launch_small_step(hx::fused_args_of(c), c->rho, c->ua, c->ub, c->dt, m, c->gbar, c->stream, false,
                                  w) != 1)
            c->launch_failed = true;
        c->counters.kernel_launches += 1;
        c->counters.stage_launches += m;
        c->steps_done += 1;
        return HX_OK;
    }
    if (m == 1) {
        launched += launch_stage_any(c, c->rho, c->rho, c->ua, c->dt, hx::kBaseSelf);
        std::swap(c->rho, c->ua);
        if (c->mixed) std::swap(c->rho32, c->ua32);
    } else {
        const double2* in = c->rho;
        double2* bufs[2] = {c->ua, c->ub};
        for (int s = 1; s <= m; ++s) {
            const double alpha = c->dt / static_cast<double>(m - s + 1);
            double2* out = (s == m) ? c->rho : bufs[(s - 1) & 1];
            launched += launch_stage_any(c, in, c->rho, out, alpha, s == 1 ? hx::kBaseSelf : hx::kBaseRho);
            in = out;
        }
    }
    c->counters.kernel_launches += launched;
    c->counters.stage_launches += m;
    c->steps_done += 1;
    return HX_OK;
}

// Energy and trace of rho_0 into out[0..2].
void launch_obs(hx_ctx* c, double* out)
{
    if (c->use_csr || c->dense)
        hx::launch_observables_csr(c->rho, c->logd, c->csr_ptr, c->csr_col, c->csr_val, out, c->stream);
    else hx::launch_observables(c->rho, c->logd, c->herm, c->hdiag, c->hflip, nullptr, out, c->stream);
}

int check_launch(const char* what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return hx::cuda_fail(e, what);
    return HX_OK;
}

int read_error_flag(hx_ctx* c)
{
    if (c->launch_failed) {
        c->launch_failed = false;
        return fail(HX_ERR_UNSUPPORTED_EXECUTION, "the tensor-core product of a stage could not be enqueued");
    }
    int flag = 0;
    HX_CUDA_TRY(cudaMemcpyAsync(&flag, c->error_flag, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    HX_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (flag != 0) {
        cudaMemsetAsync(c->error_flag, 0, sizeof(int), c->stream);
        if (c->gbar) cudaMemsetAsync(c->gbar, 0, sizeof(unsigned), c->stream);  // a barrier that gave up
        return fail(HX_ERR_DEVICE_TIMEOUT, "a device-side wait ran out of its iteration budget");
    }
    return HX_OK;
}

// Packed slab from a full row-major complex matrix (2 d^2 doubles); false
// when X - X^H exceeds rel_tol times the largest element.  Stores the upper
// triangle, or with `average` the upper triangle of the Hermitian part.
bool pack_herm_host(const double* in, int logd, double2* pk, double rel_tol = 1e-12, bool average = false)
{
    const int D = 1 << logd, P = hx::herm_elems(logd);
    double scale2 = 0.0;
    for (size_t e = 0; e < static_cast<size_t>(D) * D; ++e)
        scale2 = std::max(scale2, in[2 * e] * in[2 * e] + in[2 * e + 1] * in[2 * e + 1]);
    const double tol2 = rel_tol * rel_tol * scale2;
    for (int i = 0; i < P; ++i) {
        int r, c;
        hx::herm_coords(i, logd, r, c);
        const size_t up = static_cast<size_t>(r) * D + c, lo = static_cast<size_t>(c) * D + r;
        if (r != c) {
            const double dr = in[2 * up] - in[2 * lo], di = in[2 * up + 1] + in[2 * lo + 1];
            if (dr * dr + di * di > tol2) return false;
        }
        pk[i] = average ? make_double2(0.5 * (in[2 * up] + in[2 * lo]), 0.5 * (in[2 * up + 1] - in[2 * lo + 1]))
                        : make_double2(in[2 * up], in[2 * up + 1]);
    }
    return true;
}

// FP32 value rounded to TF32 (10 mantissa bits, to nearest, ties away from
// zero): the host twin of the device-side split in hx_tcgemm.cu.
float tf32_round_host(float v)
{
    uint32_t u;
    std::memcpy(&u, &v, sizeof(u));
    u = (u + 0x1000u) & 0xFFFFE000u;
    std::memcpy(&v, &u, sizeof(u));
    return v;
}

// f(k) for k in [0, n) on up to 16 host threads.
template <typename F>
void parallel_for(long long n, F f)
{
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int nt = static_cast<int>(std::min<long long>(n, std::min(16u, hw)));
    if (nt <= 1) {
        for (long long k = 0; k < n; ++k) f(k);
        return;
    }
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; ++t)
        pool.emplace_back([&, t] {
            for (long long k = n * t / nt; k < n * (t + 1) / nt; ++k) f(k);
        });
    for (auto& th : pool) th.join();
}

// Pinned staging for whole packed states (allocated on first use, kept).
int state_staging(hx_ctx* c, size_t elems)
{
    if (c->state_pinned_elems >= elems) return HX_OK;
    if (c->state_pinned) cudaFreeHost(c->state_pinned);
    c->state_pinned = nullptr;
    c->state_pinned_elems = 0;
    HX_CUDA_TRY(cudaMallocHost(&c->state_pinned, elems * sizeof(double2)));
    c->state_pinned_elems = elems;
    return HX_OK;
}

// count slabs of a packed device buffer into full matrices on the host.
int read_herm(hx_ctx* c, const double2* src, size_t count, double* out)
{
    const size_t n = count * c->slab_store;
    int rc = state_staging(c, n);
    if (rc != HX_OK) return rc;
    HX_CUDA_TRY(cudaMemcpyAsync(c->state_pinned, src, n * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
    HX_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->counters.d2h_bytes += n * sizeof(double2);
    const double2* pk = c->state_pinned;
    parallel_for(static_cast<long long>(count), [&](long long k) {
        hx::unpack_herm_host(pk + k * c->slab_store, c->logd, out + 2 * k * c->slab);
    });
    return HX_OK;
}

// One operator in compressed rows, host side, before upload.
struct HostCsr {
    std::vector<int32_t> ptr;  // d + 1, relative
    std::vector<int32_t> col;
    std::vector<double2> val;
};

// Copy and check a caller's CSR operator: row pointers from 0 to nnz and
// non-decreasing, columns in range, values finite, Hermitian to 1e-12 of its
// largest entry (duplicates summed).
bool take_csr(const hx_csr* a, int d, HostCsr& out, std::string& why, const std::string& name)
{
    if (!a->row_ptr || (a->nnz > 0 && (!a->col || !a->val))) {
        why = name + ": NULL array";
        return false;
    }
    if (a->row_ptr[0] != 0 || a->row_ptr[d] != static_cast<int32_t>(a->nnz)) {
        why = name + ": row pointers must run from 0 to nnz";
        return false;
    }
    out.ptr.assign(a->row_ptr, a->row_ptr + d + 1);
    out.col.assign(a->col, a->col + a->nnz);
    out.val.resize(a->nnz);
    std::map<std::pair<int, int>, std::pair<double, double>> sum;
    double big = 0.0;
    for (int r = 0; r < d; ++r) {
        if (out.ptr[r + 1] < out.ptr[r]) {
            why = name + ": row pointers decrease";
            return false;
        }
        for (int q = out.ptr[r]; q < out.ptr[r + 1]; ++q) {
            const int c = out.col[q];
            const double re = a->val[2 * q], im = a->val[2 * q + 1];
            if (c < 0 || c >= d) {
                why = name + ": column index out of range";
                return false;
            }
            if (!std::isfinite(re) || !std::isfinite(im)) {
                why = name + ": value is not finite";
                return false;
            }
            out.val[q] = make_double2(re, im);
            auto& v = sum[{r, c}];
            v.first += re;
            v.second += im;
        }
    }
    for (const auto& kv : sum) big = std::max(big, std::hypot(kv.second.first, kv.second.second));
    const double tol = 1e-12 * std::max(big, 1e-300);
    for (const auto& kv : sum) {
        const auto it = sum.find({kv.first.second, kv.first.first});
        const double tr = it == sum.end() ? 0.0 : it->second.first, ti = it == sum.end() ? 0.0 : -it->second.second;
        if (std::hypot(kv.second.first - tr, kv.second.second - ti) > tol) {
            why = name + ": operator is not Hermitian";
            return false;
        }
    }
    return true;
}

// CSR of diag(v) + sum_i w_i sigma_x(i).
HostCsr flip_csr(const double* v, const double* w, int d, int logd)
{
    HostCsr o;
    o.ptr.push_back(0);
    for (int r = 0; r < d; ++r) {
        o.col.push_back(r);
        o.val.push_back(make_double2(v ? v[r] : 0.0, 0.0));
        for (int i = 0; w && i < logd; ++i)
            if (w[i] != 0.0) {
                o.col.push_back(r ^ (1 << i));
                o.val.push_back(make_double2(w[i], 0.0));
            }
        o.ptr.push_back(static_cast<int32_t>(o.col.size()));
    }
    return o;
}

// The operator as diag(v) + sum_i w_i sigma_x(i) with real v and w, if it has
// that form: real entries only, every off-diagonal entry a single-spin flip,
// each flipped spin present once in every row with one value for all rows.
bool split_flip(const HostCsr& o, int d, int logd, std::vector<double>& v, std::vector<double>& w)
{
    v.assign(d, 0.0);
    w.assign(logd, 0.0);
    std::vector<int> count(logd, 0);
    for (int r = 0; r < d; ++r) {
        unsigned row_bits = 0;
        for (int q = o.ptr[r]; q < o.ptr[r + 1]; ++q) {
            const int c = o.col[q];
            const double2 a = o.val[q];
            if (a.y != 0.0) return false;
            if (c == r) {
                v[r] += a.x;
                continue;
            }
            const unsigned x = static_cast<unsigned>(r ^ c);
            if ((x & (x - 1)) != 0) return false;
            const int bit = __builtin_ctz(x);
            if (row_bits & x) return false;  // the same flip twice in one row
            row_bits |= x;
            if (count[bit] > 0 && w[bit] != a.x) return false;
            w[bit] = a.x;
            ++count[bit];
        }
    }
    for (int b = 0; b < logd; ++b)
        if (count[b] != 0 && count[b] != d) return false;
    return true;
}

// Mixed precision: the whole state as complex128 on the host (complex64
// hierarchy widened, ADO 0 from its double-precision slab); src32/src64 are
// matching buffers (rho32/rho, ua32/ua, ...).
int read_mixed(hx_ctx* c, const float2* src32, const double2* src64, double* out)
{
    if (c->herm) {
        const size_t P = c->slab_store, count = static_cast<size_t>(c->H) * P;
        std::vector<float2> tmp(count);
        std::vector<double2> pk0(P);
        HX_CUDA_TRY(cudaMemcpyAsync(tmp.data(), src32, count * sizeof(float2), cudaMemcpyDeviceToHost, c->stream));
        HX_CUDA_TRY(cudaMemcpyAsync(pk0.data(), src64, P * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
        HX_CUDA_TRY(cudaStreamSynchronize(c->stream));
        hx::unpack_herm_host(pk0.data(), c->logd, out);
        parallel_for(c->H - 1, [&](long long k1) {
            const long long k = k1 + 1;
            std::vector<double2> w(P);
            for (size_t i = 0; i < P; ++i) w[i] = make_double2(tmp[k * P + i].x, tmp[k * P + i].y);
            hx::unpack_herm_host(w.data(), c->logd, out + 2 * static_cast<size_t>(k) * c->slab);
        });
        c->counters.d2h_bytes += count * sizeof(float2) + P * sizeof(double2);
        return HX_OK;
    }
    const size_t count = static_cast<size_t>(c->H) * c->slab;
    std::vector<float2> tmp(count);
    HX_CUDA_TRY(cudaMemcpyAsync(tmp.data(), src32, count * sizeof(float2), cudaMemcpyDeviceToHost, c->stream));
    HX_CUDA_TRY(cudaMemcpyAsync(out, src64, c->slab * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
    HX_CUDA_TRY(cudaStreamSynchronize(c->stream));
    for (size_t i = c->slab; i < count; ++i) {
        out[2 * i] = tmp[i].x;
        out[2 * i + 1] = tmp[i].y;
    }
    c->counters.d2h_bytes += count * sizeof(float2) + c->slab * sizeof(double2);
    return HX_OK;
}

}  // namespace

extern "C" {

int hx_select_device(int device)
{
    if (device < 0) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "CUDA device index must be non-negative");
    HX_CUDA_TRY(cudaSetDevice(device));
    return HX_OK;
}

int hx_hierarchy_tables(uint32_t modes, uint32_t max_depth, int32_t* rows, int32_t* edges, uint64_t count)
{
    uint64_t H = 0;
    int rc = hx_hierarchy_size(modes, max_depth, &H);
    if (rc != HX_OK) return rc;
    if (count != H) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "count does not match hx_hierarchy_size");
    if (H == 0) return HX_OK;
    if (!rows || !edges) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL output buffer");
    if (H >= (1ull << 31)) return fail(HX_ERR_UNSUPPORTED_HIERARCHY, "hierarchy exceeds int32 indexing");
    cudaStream_t s = nullptr;
    HX_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    int32_t* dr = nullptr;
    int32_t* de = nullptr;
    cudaError_t e = cudaMalloc(&dr, H * modes * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&de, H * 2 * modes * sizeof(int32_t));
    if (e != cudaSuccess) {
        cudaFree(dr);
        cudaStreamDestroy(s);
        return hx::cuda_fail(e, "cudaMalloc tables");
    }
    rc = hx::build_tables_device(static_cast<int>(modes), static_cast<int>(max_depth), static_cast<long long>(H),
                                 dr, de, s);
    if (rc == HX_OK) {
        e = cudaMemcpyAsync(rows, dr, H * modes * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(edges, de, H * 2 * modes * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = hx::cuda_fail(e, "copy tables to host");
    }
    cudaFree(dr);
    cudaFree(de);
    cudaStreamDestroy(s);
    return rc;
}

int hx_ctx_create(const hx_problem* p, hx_ctx** out)
{
    if (!out) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL context output");
    *out = nullptr;
    if (!p) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL problem");
    const uint32_t d = p->dim;
    if (d < 2 || (d & (d - 1)) != 0)
        return fail(HX_ERR_INVALID_DIMENSION, "dim must be a power of two >= 2");
    int logd = 0;
    while ((1u << logd) < d) ++logd;
    if (logd > hx::kMaxLogDFlip)
        return fail(HX_ERR_UNSUPPORTED_EXECUTION, "dim must be at most 4096");
    if (!p->h_diag && !p->h_csr) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "h_diag is NULL");
    if (p->precision != HX_PRECISION_DOUBLE && p->precision != HX_PRECISION_MIXED)
        return fail(HX_ERR_UNSUPPORTED_PRECISION, "precision must be HX_PRECISION_DOUBLE or HX_PRECISION_MIXED");
    if (p->precision == HX_PRECISION_MIXED && (logd < 7 || logd > 10 || p->max_depth < 3))
        return fail(HX_ERR_UNSUPPORTED_PRECISION, "mixed precision needs 128 <= dim <= 1024 and max_depth >= 3");
    if (!(p->time_step > 0.0) || !std::isfinite(p->time_step))
        return fail(HX_ERR_INVALID_RUNTIME_OPTION, "time_step must be positive");
    if (p->integration_order < 1 || p->integration_order > 8)
        return fail(HX_ERR_INVALID_RUNTIME_OPTION, "integration_order must be in 1..8");
    if (p->n_baths == 0 || !p->baths) return fail(HX_ERR_UNSUPPORTED_BATH, "at least one bath is required");
    if (p->n_baths > static_cast<uint32_t>(hx::kMaxBaths)) return fail(HX_ERR_UNSUPPORTED_BATH, "too many baths");
    if (p->max_depth < 1) return fail(HX_ERR_UNSUPPORTED_HIERARCHY, "max_depth must be >= 1");
    if ((p->flags & ~(HX_FLAG_FULL_STATE | HX_FLAG_DENSE_H)) != 0)
        return fail(HX_ERR_INVALID_RUNTIME_OPTION, "unknown flags");

    const int J = static_cast<int>(p->n_baths);
    // dense H on the tensor cores: the band kernels see only the diagonal of
    // H, the rest is applied as matrix products before every stage
    const bool want_dense = (p->flags & HX_FLAG_DENSE_H) != 0;
    HostCsr dense_h;
    hx_problem dense_problem;
    std::vector<double> dense_diag, dense_zero;
    if (want_dense) {
        if (p->precision != HX_PRECISION_MIXED || !(p->flags & HX_FLAG_FULL_STATE))
            return fail(HX_ERR_UNSUPPORTED_EXECUTION, "HX_FLAG_DENSE_H needs HX_PRECISION_MIXED and HX_FLAG_FULL_STATE");
        std::string why;
        if (p->h_csr) {
            if (!take_csr(p->h_csr, static_cast<int>(d), dense_h, why, "h_csr"))
                return fail(HX_ERR_INVALID_RUNTIME_OPTION, why);
        } else {
            dense_h = flip_csr(p->h_diag, p->h_flip, static_cast<int>(d), logd);
        }
        // the real diagonal of H stays exact in the band kernels' diagonal table; the
        // products carry only the off-diagonal part (smaller terms, smaller rounding)
        dense_diag.assign(d, 0.0);
        for (uint32_t r = 0; r < d; ++r)
            for (int q = dense_h.ptr[r]; q < dense_h.ptr[r + 1]; ++q)
                if (dense_h.col[q] == static_cast<int32_t>(r)) dense_diag[r] += dense_h.val[q].x;
        dense_zero.assign(d, 0.0);
        dense_problem = *p;
        dense_problem.h_csr = nullptr;
        dense_problem.h_diag = dense_diag.data();
        dense_problem.h_flip = dense_zero.data();
        p = &dense_problem;
    }
    // general sparse operators: checked and gathered here, run on the CSR path
    // unless every operator is a diagonal plus single-spin flips (then the
    // problem is rewritten in that form and takes the faster paths)
    bool use_csr = p->h_csr != nullptr;
    for (int j = 0; j < J; ++j) use_csr = use_csr || p->baths[j].coupling_csr != nullptr;
    std::vector<HostCsr> ops;
    hx_problem lowered;
    std::vector<hx_bath> lowered_baths;
    std::vector<std::vector<double>> lowered_arrays;
    if (use_csr) {
        std::string why;
        ops.resize(J + 1);
        if (p->h_csr) {
            if (!take_csr(p->h_csr, static_cast<int>(d), ops[0], why, "h_csr"))
                return fail(HX_ERR_INVALID_RUNTIME_OPTION, why);
        } else {
            ops[0] = flip_csr(p->h_diag, p->h_flip, static_cast<int>(d), logd);
        }
        for (int j = 0; j < J; ++j) {
            const hx_bath& b = p->baths[j];
            if (b.coupling_csr) {
                if (!take_csr(b.coupling_csr, static_cast<int>(d), ops[1 + j], why,
                              "coupling_csr[" + std::to_string(j) + "]"))
                    return fail(HX_ERR_UNSUPPORTED_BATH, why);
            } else {
                if (!b.coupling_diag) return fail(HX_ERR_UNSUPPORTED_BATH, "bath coupling operator is NULL");
                ops[1 + j] = flip_csr(b.coupling_diag, b.coupling_flip, static_cast<int>(d), logd);
            }
        }
        lowered_arrays.resize(2 * (J + 1));
        bool all_flip = true;
        for (int k = 0; k <= J && all_flip; ++k)
            all_flip = split_flip(ops[k], static_cast<int>(d), logd, lowered_arrays[2 * k], lowered_arrays[2 * k + 1]);
        if (all_flip) {
            lowered = *p;
            lowered_baths.assign(p->baths, p->baths + J);
            lowered.h_csr = nullptr;
            lowered.h_diag = lowered_arrays[0].data();
            lowered.h_flip = lowered_arrays[1].data();
            for (int j = 0; j < J; ++j) {
                lowered_baths[j].coupling_csr = nullptr;
                lowered_baths[j].coupling_diag = lowered_arrays[2 * (j + 1)].data();
                lowered_baths[j].coupling_flip = lowered_arrays[2 * (j + 1) + 1].data();
            }
            lowered.baths = lowered_baths.data();
            p = &lowered;
            use_csr = false;
            ops.clear();
        } else if (p->precision != HX_PRECISION_DOUBLE) {
            return fail(HX_ERR_UNSUPPORTED_PRECISION, "sparse operators run in double precision");
        }
    }
    std::vector<hx::BathConst> bc(J);
    int M = 0;
    for (int j = 0; j < J; ++j) {
        const hx_bath& b = p->baths[j];
        if (!b.coupling_diag && !b.coupling_csr) return fail(HX_ERR_UNSUPPORTED_BATH, "bath coupling operator is NULL");
        if (!(b.inverse_temperature > 0.0) || !(b.damping > 0.0) || !std::isfinite(b.coupling_strength))
            return fail(HX_ERR_UNSUPPORTED_BATH, "bath needs positive beta and gamma and a finite coupling");
        if (b.pade_terms > 32) return fail(HX_ERR_UNSUPPORTED_BATH, "too many Pade terms");
        if (!hx::bath_constants(b.inverse_temperature, b.damping, b.coupling_strength,
                                static_cast<int>(b.pade_terms), bc[j]))
            return fail(HX_ERR_UNSUPPORTED_BATH, "bath coefficients are not finite (cot(beta gamma / 2) pole?)");
        bc[j].offset = M;
        M += static_cast<int>(b.pade_terms) + 1;
    }
    if (M > hx::kMaxModes) return fail(HX_ERR_UNSUPPORTED_HIERARCHY, "too many modes");
    uint64_t H = 0;
    int rc = hx_hierarchy_size(static_cast<uint32_t>(M), p->max_depth, &H);
    if (rc != HX_OK) return rc;
    if (H == 0 || H >= (1ull << 31)) return fail(HX_ERR_UNSUPPORTED_HIERARCHY, "hierarchy size out of range");

    hx_ctx* c = new (std::nothrow) hx_ctx();
    if (!c) return fail(HX_ERR_OUT_OF_MEMORY, "host allocation failed");
    cudaGetDevice(&c->device);
    c->d = static_cast<int>(d);
    c->logd = logd;
    c->M = M;
    c->J = J;
    c->H = static_cast<long long>(H);
    c->order = static_cast<int>(p->integration_order);
    c->dt = p->time_step;
    c->slab = static_cast<size_t>(d) * d;

    auto bail = [&](int code) {
        release(c);
        return code;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(hx::cuda_fail(e, "cudaStreamCreate"));
    c->stream = c->own_stream;

    // spin-flip parts in any coupling operator select the two-pass flip path
    std::vector<double> vf(static_cast<size_t>(J) * logd, 0.0);
    bool any_flip = false;
    for (int j = 0; j < J; ++j)
        if (p->baths[j].coupling_flip && !p->baths[j].coupling_csr)
            for (int i = 0; i < logd; ++i) {
                const double w = p->baths[j].coupling_flip[i];
                if (!std::isfinite(w)) return bail(fail(HX_ERR_UNSUPPORTED_BATH, "coupling flip weight is not finite"));
                vf[static_cast<size_t>(j) * logd + i] = w;
                any_flip = any_flip || w != 0.0;
            }
    c->use_csr = use_csr;
    c->use_large = !use_csr && !any_flip && logd >= 7 && hx::large_supported(logd, M, J);
    c->use_flip = !use_csr && (any_flip || (logd > hx::kMaxLogD && !c->use_large));
    c->mixed = p->precision == HX_PRECISION_MIXED;
    if (c->mixed && !c->use_large)
        return bail(fail(HX_ERR_UNSUPPORTED_PRECISION, "mixed precision needs diagonal coupling operators"));
    if (want_dense) {
        if (!c->use_large)
            return bail(fail(HX_ERR_UNSUPPORTED_EXECUTION,
                             "HX_FLAG_DENSE_H needs 128 <= d <= 1024 and diagonal coupling operators"));
        if (static_cast<long long>(H) * d > INT32_MAX)
            return bail(fail(HX_ERR_UNSUPPORTED_EXECUTION, "HX_FLAG_DENSE_H: H d exceeds the GEMM's row range"));
        if (!hx::tc_gemm_ready(true))
            return bail(fail(HX_ERR_UNSUPPORTED_EXECUTION, "HX_FLAG_DENSE_H: the tensor-core GEMM is unavailable"));
        for (const double2& v : dense_h.val)
            if (!std::isfinite(v.x) || !std::isfinite(v.y))
                return bail(fail(HX_ERR_INVALID_RUNTIME_OPTION, "H is not finite"));
        c->dense = true;
    }
    // fused stage kernels (d = 32, 64), on Hermitian-packed slabs unless the caller keeps full slabs
    const char* force_generic = std::getenv("HX_FORCE_GENERIC_STAGE");
    const bool want_herm = (p->flags & HX_FLAG_FULL_STATE) == 0;
    const bool fused_ok = !c->use_flip && !c->use_large && !c->use_csr && logd >= 5 && logd <= hx::kMaxLogD &&
                          hx::fused_supported(logd, M, J, want_herm ? 1 : 0) &&
                          !(force_generic && force_generic[0] == '1');
    // small slabs (d <= 16) with sigma_z couplings: batched-gather kernel (hx_small.cu)
    const char* small_env = std::getenv("HX_SMALL_STAGE");
    const bool small_ok = !c->use_flip && !c->use_large && !c->use_csr && logd <= 4 &&
                          hx::small_supported(logd, M, 1) && !(force_generic && force_generic[0] == '1') &&
                          !(small_env && small_env[0] == '0');
    c->herm = (fused_ok || c->use_large) && want_herm;
    c->slab_store = c->herm ? static_cast<size_t>(hx::herm_elems(logd)) : c->slab;
    const size_t nstate = static_cast<size_t>(H) * c->slab_store;
    if ((rc = dev_alloc(c, &c->vflip, vf.size())) || (rc = upload(c, c->vflip, vf))) return bail(rc);
    // two-pass paths: [V_j, u_n] and {V_j, u_n} for every bath and ADO
    if ((c->use_flip || c->use_csr) && (rc = dev_alloc(c, &c->Bbuf, 2 * nstate * J))) return bail(rc);
    if (c->use_csr) {
        std::vector<int32_t> ptr, col;
        std::vector<double2> val;
        for (const HostCsr& o : ops) {
            const int32_t base = static_cast<int32_t>(col.size());
            for (int32_t x : o.ptr) ptr.push_back(base + x);
            col.insert(col.end(), o.col.begin(), o.col.end());
            val.insert(val.end(), o.val.begin(), o.val.end());
        }
        if ((rc = dev_alloc(c, &c->csr_ptr, ptr.size())) || (rc = dev_alloc(c, &c->csr_col, col.size())) ||
            (rc = dev_alloc(c, &c->csr_val, val.size())) || (rc = upload(c, c->csr_ptr, ptr)) ||
            (rc = upload(c, c->csr_col, col)) || (rc = upload(c, c->csr_val, val)))
            return bail(rc);
    }
    // double-precision state: the whole hierarchy, or only ADO 0 in mixed precision
    const size_t n64 = c->mixed ? c->slab_store : nstate;
    if (c->mixed && ((rc = dev_alloc(c, &c->rho32, nstate)) || (rc = dev_alloc(c, &c->ua32, nstate)) ||
                     (rc = dev_alloc(c, &c->ub32, nstate))))
        return bail(rc);
    if ((rc = dev_alloc(c, &c->rho, n64)) || (rc = dev_alloc(c, &c->ua, n64)) ||
        (rc = dev_alloc(c, &c->ub, n64)) || (rc = dev_alloc(c, &c->rows, H * M)) ||
        (rc = dev_alloc(c, &c->edges, H * 2 * M)) || (rc = dev_alloc(c, &c->acoef, H * M)) ||
        (rc = dev_alloc(c, &c->bcoef, H * J)) || (rc = dev_alloc(c, &c->gsum, H)) ||
        (rc = dev_alloc(c, &c->hdiag, d)) || (rc = dev_alloc(c, &c->hflip, logd)) ||
        (rc = dev_alloc(c, &c->vdiag, static_cast<size_t>(J) * d)) || (rc = dev_alloc(c, &c->xi, J)) ||
        (rc = dev_alloc(c, &c->counter, J)) || (rc = dev_alloc(c, &c->bath_off, J + 1)) ||
        (rc = dev_alloc(c, &c->error_flag, 1)) || (rc = dev_alloc(c, &c->obs, 4)))
        return bail(rc);

    // host-side operator data (with sparse operators: the real parts of their diagonals)
    auto diag_of = [&](const HostCsr& o, double* outd) {
        for (uint32_t r = 0; r < d; ++r) {
            outd[r] = 0.0;
            for (int q = o.ptr[r]; q < o.ptr[r + 1]; ++q)
                if (o.col[q] == static_cast<int32_t>(r)) outd[r] += o.val[q].x;
        }
    };
    c->h_hdiag.assign(d, 0.0);
    if (p->h_csr) diag_of(ops[0], c->h_hdiag.data());
    else c->h_hdiag.assign(p->h_diag, p->h_diag + d);
    c->h_hflip.assign(logd, 0.0);
    if (p->h_flip && !p->h_csr) c->h_hflip.assign(p->h_flip, p->h_flip + logd);
    std::vector<double> vd(static_cast<size_t>(J) * d), xi(J), ct(J), nu_m(M), phi_m(M, 0.0), tc(J), ta(J);
    std::vector<int32_t> off(J + 1), mb(M), mk(M);
    for (int j = 0; j < J; ++j) {
        if (p->baths[j].coupling_csr) diag_of(ops[1 + j], vd.data() + static_cast<size_t>(j) * d);
        else std::copy(p->baths[j].coupling_diag, p->baths[j].coupling_diag + d, vd.begin() + static_cast<size_t>(j) * d);
        xi[j] = bc[j].xi;
        ct[j] = bc[j].counter;
        tc[j] = bc[j].theta_c;
        ta[j] = bc[j].theta_a;
        off[j] = bc[j].offset;
        for (int k = 0; k <= bc[j].K; ++k) {
            const int m = bc[j].offset + k;
            mb[m] = j;
            mk[m] = k;
            nu_m[m] = bc[j].nu[k];
            if (k >= 1) phi_m[m] = bc[j].phi[k - 1];
        }
    }
    off[J] = M;
    for (double v : vd)
        if (!std::isfinite(v)) return bail(fail(HX_ERR_UNSUPPORTED_BATH, "coupling operator is not finite"));
    for (double v : c->h_hdiag)
        if (!std::isfinite(v)) return bail(fail(HX_ERR_INVALID_RUNTIME_OPTION, "h_diag is not finite"));

    if ((rc = upload(c, c->hdiag, c->h_hdiag)) || (rc = upload(c, c->hflip, c->h_hflip)) ||
        (rc = upload(c, c->vdiag, vd)) || (rc = upload(c, c->xi, xi)) || (rc = upload(c, c->counter, ct)) ||
        (rc = upload(c, c->bath_off, off)))
        return bail(rc);
    if (c->dense) {
        // the real form of H without its diagonal (TF32 split) for Y = X H, stage scratch,
        // and the whole H in CSR for the energy
        const size_t D = d, W = 2 * D;
        std::vector<double> hre(D * D, 0.0), him(D * D, 0.0);
        for (size_t r = 0; r < D; ++r)
            for (int q = dense_h.ptr[r]; q < dense_h.ptr[r + 1]; ++q)
                if (dense_h.col[q] != static_cast<int32_t>(r)) {
                    hre[r * D + dense_h.col[q]] += dense_h.val[q].x;
                    him[r * D + dense_h.col[q]] += dense_h.val[q].y;
                }
        std::vector<double2> h64(D * D);
        for (size_t i = 0; i < D * D; ++i) h64[i] = make_double2(hre[i], him[i]);
        std::vector<float> hi(W * W), lo(W * W);
        auto put = [&](size_t row, size_t k, double v) {
            const float h = tf32_round_host(static_cast<float>(v));
            hi[row * W + k] = h;
            lo[row * W + k] = tf32_round_host(static_cast<float>(v - static_cast<double>(h)));
        };
        for (size_t cc = 0; cc < D; ++cc)
            for (size_t k = 0; k < D; ++k) {
                const double re = hre[k * D + cc], im = him[k * D + cc];
                put(2 * cc, 2 * k, re);
                put(2 * cc, 2 * k + 1, -im);
                put(2 * cc + 1, 2 * k, im);
                put(2 * cc + 1, 2 * k + 1, re);
            }
        if ((rc = dev_alloc(c, &c->dense_h64, h64.size())) || (rc = upload(c, c->dense_h64, h64)) ||
            (rc = dev_alloc(c, &c->dense_z0, h64.size())) ||
            (rc = dev_alloc(c, &c->dense_hr, hi.size())) || (rc = dev_alloc(c, &c->dense_hr_lo, lo.size())) ||
            (rc = upload(c, c->dense_hr, hi)) || (rc = upload(c, c->dense_hr_lo, lo)) ||
            (rc = dev_alloc(c, &c->dense_y, nstate)) || (rc = dev_alloc(c, &c->csr_ptr, dense_h.ptr.size())) ||
            (rc = dev_alloc(c, &c->csr_col, std::max<size_t>(1, dense_h.col.size()))) ||
            (rc = dev_alloc(c, &c->csr_val, std::max<size_t>(1, dense_h.val.size()))) ||
            (rc = upload(c, c->csr_ptr, dense_h.ptr)))
            return bail(rc);
        if (!dense_h.col.empty() && ((rc = upload(c, c->csr_col, dense_h.col)) || (rc = upload(c, c->csr_val, dense_h.val))))
            return bail(rc);
    }

    // per-mode temporaries for the coefficient kernel
    int32_t *dmb = nullptr, *dmk = nullptr;
    double *dnu = nullptr, *dphi = nullptr, *dtc = nullptr, *dta = nullptr;
    e = cudaMalloc(&dmb, M * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&dmk, M * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&dnu, M * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&dphi, M * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&dtc, J * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&dta, J * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpyAsync(dmb, mb.data(), M * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dmk, mk.data(), M * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dnu, nu_m.data(), M * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dphi, phi_m.data(), M * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dtc, tc.data(), J * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dta, ta.data(), J * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->error_flag, 0, sizeof(int), c->stream);
    if (e != cudaSuccess) rc = hx::cuda_fail(e, "context setup");
    if (rc == HX_OK) rc = hx::build_tables_device(M, static_cast<int>(p->max_depth), c->H, c->rows, c->edges, c->stream);
    if (rc == HX_OK) {
        hx::launch_coefficients(c->rows, c->H, M, J, dmb, dmk, dnu, dtc, dta, dphi, c->bath_off, c->acoef,
                                c->bcoef, c->gsum, c->stream);
        const long long one = c->herm ? hx::herm_index(c->d - 1, c->d - 1, logd) : static_cast<long long>(c->slab) - 1;
        hx::launch_init_state(c->rho, static_cast<long long>(n64), one, c->stream);
        if (c->mixed) {
            e = cudaMemsetAsync(c->rho32, 0, nstate * sizeof(float2), c->stream);
            if (e == cudaSuccess) hx::launch_d2f(c->rho, c->rho32, static_cast<long long>(c->slab_store), c->stream);
            if (e != cudaSuccess) rc = hx::cuda_fail(e, "mixed initial state");
        }
        rc = check_launch("setup kernels");
    }
    // fused stage kernel (d = 32, 64): neighbour entry lists, diagonal table, up-term tables
    if (rc == HX_OK && (fused_ok || c->use_large || small_ok)) {
        cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, c->device);
        int* dS = nullptr;
        if ((rc = dev_alloc(c, &c->diag_table, c->slab)) || (rc = dev_alloc(c, &c->ent_count, H)) ||
            (rc = dev_alloc(c, &c->ent_slab, H * 2 * M)) || (rc = dev_alloc(c, &c->ent_bath, H * 2 * M)) ||
            (rc = dev_alloc(c, &c->ent_wc, H * 2 * M)) || (rc = dev_alloc(c, &c->ent_wa, H * 2 * M)) ||
            (rc = dev_alloc(c, &c->ado_keep, H)) || (rc = dev_alloc(c, &c->up_slot, H)) ||
            (rc = dev_alloc(c, &c->up_ado, H)) || (rc = dev_alloc(c, &c->up_cnt, H)) || (rc = dev_alloc(c, &dS, 1))) {
        } else {
            hx::launch_diag_table(c->hdiag, c->vdiag, c->xi, c->counter, c->d, J, c->diag_table, c->stream);
            if (c->herm && (rc = dev_alloc(c, &c->diag_herm, c->slab_store)) == HX_OK)
                hx::launch_pack_herm(c->diag_table, logd, c->diag_herm, c->stream);
            // sigma_z couplings: the fused kernels take v_r from bit r of the spin, not from a table
            std::vector<int> bits(J);
            bool all_pauli = true;
            for (int j = 0; j < J; ++j) all_pauli = all_pauli && (bits[j] = hx::pauli_spin(vd.data() + static_cast<size_t>(j) * d, c->d)) >= 0;
            if (rc == HX_OK && all_pauli && (rc = dev_alloc(c, &c->vbit, J)) == HX_OK) rc = upload(c, c->vbit, bits);
            // small slabs: every up neighbour in the entry lists (no up-term pass)
            const bool want_small = small_ok && all_pauli;
            hx::launch_entries(c->rows, c->edges, c->acoef, c->bcoef, c->bath_off, c->H, M, J,
                               static_cast<int>(p->max_depth) + (want_small ? 1 : 0), c->ent_count,
                               c->ent_slab,
                               c->ent_bath, c->ent_wc, c->ent_wa, c->ado_keep, c->stream);
            rc = check_launch("fused-kernel setup");
            // tier L-1 slots: count them first, then size the per-slot tables and U
            int S = 0;
            if (rc == HX_OK && p->max_depth >= 2 && !small_ok) {
                int32_t *tmp_slab = nullptr, *tmp_bath = nullptr;
                e = cudaMalloc(&tmp_slab, H * M * sizeof(int32_t));
                if (e == cudaSuccess) e = cudaMalloc(&tmp_bath, H * M * sizeof(int32_t));
                if (e == cudaSuccess) {
                    hx::launch_upterm_tables(c->rows, c->edges, dmb, c->H, M, static_cast<int>(p->max_depth) - 1,
                                             c->up_slot, dS, c->up_ado, c->up_cnt, tmp_slab, tmp_bath, c->stream);
                    e = cudaMemcpyAsync(&S, dS, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
                }
                if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
                if (e == cudaSuccess && S > 0) {
                    rc = dev_alloc(c, &c->up_slab, static_cast<size_t>(S) * M);
                    if (rc == HX_OK) rc = dev_alloc(c, &c->up_bath, static_cast<size_t>(S) * M);
                    if (rc == HX_OK) {
                        if (c->mixed) rc = dev_alloc(c, &c->U32, static_cast<size_t>(S) * c->slab_store);
                        else rc = dev_alloc(c, &c->U, static_cast<size_t>(S) * c->slab_store);
                    }
                    if (rc == HX_OK) {
                        e = cudaMemcpyAsync(c->up_slab, tmp_slab, static_cast<size_t>(S) * M * sizeof(int32_t),
                                            cudaMemcpyDeviceToDevice, c->stream);
                        if (e == cudaSuccess)
                            e = cudaMemcpyAsync(c->up_bath, tmp_bath, static_cast<size_t>(S) * M * sizeof(int32_t),
                                                cudaMemcpyDeviceToDevice, c->stream);
                        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
                    }
                }
                if (e != cudaSuccess && rc == HX_OK) rc = hx::cuda_fail(e, "up-term tables");
                cudaFree(tmp_slab);
                cudaFree(tmp_bath);
            } else if (rc == HX_OK) {
                e = cudaMemsetAsync(c->up_slot, 0xff, H * sizeof(int32_t), c->stream);
                if (e != cudaSuccess) rc = hx::cuda_fail(e, "up-term tables");
            }
            c->up_slots = S;
            c->use_fused = (rc == HX_OK) && fused_ok;
            c->use_small = (rc == HX_OK) && want_small;
            // small slabs: the whole step in one cooperative launch when every ADO fits the resident CTAs
            const char* step_env = std::getenv("HX_SMALL_STEP");
            if (c->use_small && c->order >= 2 && !(step_env && step_env[0] == '0') &&
                (rc = dev_alloc(c, &c->gbar, 1)) == HX_OK) {
                e = cudaMemsetAsync(c->gbar, 0, sizeof(unsigned), c->stream);
                if (e != cudaSuccess) rc = hx::cuda_fail(e, "grid barrier counter");
                else
                    c->use_small_step = hx::launch_small_step(hx::fused_args_of(c), c->rho, c->ua, c->ub, c->dt,
                                                              c->order, c->gbar, c->stream, true) == 1;
            }
            // single-precision copies of the operators for the mixed band kernel
            if (rc == HX_OK && c->mixed) {
                if ((rc = dev_alloc(c, &c->diag32, c->slab)) || (rc = dev_alloc(c, &c->vdiag32, static_cast<size_t>(J) * d)) ||
                    (rc = dev_alloc(c, &c->hflip32, logd))) {
                } else {
                    hx::launch_d2f(c->herm ? c->diag_herm : c->diag_table, c->diag32,
                                   static_cast<long long>(c->slab_store), c->stream);
                    hx::launch_vec_d2f(c->vdiag, c->vdiag32, static_cast<long long>(J) * d, c->stream);
                    hx::launch_vec_d2f(c->hflip, c->hflip32, logd, c->stream);
                    rc = check_launch("mixed-precision operators");
                }
            }
        }
        cudaFree(dS);
        if (dS) c->device_bytes -= sizeof(int);
    }
    cudaFree(dmb);
    cudaFree(dmk);
    cudaFree(dnu);
    cudaFree(dphi);
    cudaFree(dtc);
    cudaFree(dta);
    if (rc == HX_OK && c->use_large && (c->diag_table == nullptr || c->ent_count == nullptr))
        rc = fail(HX_ERR_UNSUPPORTED_EXECUTION, "band-kernel tables were not built");
    if (rc == HX_OK && c->use_large) {
        const bool ok = c->mixed ? hx::prepare_large<float>(large_args32(c)) : hx::prepare_large<double>(large_args64(c));
        if (!ok) rc = fail(HX_ERR_UNSUPPORTED_EXECUTION, "band kernel does not fit in shared memory");
    }
    if (rc == HX_OK) {
        e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) rc = hx::cuda_fail(e, "context set-up");
    }
    if (rc != HX_OK) return bail(rc);
    c->counters.kernel_launches += 3;
    *out = c;
    return HX_OK;
}

void hx_ctx_destroy(hx_ctx* ctx) { release(ctx); }

int hx_ctx_set_stream(hx_ctx* c, void* stream)
{
    if (!c) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL context");
    HX_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->stream = stream ? static_cast<cudaStream_t>(stream) : c->own_stream;
    return HX_OK;
}

int hx_ctx_get_stream(hx_ctx* c, void** stream)
{
    if (!c || !stream) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL argument");
    *stream = c->stream;
    return HX_OK;
}

int hx_ctx_info(const hx_ctx* c, hx_info* info)
{
    if (!c || !info) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL argument");
    info->dim = static_cast<uint32_t>(c->d);
    info->modes = static_cast<uint32_t>(c->M);
    info->hierarchy_size = static_cast<uint64_t>(c->H);
    info->state_bytes = static_cast<uint64_t>(c->H) * c->slab_store * sizeof(double2);
    info->device_bytes = c->device_bytes;
    info->steps_done = c->steps_done;
    info->time = static_cast<double>(c->steps_done) * c->dt;
    int per_stage = (c->use_flip || c->use_csr || (c->use_fused && c->up_slots > 0)) ? 2 : 1;
    if (c->use_large) per_stage = 1 + (c->up_slots > 0 ? 1 : 0) + (c->mixed ? 1 : 0) + (c->dense ? 2 : 0);
    info->kernels_per_step = static_cast<uint32_t>(c->order) * per_stage;
    if (c->use_small_step && !c->closure) info->kernels_per_step = 1;
    info->stage_path = c->dense     ? HX_PATH_DENSE
                       : c->use_csr ? HX_PATH_CSR
                       : c->use_flip ? HX_PATH_FLIP
                       : c->use_large ? HX_PATH_BAND
                       : c->use_fused ? HX_PATH_FUSED
                       : c->use_small ? HX_PATH_SMALL
                       : HX_PATH_GENERIC;
    return HX_OK;
}

int hx_ctx_counters(const hx_ctx* c, hx_counters* out)
{
    if (!c || !out) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL argument");
    *out = c->counters;
    return HX_OK;
}

int hx_ctx_step(hx_ctx* c, uint64_t nsteps)
{
    if (!c) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL context");
    for (uint64_t s = 0; s < nsteps; ++s) enqueue_step(c);
    return check_launch("stage kernel launch");
}

int hx_ctx_sync(hx_ctx* c)
{
    if (!c) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL context");
    HX_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return read_error_flag(c);
}

int hx_ctx_step_trace(hx_ctx* c, uint64_t nsteps, double* rho0_trace, double* energy_trace)
{
    if (!c) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL context");
    // chunk of steps buffered on the device: at most 256 steps and 64 MB of rho_0 copies
    const uint64_t by_bytes = std::max<uint64_t>(1, (uint64_t(64) << 20) / (c->slab * sizeof(double2)));
    const int cap = static_cast<int>(std::min<uint64_t>(std::min<uint64_t>(std::max<uint64_t>(nsteps, 1), 256), by_bytes));
    if (c->trace_cap < cap) {
        if (c->trace_buf) cudaFree(c->trace_buf);
        if (c->energy_buf) cudaFree(c->energy_buf);
        if (c->pinned) cudaFreeHost(c->pinned);
        c->trace_buf = nullptr;
        c->energy_buf = nullptr;
        c->pinned = nullptr;
        c->trace_cap = 0;
        HX_CUDA_TRY(cudaMalloc(&c->trace_buf, cap * c->slab * sizeof(double2)));
        HX_CUDA_TRY(cudaMalloc(&c->energy_buf, cap * 3 * sizeof(double)));
        c->pinned_bytes = cap * (c->slab * sizeof(double2) + 3 * sizeof(double));
        HX_CUDA_TRY(cudaMallocHost(&c->pinned, c->pinned_bytes));
        c->trace_cap = cap;
    }
    double* pin_rho = c->pinned;
    double* pin_en = c->pinned + static_cast<size_t>(c->trace_cap) * c->slab * 2;
    uint64_t done = 0;
    while (done < nsteps) {
        const int chunk = static_cast<int>(std::min<uint64_t>(nsteps - done, c->trace_cap));
        for (int t = 0; t < chunk; ++t) {
            enqueue_step(c);
            launch_obs(c, c->energy_buf + 3 * t);
            c->counters.kernel_launches += 1;
            if (rho0_trace)
                HX_CUDA_TRY(cudaMemcpyAsync(c->trace_buf + static_cast<size_t>(t) * c->slab_store, c->rho,
                                            c->slab_store * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream));
        }
        int rc = check_launch("trace step");
        if (rc != HX_OK) return rc;
        if (rho0_trace) {
            HX_CUDA_TRY(cudaMemcpyAsync(pin_rho, c->trace_buf, chunk * c->slab_store * sizeof(double2),
                                        cudaMemcpyDeviceToHost, c->stream));
            c->counters.d2h_bytes += chunk * c->slab_store * sizeof(double2);
        }
        if (energy_trace) {
            HX_CUDA_TRY(cudaMemcpyAsync(pin_en, c->energy_buf, chunk * 3 * sizeof(double), cudaMemcpyDeviceToHost,
                                        c->stream));
            c->counters.d2h_bytes += chunk * 3 * sizeof(double);
        }
        HX_CUDA_TRY(cudaStreamSynchronize(c->stream));
        if (rho0_trace && c->herm) {
            for (int t = 0; t < chunk; ++t)
                hx::unpack_herm_host(reinterpret_cast<const double2*>(pin_rho) + static_cast<size_t>(t) * c->slab_store,
                                     c->logd, rho0_trace + (done + t) * c->slab * 2);
        } else if (rho0_trace) {
            std::memcpy(rho0_trace + done * c->slab * 2, pin_rho, chunk * c->slab * sizeof(double2));
        }
        if (energy_trace)
            for (int t = 0; t < chunk; ++t) energy_trace[done + t] = pin_en[3 * t];
        done += chunk;
    }
    return read_error_flag(c);
}

int hx_ctx_read_rho0(hx_ctx* c, double* out, uint64_t n)
{
    if (!c || !out) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL argument");
    if (n < 2 * c->slab) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "output buffer too small");
    if (c->herm) {
        const int rc = read_herm(c, c->rho, 1, out);
        return rc != HX_OK ? rc : read_error_flag(c);
    }
    HX_CUDA_TRY(cudaMemcpyAsync(out, c->rho, c->slab * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
    HX_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->counters.d2h_bytes += c->slab * sizeof(double2);
    return read_error_flag(c);
}

int hx_ctx_observables(hx_ctx* c, double* energy, double* trace_re, double* trace_im)
{
    if (!c) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL context");
    launch_obs(c, c->obs);
    c->counters.kernel_launches += 1;
    int rc = check_launch("observables kernel");
    if (rc != HX_OK) return rc;
    double h[3];
    HX_CUDA_TRY(cudaMemcpyAsync(h, c->obs, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    HX_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (energy) *energy = h[0];
    if (trace_re) *trace_re = h[1];
    if (trace_im) *trace_im = h[2];
    return read_error_flag(c);
}

int hx_ctx_read_state(hx_ctx* c, double* out, uint64_t n)
{
    if (!c || !out) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL argument");
    const size_t count = static_cast<size_t>(c->H) * c->slab;
    if (n < 2 * count) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "output buffer too small");
    if (c->mixed) {
        const int rc = read_mixed(c, c->rho32, c->rho, out);
        return rc != HX_OK ? rc : read_error_flag(c);
    }
    if (c->herm) {
        const int rc = read_herm(c, c->rho, static_cast<size_t>(c->H), out);
        return rc != HX_OK ? rc : read_error_flag(c);
    }
    HX_CUDA_TRY(cudaMemcpyAsync(out, c->rho, count * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
    HX_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->counters.d2h_bytes += count * sizeof(double2);
    return read_error_flag(c);
}

namespace {

constexpr int kNoStaging = -1;

// Mixed precision: upload the FP64 state into a temporary device buffer, check
// Hermiticity there when the context needs it (packed slabs, or a dense H),
// and convert (and pack) on the device.  kNoStaging when the temporary buffer
// cannot be had; the caller then converts on the host.
int write_state_mixed_device(hx_ctx* c, const double* in)
{
    const size_t count = static_cast<size_t>(c->H) * c->slab;
    double2* stage = nullptr;
    if (cudaMalloc(&stage, count * sizeof(double2)) != cudaSuccess) {
        cudaGetLastError();  // clear the allocation failure
        return kNoStaging;
    }
    auto done = [&](int rc) {
        cudaStreamSynchronize(c->stream);
        cudaFree(stage);
        return rc;
    };
    cudaError_t e = cudaMemcpyAsync(stage, in, count * sizeof(double2), cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return done(hx::cuda_fail(e, "state upload"));
    c->counters.h2d_bytes += count * sizeof(double2);
    if (c->herm || c->dense) {
        int rc = HX_OK;
        if (!c->pack_scale && ((rc = dev_alloc(c, &c->pack_scale, c->H)) || (rc = dev_alloc(c, &c->pack_bad, 1))))
            return done(rc);
        e = cudaMemsetAsync(c->pack_bad, 0x7f, sizeof(int), c->stream);
        if (e != cudaSuccess) return done(hx::cuda_fail(e, "state check"));
        hx::launch_herm_check(stage, c->H, c->logd, 1e-12, c->pack_scale, 0, c->pack_bad, c->stream);
        int bad = 0;
        e = cudaMemcpyAsync(&bad, c->pack_bad, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) return done(hx::cuda_fail(e, "state check"));
        if (bad != 0x7f7f7f7f)
            return done(fail(HX_ERR_INVALID_RUNTIME_OPTION,
                             "ADO " + std::to_string(bad) +
                                 (c->dense ? " is not Hermitian, which HX_FLAG_DENSE_H requires"
                                           : " is not Hermitian; this context keeps Hermitian-packed slabs (create it "
                                             "with HX_FLAG_FULL_STATE for general states)")));
    }
    if (c->herm) {
        hx::launch_herm_pack_f32(stage, c->H, c->logd, 0, c->rho32, c->stream);
        hx::launch_herm_pack(stage, 1, c->logd, 0, c->rho, c->stream);
    } else {
        hx::launch_d2f(stage, c->rho32, static_cast<long long>(count), c->stream);
        e = cudaMemcpyAsync(c->rho, stage, c->slab * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream);
        if (e != cudaSuccess) return done(hx::cuda_fail(e, "state upload"));
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return done(hx::cuda_fail(e, "state conversion"));
    return done(HX_OK);
}

}  // namespace

int hx_ctx_write_state(hx_ctx* c, const double* in, uint64_t n)
{
    if (!c || !in) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL argument");
    const size_t count = static_cast<size_t>(c->H) * c->slab;
    if (n < 2 * count) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "input buffer too small");
    if (c->mixed) {
        const int rc = write_state_mixed_device(c, in);
        if (rc != kNoStaging) return rc;
    }
    if (c->mixed && c->herm) {
        const size_t P = c->slab_store;
        std::vector<double2> pk(static_cast<size_t>(c->H) * P);
        std::vector<char> ok(static_cast<size_t>(c->H), 1);
        parallel_for(c->H, [&](long long k) {
            ok[k] = pack_herm_host(in + 2 * static_cast<size_t>(k) * c->slab, c->logd, pk.data() + k * P);
        });
        for (long long k = 0; k < c->H; ++k)
            if (!ok[k])
                return fail(HX_ERR_INVALID_RUNTIME_OPTION,
                            "ADO " + std::to_string(k) +
                                " is not Hermitian; this context keeps Hermitian-packed slabs (create it with "
                                "HX_FLAG_FULL_STATE for general states)");
        std::vector<float2> tmp(pk.size());
        for (size_t i = 0; i < pk.size(); ++i)
            tmp[i] = make_float2(static_cast<float>(pk[i].x), static_cast<float>(pk[i].y));
        HX_CUDA_TRY(cudaMemcpyAsync(c->rho32, tmp.data(), tmp.size() * sizeof(float2), cudaMemcpyHostToDevice, c->stream));
        HX_CUDA_TRY(cudaMemcpyAsync(c->rho, pk.data(), P * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
        c->counters.h2d_bytes += tmp.size() * sizeof(float2) + P * sizeof(double2);
        HX_CUDA_TRY(cudaStreamSynchronize(c->stream));
        return HX_OK;
    }
    if (c->dense) {
        // the tensor-core product takes H X_n as (X_n H)^dagger, which needs Hermitian ADOs
        std::vector<char> ok(static_cast<size_t>(c->H), 1);
        parallel_for(c->H, [&](long long k) {
            const double* x = in + 2 * static_cast<size_t>(k) * c->slab;
            double scale2 = 0.0, worst2 = 0.0;
            for (int r = 0; r < c->d; ++r)
                for (int cc = 0; cc < c->d; ++cc) {
                    const size_t up = static_cast<size_t>(r) * c->d + cc, lo = static_cast<size_t>(cc) * c->d + r;
                    scale2 = std::max(scale2, x[2 * up] * x[2 * up] + x[2 * up + 1] * x[2 * up + 1]);
                    const double dr = x[2 * up] - x[2 * lo], di = x[2 * up + 1] + x[2 * lo + 1];
                    worst2 = std::max(worst2, dr * dr + di * di);
                }
            ok[k] = !(worst2 > 1e-24 * scale2);
        });
        for (long long k = 0; k < c->H; ++k)
            if (!ok[k])
                return fail(HX_ERR_INVALID_RUNTIME_OPTION,
                            "ADO " + std::to_string(k) + " is not Hermitian, which HX_FLAG_DENSE_H requires");
    }
    if (c->mixed) {
        std::vector<float2> tmp(count);
        for (size_t i = 0; i < count; ++i)
            tmp[i] = make_float2(static_cast<float>(in[2 * i]), static_cast<float>(in[2 * i + 1]));
        HX_CUDA_TRY(cudaMemcpyAsync(c->rho32, tmp.data(), count * sizeof(float2), cudaMemcpyHostToDevice, c->stream));
        HX_CUDA_TRY(cudaMemcpyAsync(c->rho, in, c->slab * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
        c->counters.h2d_bytes += count * sizeof(float2) + c->slab * sizeof(double2);
        HX_CUDA_TRY(cudaStreamSynchronize(c->stream));
        return HX_OK;
    }
    // full slabs that fit in the two stage buffers (scratch between steps)
    const long long per_buf =
        c->herm ? static_cast<long long>(static_cast<size_t>(c->H) * c->slab_store / c->slab) : 0;
    if (c->herm && 2 * per_buf < c->H) {
        // a tiny hierarchy: pack on the host
        const size_t n = static_cast<size_t>(c->H) * c->slab_store;
        int rc = state_staging(c, n);
        if (rc != HX_OK) return rc;
        HX_CUDA_TRY(cudaStreamSynchronize(c->stream));  // the staging buffer may still feed an earlier copy
        double2* pk = c->state_pinned;
        for (long long k = 0; k < c->H; ++k)
            if (!pack_herm_host(in + 2 * static_cast<size_t>(k) * c->slab, c->logd, pk + k * c->slab_store))
                return fail(HX_ERR_INVALID_RUNTIME_OPTION,
                            "ADO " + std::to_string(k) +
                                " is not Hermitian; this context keeps Hermitian-packed slabs (create it with "
                                "HX_FLAG_FULL_STATE for general states)");
        HX_CUDA_TRY(cudaMemcpyAsync(c->rho, pk, n * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
        c->counters.h2d_bytes += n * sizeof(double2);
        HX_CUDA_TRY(cudaStreamSynchronize(c->stream));
        return HX_OK;
    }
    if (c->herm) {
        // the full slabs go up into the two stage buffers, are checked for
        // Hermiticity on the device and only then packed into rho, so a
        // rejected state leaves the context's state as it was
        int rc = HX_OK;
        if (!c->pack_scale && ((rc = dev_alloc(c, &c->pack_scale, c->H)) || (rc = dev_alloc(c, &c->pack_bad, 1))))
            return rc;
        const long long n0 = std::min<long long>(per_buf, c->H), n1 = c->H - n0;
        const long long part_first[2] = {0, n0}, part_cnt[2] = {n0, n1};
        double2* bufs[2] = {c->ua, c->ub};
        HX_CUDA_TRY(cudaMemsetAsync(c->pack_bad, 0x7f, sizeof(int), c->stream));
        for (int b = 0; b < 2; ++b) {
            if (part_cnt[b] == 0) continue;
            HX_CUDA_TRY(cudaMemcpyAsync(bufs[b], in + 2 * static_cast<size_t>(part_first[b]) * c->slab,
                                        static_cast<size_t>(part_cnt[b]) * c->slab * sizeof(double2),
                                        cudaMemcpyHostToDevice, c->stream));
            hx::launch_herm_check(bufs[b], part_cnt[b], c->logd, 1e-12, c->pack_scale, part_first[b], c->pack_bad,
                                  c->stream);
            c->counters.h2d_bytes += static_cast<size_t>(part_cnt[b]) * c->slab * sizeof(double2);
        }
        HX_CUDA_TRY(cudaGetLastError());
        int bad = 0;
        HX_CUDA_TRY(cudaMemcpyAsync(&bad, c->pack_bad, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        HX_CUDA_TRY(cudaStreamSynchronize(c->stream));
        if (bad != 0x7f7f7f7f)
            return fail(HX_ERR_INVALID_RUNTIME_OPTION,
                        "ADO " + std::to_string(bad) +
                            " is not Hermitian; this context keeps Hermitian-packed slabs (create it with "
                            "HX_FLAG_FULL_STATE for general states)");
        for (int b = 0; b < 2; ++b) hx::launch_herm_pack(bufs[b], part_cnt[b], c->logd, part_first[b], c->rho, c->stream);
        HX_CUDA_TRY(cudaGetLastError());
        HX_CUDA_TRY(cudaStreamSynchronize(c->stream));
        return HX_OK;
    }
    HX_CUDA_TRY(cudaMemcpyAsync(c->rho, in, count * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
    c->counters.h2d_bytes += count * sizeof(double2);
    HX_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return HX_OK;
}

int hx_ctx_save_snapshot(hx_ctx* c, const char* path, uint32_t real_bytes)
{
    if (!c || !path) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL argument");
    if (real_bytes != 4 && real_bytes != 8) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "real_bytes must be 4 or 8");
    const size_t count = static_cast<size_t>(c->H) * c->slab;
    std::vector<double> all(2 * count);
    int rc = hx_ctx_read_state(c, all.data(), all.size());
    if (rc != HX_OK) return rc;
    std::FILE* f = std::fopen(path, "wb");
    if (!f) return fail(HX_ERR_INVALID_RUNTIME_OPTION, std::string("cannot open ") + path + " for writing");
    size_t wrote = 0;
    if (real_bytes == 8) {
        wrote = std::fwrite(all.data(), sizeof(double), all.size(), f);
    } else {
        std::vector<float> narrow(all.size());
        for (size_t i = 0; i < all.size(); ++i) narrow[i] = static_cast<float>(all[i]);
        wrote = std::fwrite(narrow.data(), sizeof(float), narrow.size(), f);
    }
    const bool closed = std::fclose(f) == 0;
    if (wrote != all.size() || !closed) return fail(HX_ERR_INVALID_RUNTIME_OPTION, std::string("short write to ") + path);
    return HX_OK;
}

int hx_ctx_load_snapshot(hx_ctx* c, const char* path, uint32_t real_bytes)
{
    if (!c || !path) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL argument");
    if (real_bytes != 4 && real_bytes != 8) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "real_bytes must be 4 or 8");
    const size_t count = static_cast<size_t>(c->H) * c->slab;
    std::FILE* f = std::fopen(path, "rb");
    if (!f) return fail(HX_ERR_INVALID_RUNTIME_OPTION, std::string("cannot open ") + path);
    std::fseek(f, 0, SEEK_END);
    const long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (size < 0 || static_cast<size_t>(size) != 2 * count * real_bytes) {
        std::fclose(f);
        return fail(HX_ERR_INVALID_RUNTIME_OPTION,
                    std::string(path) + " holds " + std::to_string(size) + " bytes; this hierarchy needs " +
                        std::to_string(2 * count * real_bytes));
    }
    std::vector<double> all(2 * count);
    size_t got = 0;
    if (real_bytes == 8) {
        got = std::fread(all.data(), sizeof(double), all.size(), f);
    } else {
        std::vector<float> narrow(all.size());
        got = std::fread(narrow.data(), sizeof(float), narrow.size(), f);
        for (size_t i = 0; i < all.size(); ++i) all[i] = narrow[i];
    }
    std::fclose(f);
    if (got != all.size()) return fail(HX_ERR_INVALID_RUNTIME_OPTION, std::string("short read from ") + path);
    if (!c->herm) return hx_ctx_write_state(c, all.data(), all.size());
    // Packed slabs hold the Hermitian part.  A snapshot written by another
    // program (the reference computes (r, c) and (c, r) separately, in single
    // precision by default) is Hermitian to its rounding only: accept up to
    // 1e-5 of each ADO's largest element and store the Hermitian part.
    const int D = c->d;
    std::vector<char> ok(static_cast<size_t>(c->H), 1);
    parallel_for(c->H, [&](long long k) {
        double* x = all.data() + 2 * static_cast<size_t>(k) * c->slab;
        double big2 = 0.0;
        for (size_t e = 0; e < c->slab; ++e) big2 = std::max(big2, x[2 * e] * x[2 * e] + x[2 * e + 1] * x[2 * e + 1]);
        const double tol2 = 1e-10 * big2;
        for (int r = 0; r < D && ok[k]; ++r)
            for (int q = r; q < D; ++q) {
                double* a = x + 2 * (static_cast<size_t>(r) * D + q);
                double* b = x + 2 * (static_cast<size_t>(q) * D + r);
                const double dr = a[0] - b[0], di = a[1] + b[1];
                if (dr * dr + di * di > tol2) {
                    ok[k] = 0;
                    break;
                }
                const double re = 0.5 * (a[0] + b[0]), im = 0.5 * (a[1] - b[1]);
                a[0] = re;
                a[1] = im;
                b[0] = re;
                b[1] = r == q ? im : -im;
            }
    });
    for (long long k = 0; k < c->H; ++k)
        if (!ok[k])
            return fail(HX_ERR_INVALID_RUNTIME_OPTION,
                        "ADO " + std::to_string(k) + " of " + path +
                            " is not Hermitian; load it into a context made with HX_FLAG_FULL_STATE");
    return hx_ctx_write_state(c, all.data(), all.size());
}

int hx_ctx_state_device_ptr(hx_ctx* c, void** ptr)
{
    if (!c || !ptr) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL argument");
    *ptr = c->rho;
    return HX_OK;
}

int hx_ctx_inject_wait_timeout(hx_ctx* c)
{
    if (!c) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL context");
    if (!c->use_small_step || c->closure)
        return fail(HX_ERR_UNSUPPORTED_EXECUTION, "no grid-barrier waits in this context's steps");
    c->stall_next_step = true;
    return HX_OK;
}

int hx_ctx_dense_product(hx_ctx* c, uint32_t count)
{
    if (!c) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL context");
    if (!c->dense) return fail(HX_ERR_UNSUPPORTED_EXECUTION, "not an HX_FLAG_DENSE_H context");
    for (uint32_t i = 0; i < count; ++i) c->counters.kernel_launches += launch_dense_product(c, c->rho32);
    const int rc = check_launch("dense product");
    if (rc != HX_OK) return rc;
    if (c->launch_failed) {
        c->launch_failed = false;
        return fail(HX_ERR_UNSUPPORTED_EXECUTION, "the tensor-core product could not be enqueued");
    }
    return HX_OK;
}

int hx_ctx_rhs(hx_ctx* c, double* out, uint64_t n)
{
    if (!c || !out) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL argument");
    const size_t count = static_cast<size_t>(c->H) * c->slab;
    if (n < 2 * count) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "output buffer too small");
    c->counters.kernel_launches += launch_stage_any(c, c->rho, c->rho, c->ua, 1.0, hx::kBaseZero);
    int rc = check_launch("stage kernel launch");
    if (rc != HX_OK) return rc;
    if (c->mixed) {
        rc = read_mixed(c, c->ua32, c->ua, out);
        return rc != HX_OK ? rc : read_error_flag(c);
    }
    if (c->herm) {
        rc = read_herm(c, c->ua, static_cast<size_t>(c->H), out);
        return rc != HX_OK ? rc : read_error_flag(c);
    }
    HX_CUDA_TRY(cudaMemcpyAsync(out, c->ua, count * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
    HX_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return read_error_flag(c);
}

int hx_ctx_set_closure(hx_ctx* c, hx_closure* cl)
{
    if (!c) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL context");
    if (cl) {
        uint32_t top = 0;
        hx_closure_info(cl, &top, nullptr, nullptr, nullptr, nullptr);
        if (c->mixed || c->use_flip || c->use_large || c->use_csr || c->d > 64)
            return fail(HX_ERR_UNSUPPORTED_EXECUTION, "closures run with double precision and dim <= 64");
        if (!hx::closure_matches_hierarchy(cl, c->d, c->M, c->H))
            return fail(HX_ERR_INVALID_RUNTIME_OPTION, "the closure was made for another hierarchy");
    }
    c->closure = cl;
    return HX_OK;
}

int hx_ctx_check_finite(hx_ctx* c)
{
    if (!c) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL context");
    if (c->mixed) {
        std::vector<double> all(2 * static_cast<size_t>(c->H) * c->slab);
        const int rc = read_mixed(c, c->rho32, c->rho, all.data());
        if (rc != HX_OK) return rc;
        for (double v : all)
            if (!std::isfinite(v)) return fail(HX_ERR_NON_FINITE, "state holds non-finite values");
        return read_error_flag(c);
    }
    int host = 0;
    int* scratch = reinterpret_cast<int*>(c->obs + 3);
    HX_CUDA_TRY(cudaMemsetAsync(scratch, 0, sizeof(int), c->stream));
    hx::launch_finite_check(c->rho, static_cast<long long>(c->H) * c->slab_store, scratch, c->stream);
    c->counters.kernel_launches += 1;
    int rc = check_launch("finite check");
    if (rc != HX_OK) return rc;
    HX_CUDA_TRY(cudaMemcpyAsync(&host, scratch, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    HX_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (host != 0) return fail(HX_ERR_NON_FINITE, "state holds non-finite values");
    return read_error_flag(c);
}

}  // extern "C"
