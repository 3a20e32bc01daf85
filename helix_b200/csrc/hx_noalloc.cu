// hx_rhs_noalloc: one evaluation of the HEOM right-hand side that allocates
// no memory.
//
// Who needs it: callers that cannot call cudaMalloc while they run us, for
// example a host framework that hands out every byte of device memory from
// its own pool, or a process that has used up its device-memory budget; for
// them even the temporary allocations of hx_ctx_create are not possible.
// They pass the state and the result buffer (device memory they already
// own), and the entry point keeps its working tables (hierarchy rows and
// neighbour edges, per-ADO weights, operator diagonals, the error word) in
// one fixed-size array compiled into this library.
//
// Facts a caller must know:
//  * the array is kNoallocScratchBytes (8 MiB) of device memory, reserved on
//    every GPU that loads the library until the process exits;
//  * a problem whose tables do not fit is rejected with
//    HX_ERR_UNSUPPORTED_HIERARCHY and a message that states the size needed;
//  * the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) with that device current and caches it; make
//    that first call before any stream capture.  The cached address belongs
//    to the device's primary context: after cudaDeviceReset on that device
//    it is stale, so do not call this entry point again in that process;
//  * `rho_device` and `drho_device` must be 16-byte aligned (the state is
//    read by bulk copies) and must not overlap: every block reads other ADOs'
//    slabs of `rho_device` while others write `drho_device`, so an in-place
//    call would race; both are checked and rejected with
//    HX_ERR_INVALID_RUNTIME_OPTION;
//  * `stream` must belong to the current device (checked);
//  * all calls share the one array and it keeps the previous call's
//    contents: every table is rewritten and the error word is cleared at the
//    start of each call, and two calls that overlap on the GPU (different
//    streams, or different host threads) race on the array;
//  * the call returns when the result is complete.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "hx_internal.h"

namespace {

constexpr size_t kNoallocScratchBytes = size_t(8) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array for the current device (set up once).
int scratch_address(void** out)
{
    int dev = 0;
    HX_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return hx::fail(HX_ERR_CUDA, "device index outside the scratch table");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return hx::cuda_fail(e, "cudaGetSymbolAddress(noalloc scratch)");
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return HX_OK;
}

// Bump allocator over the scratch array (256-byte aligned pieces).
struct Carve {
    unsigned char* base;
    size_t used = 0;
    template <typename T>
    T* take(size_t count)
    {
        used = (used + 255) & ~size_t(255);
        T* p = reinterpret_cast<T*>(base + used);
        used += std::max<size_t>(count, 1) * sizeof(T);
        return p;
    }
};

}  // namespace

extern "C" int hx_rhs_noalloc(const hx_problem* p, const double* rho_device, double* drho_device, void* stream)
{
    using hx::fail;
    if (!p || !rho_device || !drho_device) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL argument");
    const uint32_t d = p->dim;
    if (d < 2 || (d & (d - 1)) != 0) return fail(HX_ERR_INVALID_DIMENSION, "dim must be a power of two >= 2");
    int logd = 0;
    while ((1u << logd) < d) ++logd;
    if (logd > hx::kMaxLogD) return fail(HX_ERR_UNSUPPORTED_EXECUTION, "the right-hand side supports dim <= 64");
    if (!p->h_diag) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "h_diag is NULL");
    if (p->precision != HX_PRECISION_DOUBLE) return fail(HX_ERR_UNSUPPORTED_PRECISION, "double precision only");
    if (p->n_baths == 0 || !p->baths || p->n_baths > static_cast<uint32_t>(hx::kMaxBaths))
        return fail(HX_ERR_UNSUPPORTED_BATH, "1..64 baths are required");
    if (p->max_depth < 1) return fail(HX_ERR_UNSUPPORTED_HIERARCHY, "max_depth must be >= 1");
    if ((reinterpret_cast<uintptr_t>(rho_device) | reinterpret_cast<uintptr_t>(drho_device)) % 16 != 0)
        return fail(HX_ERR_INVALID_RUNTIME_OPTION, "rho_device and drho_device must be 16-byte aligned");

    const int J = static_cast<int>(p->n_baths);
    if (p->h_csr) return fail(HX_ERR_UNSUPPORTED_EXECUTION, "hx_rhs_noalloc takes diagonal plus flip Hamiltonians only");
    for (int j = 0; j < J; ++j)
        if (p->baths[j].coupling_csr)
            return fail(HX_ERR_UNSUPPORTED_BATH, "hx_rhs_noalloc supports diagonal coupling operators only");
    for (int j = 0; j < J; ++j)
        if (p->baths[j].coupling_flip)
            for (int i = 0; i < logd; ++i)
                if (p->baths[j].coupling_flip[i] != 0.0)
                    return fail(HX_ERR_UNSUPPORTED_BATH, "hx_rhs_noalloc supports diagonal coupling operators only");
    std::vector<hx::BathConst> bc(J);
    int M = 0;
    for (int j = 0; j < J; ++j) {
        const hx_bath& b = p->baths[j];
        if (!b.coupling_diag || !(b.inverse_temperature > 0.0) || !(b.damping > 0.0) || b.pade_terms > 32 ||
            !hx::bath_constants(b.inverse_temperature, b.damping, b.coupling_strength, static_cast<int>(b.pade_terms),
                                bc[j]))
            return fail(HX_ERR_UNSUPPORTED_BATH, "invalid bath");
        bc[j].offset = M;
        M += static_cast<int>(b.pade_terms) + 1;
    }
    if (M > hx::kMaxModes) return fail(HX_ERR_UNSUPPORTED_HIERARCHY, "too many modes");
    uint64_t Hu = 0;
    int rc = hx_hierarchy_size(static_cast<uint32_t>(M), p->max_depth, &Hu);
    if (rc != HX_OK) return rc;
    const long long H = static_cast<long long>(Hu);
    {
        const uintptr_t bytes = static_cast<uintptr_t>(Hu) * d * d * 2 * sizeof(double);
        const uintptr_t a = reinterpret_cast<uintptr_t>(rho_device), b = reinterpret_cast<uintptr_t>(drho_device);
        if (a < b + bytes && b < a + bytes)
            return fail(HX_ERR_INVALID_RUNTIME_OPTION, "rho_device and drho_device must not overlap");
    }
    const int D = static_cast<int>(p->max_depth);
    const int nmax = M + D + 1;
    const int kcols = M + 1;
    if (nmax > 192) return fail(HX_ERR_UNSUPPORTED_HIERARCHY, "hierarchy too deep for the table builder");

    // host copies of the small inputs
    std::vector<unsigned long long> binom(static_cast<size_t>(nmax) * kcols, 0ull);
    for (int n = 0; n < nmax; ++n)
        for (int k = 0; k <= M && k <= n; ++k) binom[n * kcols + k] = hx::binom_u64(n, k);
    std::vector<double> hflip(logd, 0.0), vd(static_cast<size_t>(J) * d), xi(J), ct(J), tc(J), ta(J), nu(M),
        phi(M, 0.0);
    if (p->h_flip) std::copy(p->h_flip, p->h_flip + logd, hflip.begin());
    std::vector<int32_t> off(J + 1), mb(M), mk(M);
    for (int j = 0; j < J; ++j) {
        std::copy(p->baths[j].coupling_diag, p->baths[j].coupling_diag + d, vd.begin() + static_cast<size_t>(j) * d);
        xi[j] = bc[j].xi;
        ct[j] = bc[j].counter;
        tc[j] = bc[j].theta_c;
        ta[j] = bc[j].theta_a;
        off[j] = bc[j].offset;
        for (int k = 0; k <= bc[j].K; ++k) {
            const int m = bc[j].offset + k;
            mb[m] = j;
            mk[m] = k;
            nu[m] = bc[j].nu[k];
            if (k >= 1) phi[m] = bc[j].phi[k - 1];
        }
    }
    off[J] = M;

    // carve the scratch array; reject problems that do not fit
    Carve sizing{nullptr};
    sizing.take<unsigned long long>(binom.size());
    sizing.take<int32_t>(static_cast<size_t>(H) * M);
    sizing.take<int32_t>(static_cast<size_t>(H) * 2 * M);
    sizing.take<double>(static_cast<size_t>(H) * M);
    sizing.take<double>(static_cast<size_t>(H) * J);
    sizing.take<double>(static_cast<size_t>(H));
    sizing.take<double>(d);
    sizing.take<double>(logd);
    sizing.take<double>(vd.size());
    for (int i = 0; i < 4; ++i) sizing.take<double>(J);
    sizing.take<double>(M);
    sizing.take<double>(M);
    for (int i = 0; i < 3; ++i) sizing.take<int32_t>(M + J + 1);
    sizing.take<int>(1);
    if (sizing.used > kNoallocScratchBytes)
        return fail(HX_ERR_UNSUPPORTED_HIERARCHY,
                    "hx_rhs_noalloc needs " + std::to_string(sizing.used) + " bytes of scratch for this hierarchy; "
                    "its fixed scratch array holds " + std::to_string(kNoallocScratchBytes) + " bytes");

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    {
        int cur = 0, sdev = 0;
        HX_CUDA_TRY(cudaGetDevice(&cur));
        HX_CUDA_TRY(cudaStreamGetDevice(s, &sdev));
        if (sdev != cur) return fail(HX_ERR_INVALID_RUNTIME_OPTION, "stream belongs to another device than the current one");
    }
    void* base = nullptr;
    if ((rc = scratch_address(&base)) != HX_OK) return rc;
    Carve cv{static_cast<unsigned char*>(base)};
    auto* d_binom = cv.take<unsigned long long>(binom.size());
    auto* d_rows = cv.take<int32_t>(static_cast<size_t>(H) * M);
    auto* d_edges = cv.take<int32_t>(static_cast<size_t>(H) * 2 * M);
    auto* d_acoef = cv.take<double>(static_cast<size_t>(H) * M);
    auto* d_bcoef = cv.take<double>(static_cast<size_t>(H) * J);
    auto* d_gsum = cv.take<double>(static_cast<size_t>(H));
    auto* d_hdiag = cv.take<double>(d);
    auto* d_hflip = cv.take<double>(logd);
    auto* d_vdiag = cv.take<double>(vd.size());
    auto* d_xi = cv.take<double>(J);
    auto* d_ct = cv.take<double>(J);
    auto* d_tc = cv.take<double>(J);
    auto* d_ta = cv.take<double>(J);
    auto* d_nu = cv.take<double>(M);
    auto* d_phi = cv.take<double>(M);
    auto* d_off = cv.take<int32_t>(M + J + 1);
    auto* d_mb = cv.take<int32_t>(M + J + 1);
    auto* d_mk = cv.take<int32_t>(M + J + 1);
    auto* d_flag = cv.take<int>(1);

    auto up = [&](void* dst, const void* src, size_t bytes) {
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
    };
    cudaError_t e = up(d_binom, binom.data(), binom.size() * sizeof(unsigned long long));
    if (e == cudaSuccess) e = up(d_hdiag, p->h_diag, d * sizeof(double));
    if (e == cudaSuccess) e = up(d_hflip, hflip.data(), logd * sizeof(double));
    if (e == cudaSuccess) e = up(d_vdiag, vd.data(), vd.size() * sizeof(double));
    if (e == cudaSuccess) e = up(d_xi, xi.data(), J * sizeof(double));
    if (e == cudaSuccess) e = up(d_ct, ct.data(), J * sizeof(double));
    if (e == cudaSuccess) e = up(d_tc, tc.data(), J * sizeof(double));
    if (e == cudaSuccess) e = up(d_ta, ta.data(), J * sizeof(double));
    if (e == cudaSuccess) e = up(d_nu, nu.data(), M * sizeof(double));
    if (e == cudaSuccess) e = up(d_phi, phi.data(), M * sizeof(double));
    if (e == cudaSuccess) e = up(d_off, off.data(), (J + 1) * sizeof(int32_t));
    if (e == cudaSuccess) e = up(d_mb, mb.data(), M * sizeof(int32_t));
    if (e == cudaSuccess) e = up(d_mk, mk.data(), M * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMemsetAsync(d_flag, 0, sizeof(int), s);  // the error word must start at zero
    if (e != cudaSuccess) return hx::cuda_fail(e, "hx_rhs_noalloc upload");

    hx::launch_tables_with_binomials(d_binom, kcols, M, D, H, d_rows, d_edges, s);
    hx::launch_coefficients(d_rows, H, M, J, d_mb, d_mk, d_nu, d_tc, d_ta, d_phi, d_off, d_acoef, d_bcoef, d_gsum, s);
    hx::StageTables t{};
    t.edges = d_edges;
    t.acoef = d_acoef;
    t.bcoef = d_bcoef;
    t.gsum = d_gsum;
    t.hdiag = d_hdiag;
    t.hflip = d_hflip;
    t.vdiag = d_vdiag;
    t.xi = d_xi;
    t.counter = d_ct;
    t.bath_off = d_off;
    t.order = nullptr;
    t.error_flag = d_flag;
    t.H = H;
    t.M = M;
    t.J = J;
    t.logd = logd;
    hx::launch_stage(t, reinterpret_cast<const double2*>(rho_device), reinterpret_cast<const double2*>(rho_device),
                     reinterpret_cast<double2*>(drho_device), 1.0, hx::kBaseZero, s);
    e = cudaGetLastError();
    if (e != cudaSuccess) return hx::cuda_fail(e, "hx_rhs_noalloc launch");
    int flag = 0;
    e = cudaMemcpyAsync(&flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // host inputs above must outlive their copies
    if (e != cudaSuccess) return hx::cuda_fail(e, "hx_rhs_noalloc");
    if (flag != 0) return fail(HX_ERR_DEVICE_TIMEOUT, "a device-side wait ran out of its iteration budget");
    return HX_OK;
}
