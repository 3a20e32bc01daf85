// Host-side math of helix_b200: Pade decomposition, bath constants,
// binomials, error text and the seeded instance generator.

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "hx_internal.h"

namespace hx {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int code, const std::string& msg)
{
    g_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char* what)
{
    const int code = (e == cudaErrorMemoryAllocation) ? HX_ERR_OUT_OF_MEMORY : HX_ERR_CUDA;
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return code;
}

namespace {

// Symmetric eigenvalues by cyclic-pivot Jacobi rotations with the largest
// off-diagonal element chosen each iteration; converged when the strict
// lower-triangle L1 norm is <= 1e-14 (the criterion of the reference's
// getEigval, src/psd/eigenvalues.cu:92-128).  Returns sorted ascending.
bool symmetric_eigenvalues(int n, std::vector<double> a, std::vector<double>& eig)
{
    auto at = [&](int r, int c) -> double& { return a[static_cast<size_t>(c) * n + r]; };
    auto lower_norm = [&]() {
        double s = 0.0;
        for (int c = 0; c < n; ++c)
            for (int r = c + 1; r < n; ++r) s += std::fabs(at(r, c));
        return s;
    };
    const int limit = std::max(16, 100 * n * n);
    double res = lower_norm();
    for (int it = 0; it < limit && res > 1.0e-14; ++it) {
        int pr = 1, pc = 0;
        double big = std::fabs(at(1, 0));
        for (int c = 0; c < n; ++c)
            for (int r = c + 1; r < n; ++r) {
                const double v = std::fabs(at(r, c));
                if (v > big) { big = v; pr = r; pc = c; }
            }
        const int p = pc, q = pr;
        const double app = at(p, p), aqq = at(q, q), apq = at(p, q);
        if (apq != 0.0) {
            const double ang = 0.5 * std::atan2(2.0 * apq, aqq - app);
            const double cs = std::cos(ang), sn = std::sin(ang);
            for (int k = 0; k < n; ++k) {
                if (k == p || k == q) continue;
                const double akp = at(k, p), akq = at(k, q);
                const double np = cs * akp - sn * akq;
                const double nq = sn * akp + cs * akq;
                at(k, p) = np; at(p, k) = np;
                at(k, q) = nq; at(q, k) = nq;
            }
            at(p, p) = cs * cs * app - 2.0 * sn * cs * apq + sn * sn * aqq;
            at(q, q) = sn * sn * app + 2.0 * sn * cs * apq + cs * cs * aqq;
            at(p, q) = 0.0; at(q, p) = 0.0;
        }
        res = lower_norm();
    }
    if (res > 1.0e-14) return false;
    eig.resize(n);
    for (int i = 0; i < n; ++i) eig[i] = at(i, i);
    std::sort(eig.begin(), eig.end());
    return true;
}

std::vector<double> tridiagonal(int n, int shift)
{
    // off-diagonals 1/sqrt(b_{x+shift} b_{y+shift}), b_m = 2m + 1 (Bose)
    std::vector<double> a(static_cast<size_t>(n) * n, 0.0);
    for (int x = 0; x < n; ++x)
        for (int y = 0; y < n; ++y)
            if (std::abs(x - y) == 1)
                a[static_cast<size_t>(x) * n + y] =
                    1.0 / std::sqrt(1.0 * (2 * (x + shift) + 1) * (2 * (y + shift) + 1));
    return a;
}

}  // namespace

bool psd_bose(int K, double* poles, double* residues)
{
    if (K <= 0) return true;
    std::vector<double> e1, e2;
    const int n1 = 2 * K;
    if (!symmetric_eigenvalues(n1, tridiagonal(n1, 1), e1)) return false;
    for (int i = 0; i < K; ++i) poles[i] = 2.0 / e1[n1 - 1 - i];
    const int n2 = n1 - 1;
    if (!symmetric_eigenvalues(n2, tridiagonal(n2, 2), e2)) return false;
    const int m = n2 / 2;
    std::vector<double> xi(K), zeta(m);
    for (int i = 0; i < K; ++i) xi[i] = poles[i] * poles[i];
    for (int i = 0; i < m; ++i) zeta[i] = 4.0 / (e2[n2 - 1 - i] * e2[n2 - 1 - i]);
    const double scale = K * (2 * (K + 1) + 1);
    for (int i = 0; i < K; ++i) {
        double t = (i == K - 1) ? 0.5 * scale : 0.5 * scale * (zeta[i] - xi[i]) / (xi[K - 1] - xi[i]);
        for (int j = 0; j < m; ++j)
            if (j != i) t *= (zeta[j] - xi[i]) / (xi[j] - xi[i]);
        residues[i] = t;
    }
    return true;
}

bool bath_constants(double beta, double gamma, double zeta, int K, BathConst& b)
{
    std::vector<double> poles(std::max(K, 1)), res(std::max(K, 1));
    if (!psd_bose(K, poles.data(), res.data())) return false;
    const double omega0 = 1.0;
    b.K = K;
    b.nu.assign(K + 1, 0.0);
    b.nu[0] = gamma;
    for (int k = 1; k <= K; ++k) b.nu[k] = poles[k - 1] / beta;
    const double bgh = 0.5 * beta * gamma;
    const double bo = beta * omega0;
    double sigma = 1.0 - bgh / std::tan(bgh);
    for (int k = 1; k <= K; ++k)
        sigma = sigma - 2.0 * res[k - 1] * gamma * gamma / ((b.nu[k] * b.nu[k]) - gamma * gamma);
    b.xi = sigma * (zeta / bo);
    b.counter = zeta * bgh / bo;
    b.phi.assign(K, 0.0);
    for (int k = 1; k <= K; ++k)
        b.phi[k - 1] = (zeta / bo) * 2.0 * res[k - 1] * gamma * gamma / ((b.nu[k] * b.nu[k]) - gamma * gamma);
    b.theta_c = beta * gamma * 0.5 / std::tan(beta * gamma * 0.5) * zeta / bo;
    b.theta_a = beta * gamma * 0.5 * zeta / bo;
    return std::isfinite(b.xi) && std::isfinite(b.theta_c);
}

uint64_t binom_u64(int n, int k)
{
    if (k < 0 || n < 0 || k > n) return 0;
    k = std::min(k, n - k);
    unsigned __int128 r = 1;
    for (int i = 1; i <= k; ++i) r = r * static_cast<unsigned>(n - k + i) / static_cast<unsigned>(i);
    return static_cast<uint64_t>(r);
}

int pauli_spin(const double* v, int D)
{
    for (int p = 0; (1 << p) < D; ++p) {
        bool ok = true;
        for (int r = 0; r < D && ok; ++r) ok = v[r] == (((r >> p) & 1) ? 1.0 : -1.0);
        if (ok) return p;
    }
    return -1;
}

}  // namespace hx

// ---------------------------------------------------------------------------
// C ABI: host-only entry points
// ---------------------------------------------------------------------------

extern "C" {

const char* hx_last_error(void) { return hx::g_last_error.c_str(); }

const char* hx_version(void) { return "helix_b200 0.1.0"; }

int hx_hierarchy_size(uint32_t modes, uint32_t max_depth, uint64_t* count)
{
    if (!count) return hx::fail(HX_ERR_INVALID_RUNTIME_OPTION, "count pointer is NULL");
    if (modes == 0) return hx::fail(HX_ERR_UNSUPPORTED_HIERARCHY, "hierarchy needs at least one mode");
    // C(modes + max_depth - 1, modes): vectors with sum < max_depth
    *count = max_depth == 0 ? 0 : hx::binom_u64(static_cast<int>(modes + max_depth - 1), static_cast<int>(modes));
    return HX_OK;
}

int hx_psd(uint32_t K, double* poles, double* residues)
{
    if (K > 0 && (!poles || !residues)) return hx::fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL output");
    if (!hx::psd_bose(static_cast<int>(K), poles, residues))
        return hx::fail(HX_ERR_UNSUPPORTED_BATH, "Pade decomposition did not converge");
    return HX_OK;
}

int hx_seeded_couplings(uint32_t n, uint64_t seed, double* J)
{
    if (!J) return hx::fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL output");
    uint64_t state = seed;
    auto next = [&]() {
        state += 0x9E3779B97F4A7C15ull;
        uint64_t z = state;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    auto uniform = [&]() { return static_cast<double>(next() >> 11) * (1.0 / 9007199254740992.0); };
    const double two_pi = 6.283185307179586;
    std::memset(J, 0, sizeof(double) * n * n);
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t j = i + 1; j < n; ++j) {
            const double u1 = 1.0 - uniform();
            const double u2 = uniform();
            const double z = std::sqrt(-2.0 * std::log(u1)) * std::cos(two_pi * u2);
            J[i * n + j] = z;
            J[j * n + i] = z;
        }
    return HX_OK;
}

int hx_write_energy_trace(const char* path, const double* times, const double* energies, uint64_t n)
{
    if (!path || (n > 0 && (!times || !energies))) return hx::fail(HX_ERR_INVALID_RUNTIME_OPTION, "NULL argument");
    std::FILE* f = std::fopen(path, "w");
    if (!f) return hx::fail(HX_ERR_INVALID_RUNTIME_OPTION, std::string("cannot open ") + path + " for writing");
    bool ok = true;
    for (uint64_t i = 0; i < n && ok; ++i) ok = std::fprintf(f, "%.8g %.8g\n", times[i], energies[i]) > 0;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? HX_OK : hx::fail(HX_ERR_INVALID_RUNTIME_OPTION, std::string("short write to ") + path);
}

}  // extern "C"
