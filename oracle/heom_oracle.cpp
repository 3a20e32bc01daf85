// HEOM CPU oracle — TEST INFRASTRUCTURE ONLY.
//
// A plain FP64 CPU restatement of the reference HEOM propagator (HELIX,
// src/liouville.cu + src/initialize.cu + src/initialize_detail.h +
// src/psd/*.cu).  It exists so that tests, the smoke check and the CPU
// baseline leg of bench.py can check the CUDA product path against an
// independent implementation.  Nothing in the product library links or calls
// this file, and the product path never falls back to it.
//
// Generalisation beyond the reference: the reference has exactly one bath and
// one coupling operator V.  Here every bath j carries its own coupling
// operator V_j and its own Drude-Lorentz/Pade parameters; every per-bath term
// of the reference right-hand side (src/liouville.cu:813-860) is summed over
// j.  With one bath the formulas reduce term for term to the reference.
// Mode order is bath-major: mode = offset_j + k, k = 0 the Drude mode.
//
// Parity status: pinned.  PSD constants against tests/unit/psd_reference_tests.cu,
// hierarchy tables bit-exact against the reference's own initialize_detail.h
// functions compiled from source (oracle/ref_host_shim.cu), and the
// legacy-model energy trace against examples/outputEnergy.txt.
//
// Build: g++ -O3 -march=x86-64-v3 -ffp-contract=off -fopenmp -shared -fPIC (oracle/build.py).

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <new>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using cplx = std::complex<double>;

// ---------------------------------------------------------------------------
// Hierarchy tables (reference: src/initialize_detail.h:159-269)
// ---------------------------------------------------------------------------

// Number of index vectors n in N^M with sum(n) < maxLevel.  Same recursion as
// hierarchySizeFor (initialize_detail.h:159-172).
long long hierarchy_size(int modes, int maxLevel)
{
    if (maxLevel <= 0) return 0;
    if (modes == 1) return maxLevel;
    long long total = 0;
    for (int i = 0; i < maxLevel; ++i) total += hierarchy_size(modes - 1, maxLevel - i);
    return total;
}

// Rows in lexicographic order, mode 0 most significant, sum(n) < maxLevel
// (the order appendHierarchyRows emits, initialize_detail.h:174-214, for
// modeCount != 2; see DESIGN notes for the modeCount == 2 overflow there).
void emit_rows(int depth, int modes, int maxLevel, int partial, std::vector<int>& prefix,
               std::vector<int>& out)
{
    if (depth == modes) {
        out.insert(out.end(), prefix.begin(), prefix.end());
        return;
    }
    for (int i = 0; partial + i < maxLevel; ++i) {
        prefix[depth] = i;
        emit_rows(depth + 1, modes, maxLevel, partial + i, prefix, out);
    }
    prefix[depth] = 0;
}

// edges[i][k] = index of n_i + e_k, edges[i][M+k] = index of n_i - e_k,
// sentinel = H when the neighbour is outside the truncated hierarchy
// (buildHierarchyEdges, initialize_detail.h:234-269).  A map lookup replaces
// the reference's O(H^2 M) search; rows are unique, so the result is equal.
void build_edges(const std::vector<int>& rows, int modes, long long H, std::vector<int>& edges)
{
    edges.assign(static_cast<size_t>(H) * 2 * modes, static_cast<int>(H));
    std::map<std::vector<int>, int> index;
    for (long long i = 0; i < H; ++i)
        index.emplace(std::vector<int>(rows.begin() + i * modes, rows.begin() + (i + 1) * modes),
                      static_cast<int>(i));
    std::vector<int> probe(modes);
    for (long long i = 0; i < H; ++i) {
        for (int k = 0; k < modes; ++k) {
            std::copy(rows.begin() + i * modes, rows.begin() + (i + 1) * modes, probe.begin());
            probe[k] += 1;
            auto it = index.find(probe);
            if (it != index.end()) {
                edges[i * 2 * modes + k] = it->second;
                edges[static_cast<size_t>(it->second) * 2 * modes + modes + k] = static_cast<int>(i);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Pade spectrum decomposition of the Bose function, [N-1/N]
// (reference: src/psd/psd.cu:12-113 with the Jacobi eigen-solver of
// src/psd/eigenvalues.cu:92-128).
// ---------------------------------------------------------------------------

// Classical Jacobi eigenvalue iteration for a real symmetric matrix (largest
// off-diagonal pivot each sweep), tolerance 1e-14 on the off-diagonal L1 norm.
bool jacobi_eigenvalues(int n, std::vector<double>& a, std::vector<double>& eig)
{
    auto A = [&](int r, int c) -> double& { return a[static_cast<size_t>(r) * n + c]; };
    auto offnorm = [&]() {
        double s = 0.0;
        for (int c = 0; c < n; ++c)
            for (int r = c + 1; r < n; ++r) s += std::fabs(A(r, c));
        return s;
    };
    const int maxIter = std::max(16, 100 * n * n);
    double res = offnorm();
    for (int it = 0; it < maxIter && res > 1.0e-14; ++it) {
        int p = 0, q = 1;
        double best = -1.0;
        for (int c = 0; c < n; ++c)
            for (int r = c + 1; r < n; ++r)
                if (std::fabs(A(r, c)) > best) { best = std::fabs(A(r, c)); p = c; q = r; }
        const double app = A(p, p), aqq = A(q, q), apq = A(p, q);
        if (apq != 0.0) {
            const double th = 0.5 * std::atan2(2.0 * apq, aqq - app);
            const double cs = std::cos(th), sn = std::sin(th);
            for (int k = 0; k < n; ++k) {
                if (k == p || k == q) continue;
                const double akp = A(k, p), akq = A(k, q);
                A(k, p) = A(p, k) = cs * akp - sn * akq;
                A(k, q) = A(q, k) = sn * akp + cs * akq;
            }
            A(p, p) = cs * cs * app - 2.0 * sn * cs * apq + sn * sn * aqq;
            A(q, q) = sn * sn * app + 2.0 * sn * cs * apq + cs * cs * aqq;
            A(p, q) = A(q, p) = 0.0;
        }
        res = offnorm();
    }
    if (res > 1.0e-14) return false;
    eig.resize(n);
    for (int i = 0; i < n; ++i) eig[i] = A(i, i);
    std::sort(eig.begin(), eig.end());
    return true;
}

// Poles xi_k (k < K) and residues eta_k of the [K-1/K] Pade approximant of
// the Bose function: poles are 2/eigenvalue of the 2K tridiagonal matrix
// with off-diagonals 1/sqrt(b_i b_j), b_m = 2m+1; residues from the
// (2K-1) matrix built on b_{m+1} (psd.cu:17-111).
bool psd_bose(int K, double* poles, double* residues)
{
    if (K <= 0) return true;
    auto b = [](int m) { return 2 * m + 1; };
    int n = 2 * K;
    std::vector<double> a(static_cast<size_t>(n) * n, 0.0), e1, e2;
    for (int x = 0; x < n; ++x)
        for (int y = 0; y < n; ++y)
            if (std::abs(x - y) == 1) a[x * n + y] = 1.0 / std::sqrt(1.0 * b(x + 1) * b(y + 1));
    if (!jacobi_eigenvalues(n, a, e1)) return false;
    for (int i = 0; i < K; ++i) poles[i] = 2.0 / e1[n - 1 - i];
    n -= 1;
    a.assign(static_cast<size_t>(n) * n, 0.0);
    for (int x = 0; x < n; ++x)
        for (int y = 0; y < n; ++y)
            if (std::abs(x - y) == 1) a[x * n + y] = 1.0 / std::sqrt(1.0 * b(x + 2) * b(y + 2));
    if (n > 0 && !jacobi_eigenvalues(n, a, e2)) return false;
    const int m = n / 2;
    std::vector<double> xi(K), zeta(m);
    for (int i = 0; i < K; ++i) xi[i] = poles[i] * poles[i];
    for (int i = 0; i < m; ++i) zeta[i] = 4.0 / (e2[n - 1 - i] * e2[n - 1 - i]);
    const double scale = K * b(K + 1);
    for (int i = 0; i < K; ++i) {
        double t = (i == K - 1) ? 0.5 * scale : 0.5 * scale * (zeta[i] - xi[i]) / (xi[K - 1] - xi[i]);
        for (int j = 0; j < m; ++j) {
            if (i == j) continue;
            t *= (zeta[j] - xi[i]) / (xi[j] - xi[i]);
        }
        residues[i] = t;
    }
    return true;
}

// ---------------------------------------------------------------------------
// Operators
// ---------------------------------------------------------------------------

struct Csr {
    int n = 0;
    std::vector<int> ptr, col;
    std::vector<cplx> val;
};

Csr make_csr(int n, const int* ptr, const int* col, const double* val_re_im)
{
    Csr m;
    m.n = n;
    m.ptr.assign(ptr, ptr + n + 1);
    const int nnz = ptr[n];
    m.col.assign(col, col + nnz);
    m.val.resize(nnz);
    for (int i = 0; i < nnz; ++i) m.val[i] = cplx(val_re_im[2 * i], val_re_im[2 * i + 1]);
    return m;
}

Csr transpose(const Csr& a)
{
    Csr t;
    t.n = a.n;
    t.ptr.assign(a.n + 1, 0);
    for (int c : a.col) t.ptr[c + 1]++;
    for (int i = 0; i < a.n; ++i) t.ptr[i + 1] += t.ptr[i];
    t.col.resize(a.col.size());
    t.val.resize(a.val.size());
    std::vector<int> fill(t.ptr.begin(), t.ptr.end() - 1);
    for (int r = 0; r < a.n; ++r)
        for (int p = a.ptr[r]; p < a.ptr[r + 1]; ++p) {
            const int dst = fill[a.col[p]]++;
            t.col[dst] = r;
            t.val[dst] = a.val[p];
        }
    return t;
}

// out += alpha * (A X)          X, out: d x d row-major
void acc_left(const Csr& A, const cplx* X, cplx alpha, cplx* out)
{
    const int d = A.n;
    for (int r = 0; r < d; ++r)
        for (int p = A.ptr[r]; p < A.ptr[r + 1]; ++p) {
            const cplx a = alpha * A.val[p];
            const cplx* xr = X + static_cast<size_t>(A.col[p]) * d;
            cplx* orow = out + static_cast<size_t>(r) * d;
            for (int c = 0; c < d; ++c) orow[c] += a * xr[c];
        }
}

// out += alpha * (X A)   using At = transpose(A): (XA)[r][c] = sum_q X[r][q] At[c][q]
void acc_right(const Csr& At, const cplx* X, cplx alpha, cplx* out)
{
    const int d = At.n;
    for (int r = 0; r < d; ++r) {
        const cplx* xr = X + static_cast<size_t>(r) * d;
        cplx* orow = out + static_cast<size_t>(r) * d;
        for (int c = 0; c < d; ++c) {
            cplx s = 0.0;
            for (int p = At.ptr[c]; p < At.ptr[c + 1]; ++p) s += xr[At.col[p]] * At.val[p];
            orow[c] += alpha * s;
        }
    }
}

// out += k [A, X]   (k [V,X] semantics of CommutateSparse/addCommutateSparse, liouville.cu:275-337)
void acc_comm(const Csr& A, const Csr& At, const cplx* X, cplx k, cplx* out)
{
    acc_left(A, X, k, out);
    acc_right(At, X, -k, out);
}

// out += k {A, X}   (addAntiCommutateSparse, liouville.cu:338-366)
void acc_anti(const Csr& A, const Csr& At, const cplx* X, cplx k, cplx* out)
{
    acc_left(A, X, k, out);
    acc_right(At, X, k, out);
}

// ---------------------------------------------------------------------------
// Problem / context
// ---------------------------------------------------------------------------

struct Bath {
    double beta, gamma, zeta;  // zeta: reference coupling units, lambda = zeta*gamma/(2*omega0), omega0 = 1
    int K;
    Csr V, Vt;
    int offset;                // first mode index of this bath
    std::vector<double> nu;    // K+1 frequencies: nu_0 = gamma, nu_k = pole_{k-1}/beta
    cplx kxi, kxiCounter, kthetaC, kthetaA;
    std::vector<cplx> kphi;    // K
};

struct Ctx {
    int d = 0;
    Csr Hm, Hmt;
    std::vector<Bath> baths;
    int modes = 0;
    int maxDepth = 0;
    long long H = 0;
    std::vector<int> rows, edges;
    std::vector<cplx> rho, F, B, cur, nxt;   // state and Taylor scratch (H*d*d)
    std::vector<cplx> comm;                  // [V_j, rho_i] per (i, j)
};

// Bath coefficients, restating initializeBathCoefficients / calculateSigma /
// buildKPhi (src/initialize.cu:160-218) with omega0 = 1.
bool init_bath(Bath& b)
{
    std::vector<double> poles(b.K), residues(b.K);
    if (!psd_bose(b.K, poles.data(), residues.data())) return false;
    const double omega0 = 1.0;
    b.nu.resize(b.K + 1);
    b.nu[0] = b.gamma;
    for (int k = 1; k <= b.K; ++k) b.nu[k] = poles[k - 1] / b.beta;
    const double bgh = 0.5 * b.beta * b.gamma;
    const double bo = b.beta * omega0;
    double sigma = 1.0 - bgh / std::tan(bgh);
    for (int k = 1; k <= b.K; ++k)
        sigma = sigma - 2.0 * residues[k - 1] * b.gamma * b.gamma / (b.nu[k] * b.nu[k] - b.gamma * b.gamma);
    b.kxi = cplx(sigma * (b.zeta / bo), 0.0);
    b.kxiCounter = cplx(0.0, b.zeta * bgh / bo);
    b.kphi.resize(b.K);
    for (int k = 1; k <= b.K; ++k)
        b.kphi[k - 1] = cplx(0.0, (b.zeta / bo) * 2.0 * residues[k - 1] * b.gamma * b.gamma /
                                       (b.nu[k] * b.nu[k] - b.gamma * b.gamma));
    b.kthetaC = cplx(0.0, b.beta * b.gamma * 0.5 / std::tan(b.beta * b.gamma * 0.5) * b.zeta / bo);
    b.kthetaA = cplx(b.beta * b.gamma * 0.5 * b.zeta / bo, 0.0);
    return true;
}

// Right-hand side of the HEOM for all ADOs (getdRhoSparse, liouville.cu:749-869):
// stage 1 builds -i[H,rho_i] and the per-bath commutators [V_j, rho_i];
// stage 2 accumulates phi, psi, theta, theta2, sigma, Xi and counter terms in
// the reference order, per bath.  Missing neighbours contribute zero.
void rhs(Ctx& c, const cplx* in, cplx* out)
{
    const int d = c.d;
    const size_t slab = static_cast<size_t>(d) * d;
    const long long H = c.H;
    const int nb = static_cast<int>(c.baths.size());
    const cplx I(0.0, 1.0), mI(0.0, -1.0);

#pragma omp parallel for schedule(dynamic, 1)
    for (long long i = 0; i < H; ++i) {
        cplx* o = out + i * slab;
        std::fill(o, o + slab, cplx(0.0));
        acc_comm(c.Hm, c.Hmt, in + i * slab, mI, o);
        for (int j = 0; j < nb; ++j) {
            cplx* cb = c.comm.data() + (static_cast<size_t>(i) * nb + j) * slab;
            std::fill(cb, cb + slab, cplx(0.0));
            acc_comm(c.baths[j].V, c.baths[j].Vt, in + i * slab, cplx(1.0), cb);
        }
    }

    const int M = c.modes;
#pragma omp parallel for schedule(dynamic, 1)
    for (long long i = 0; i < H; ++i) {
        cplx* o = out + i * slab;
        const int* n = c.rows.data() + i * M;
        const int* e = c.edges.data() + i * 2 * M;
        for (int j = 0; j < nb; ++j) {
            const Bath& b = c.baths[j];
            auto commOf = [&](long long a) { return c.comm.data() + (static_cast<size_t>(a) * nb + j) * slab; };
            auto addMat = [&](cplx k, const cplx* x) {
                for (size_t t = 0; t < slab; ++t) o[t] += k * x[t];
            };
            // phi: -i [V, rho_{n+e_k}]
            for (int k = 0; k <= b.K; ++k) {
                const int up = e[b.offset + k];
                if (up < H) addMat(mI, commOf(up));
            }
            // psi: (-nu_k n_k) KPhi_k [V, rho_{n-e_k}], k >= 1
            for (int k = 1; k <= b.K; ++k) {
                const int dn = e[M + b.offset + k];
                const double jnu = -b.nu[k] * n[b.offset + k];
                if (dn < H) addMat(b.kphi[k - 1] * jnu, commOf(dn));
            }
            const int dn0 = e[M + b.offset];
            const double ngamma = -b.nu[0] * n[b.offset];
            // theta: (-gamma n_0) KThetaCommutate [V, rho_{n-e_0}]
            if (dn0 < H) addMat(b.kthetaC * ngamma, commOf(dn0));
            // theta2: (-gamma n_0) KThetaAntiCommutate {V, rho_{n-e_0}}
            if (dn0 < H) acc_anti(b.V, b.Vt, in + static_cast<size_t>(dn0) * slab, b.kthetaA * ngamma, o);
            // sigma: -(sum_k nu_k n_k) rho_n
            double s = 0.0;
            for (int k = 0; k <= b.K; ++k) s += b.nu[k] * n[b.offset + k];
            addMat(cplx(-s, 0.0), in + i * slab);
            // Xi: -KXi [V, [V, rho_n]]
            acc_comm(b.V, b.Vt, commOf(i), -b.kxi, o);
            // counter: -KXiCounter {V, [V, rho_n]}
            acc_anti(b.V, b.Vt, commOf(i), -b.kxiCounter, o);
        }
    }
    (void)I;
}

// One step of the reference integrator (develop(), liouville.cu:502-590):
// F = rho; cur = rho; for j = 1..order: cur = (dt/j) L cur; F += cur; rho = F.
void develop(Ctx& c, double dt, int order)
{
    const size_t n = c.rho.size();
    c.F = c.rho;
    const cplx* cur = c.rho.data();
    for (int j = 1; j <= order; ++j) {
        rhs(c, cur, c.nxt.data());
        const double f = dt / j;
#pragma omp parallel for
        for (long long t = 0; t < static_cast<long long>(n); ++t) {
            c.nxt[t] *= f;
            c.F[t] += c.nxt[t];
        }
        std::swap(c.cur, c.nxt);
        cur = c.cur.data();
    }
    c.rho = c.F;
}

// Hermitian eigenvalues via the real symmetric embedding [[A,-B],[B,A]]
// (each eigenvalue appears twice).
bool hermitian_eigs(int d, const cplx* m, std::vector<double>& out)
{
    const int n = 2 * d;
    std::vector<double> a(static_cast<size_t>(n) * n);
    for (int r = 0; r < d; ++r)
        for (int c = 0; c < d; ++c) {
            const cplx v = 0.5 * (m[r * d + c] + std::conj(m[c * d + r]));
            a[r * n + c] = v.real();
            a[(r + d) * n + (c + d)] = v.real();
            a[(r + d) * n + c] = v.imag();
            a[r * n + (c + d)] = -v.imag();
        }
    std::vector<double> e;
    if (!jacobi_eigenvalues(n, a, e)) return false;
    out.resize(d);
    for (int i = 0; i < d; ++i) out[i] = e[2 * i];
    return true;
}

}  // namespace

// ---------------------------------------------------------------------------
// C interface (ctypes; oracle/oracle.py)
// ---------------------------------------------------------------------------

extern "C" {

typedef struct or_csr {
    const int* ptr;
    const int* col;
    const double* val;  // interleaved re, im
    int nnz;
} or_csr;

typedef struct or_bath {
    double beta, gamma, zeta;
    int K;
    or_csr V;
} or_bath;

long long or_hierarchy_size(int modes, int maxDepth) { return hierarchy_size(modes, maxDepth); }

// rows: H*M ints, edges: H*2M ints (caller-sized by or_hierarchy_size)
int or_hierarchy_tables(int modes, int maxDepth, int* rows, int* edges)
{
    if (modes <= 0 || maxDepth <= 0) return 1;
    const long long H = hierarchy_size(modes, maxDepth);
    std::vector<int> r, e, prefix(modes, 0);
    r.reserve(static_cast<size_t>(H) * modes);
    emit_rows(0, modes, maxDepth, 0, prefix, r);
    if (static_cast<long long>(r.size()) != H * modes) return 2;
    build_edges(r, modes, H, e);
    std::memcpy(rows, r.data(), r.size() * sizeof(int));
    std::memcpy(edges, e.data(), e.size() * sizeof(int));
    return 0;
}

int or_psd(int K, double* poles, double* residues) { return psd_bose(K, poles, residues) ? 0 : 1; }

// bath coefficients in reference form: out[0..] = kxi.re, kxiCounter.im, kthetaC.im,
// kthetaA.re, then nu[0..K], then kphi.im[0..K-1]
int or_bath_coefficients(double beta, double gamma, double zeta, int K, double* out)
{
    Bath b{};
    b.beta = beta; b.gamma = gamma; b.zeta = zeta; b.K = K;
    if (!init_bath(b)) return 1;
    out[0] = b.kxi.real();
    out[1] = b.kxiCounter.imag();
    out[2] = b.kthetaC.imag();
    out[3] = b.kthetaA.real();
    for (int k = 0; k <= K; ++k) out[4 + k] = b.nu[k];
    for (int k = 0; k < K; ++k) out[5 + K + k] = b.kphi[k].imag();
    return 0;
}

void* or_create(int d, or_csr Hop, int nbaths, const or_bath* baths, int maxDepth)
{
    std::unique_ptr<Ctx> c(new (std::nothrow) Ctx());
    if (!c || d <= 0 || nbaths <= 0 || maxDepth <= 0) return nullptr;
    c->d = d;
    c->Hm = make_csr(d, Hop.ptr, Hop.col, Hop.val);
    c->Hmt = transpose(c->Hm);
    int offset = 0;
    for (int j = 0; j < nbaths; ++j) {
        Bath b{};
        b.beta = baths[j].beta; b.gamma = baths[j].gamma; b.zeta = baths[j].zeta; b.K = baths[j].K;
        b.V = make_csr(d, baths[j].V.ptr, baths[j].V.col, baths[j].V.val);
        b.Vt = transpose(b.V);
        b.offset = offset;
        if (!init_bath(b)) return nullptr;
        offset += b.K + 1;
        c->baths.push_back(std::move(b));
    }
    c->modes = offset;
    c->maxDepth = maxDepth;
    c->H = hierarchy_size(c->modes, maxDepth);
    c->rows.resize(static_cast<size_t>(c->H) * c->modes);
    c->edges.resize(static_cast<size_t>(c->H) * 2 * c->modes);
    if (or_hierarchy_tables(c->modes, maxDepth, c->rows.data(), c->edges.data()) != 0) return nullptr;
    const size_t n = static_cast<size_t>(c->H) * d * d;
    c->rho.assign(n, cplx(0.0));
    c->F.assign(n, cplx(0.0));
    c->cur.assign(n, cplx(0.0));
    c->nxt.assign(n, cplx(0.0));
    c->comm.assign(n * nbaths, cplx(0.0));
    // reference initial state: rho_0 = |d-1><d-1|, all other ADOs zero (initialize.cu:287-301)
    c->rho[static_cast<size_t>(d) * d - 1] = cplx(1.0, 0.0);
    return c.release();
}

void or_destroy(void* h) { delete static_cast<Ctx*>(h); }

long long or_size(void* h) { return static_cast<Ctx*>(h)->H; }
int or_modes(void* h) { return static_cast<Ctx*>(h)->modes; }

void or_get_state(void* h, double* out)
{
    Ctx* c = static_cast<Ctx*>(h);
    std::memcpy(out, c->rho.data(), c->rho.size() * sizeof(cplx));
}

void or_set_state(void* h, const double* in)
{
    Ctx* c = static_cast<Ctx*>(h);
    std::memcpy(c->rho.data(), in, c->rho.size() * sizeof(cplx));
}

void or_rhs(void* h, const double* in, double* out)
{
    Ctx* c = static_cast<Ctx*>(h);
    rhs(*c, reinterpret_cast<const cplx*>(in), reinterpret_cast<cplx*>(out));
}

// nsteps steps of the Taylor-4 integrator; if rho0_trace != NULL, writes rho_0
// (d*d complex) after every step; if energy_trace != NULL writes Tr(H rho_0).
void or_run(void* h, long long nsteps, double dt, int order, double* rho0_trace, double* energy_trace);

double or_energy(void* h)
{
    Ctx* c = static_cast<Ctx*>(h);
    const int d = c->d;
    // Tr(H rho_0) = sum_r sum_p H[r][col_p] rho_0[col_p][r]
    cplx s = 0.0;
    for (int r = 0; r < d; ++r)
        for (int p = c->Hm.ptr[r]; p < c->Hm.ptr[r + 1]; ++p)
            s += c->Hm.val[p] * c->rho[static_cast<size_t>(c->Hm.col[p]) * d + r];
    return s.real();
}

void or_run(void* h, long long nsteps, double dt, int order, double* rho0_trace, double* energy_trace)
{
    Ctx* c = static_cast<Ctx*>(h);
    const size_t slab = static_cast<size_t>(c->d) * c->d;
    for (long long s = 0; s < nsteps; ++s) {
        develop(*c, dt, order);
        if (rho0_trace) std::memcpy(rho0_trace + 2 * slab * s, c->rho.data(), slab * sizeof(cplx));
        if (energy_trace) energy_trace[s] = or_energy(h);
    }
}

// 0.5 * || A - B ||_1 for d x d Hermitian matrices (interleaved complex)
double or_trace_distance(int d, const double* a, const double* b)
{
    std::vector<cplx> m(static_cast<size_t>(d) * d);
    for (size_t i = 0; i < m.size(); ++i) m[i] = cplx(a[2 * i] - b[2 * i], a[2 * i + 1] - b[2 * i + 1]);
    std::vector<double> e;
    if (!hermitian_eigs(d, m.data(), e)) return -1.0;
    double s = 0.0;
    for (double x : e) s += std::fabs(x);
    return 0.5 * s;
}

int or_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// Threads of the following calls (n >= 1).
void or_set_threads(int n)
{
#ifdef _OPENMP
    if (n >= 1) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

}  // extern "C"
