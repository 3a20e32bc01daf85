// helix:: C++ API over the helix_b200 C ABI.
//
// Mirrors the reference's public behaviour (HELIX src/helix.cpp): the same
// validation order and StatusCode mapping, the one-active-Context lease
// (src/helix.cpp:73-104), exceptions mapped to InvalidRuntimeOption
// (src/helix.cpp:715-719, 766-769), RunResult packing with a row-major
// reduced density and times = {steps * dt} (src/helix.cpp:706-713).
// Execution is the fused sm_100a propagator behind <helix_b200.h>; this file
// calls no CUDA API itself.

#include <helix/helix.h>
#include <helix_b200.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <sstream>
#include <stdexcept>
#include <utility>

namespace helix {

const char* runtimeVersion() noexcept { return hx_version(); }

void Diagnostics::add(StatusCode code, std::string message)
{
    entries_.push_back({code, std::move(message)});
    status = RunStatus::Failed;
}

bool Diagnostics::ok() const noexcept { return entries_.empty(); }

bool Diagnostics::hasError(StatusCode code) const noexcept
{
    return std::any_of(entries_.begin(), entries_.end(), [code](const Diagnostic& d) { return d.code == code; });
}

std::string Diagnostics::message(StatusCode code) const
{
    for (const auto& d : entries_)
        if (d.code == code) return d.message;
    return {};
}

std::string Diagnostics::summary() const
{
    std::ostringstream out;
    for (std::size_t i = 0; i < entries_.size(); ++i) {
        if (i) out << "; ";
        out << entries_[i].message;
    }
    return out.str();
}

const std::vector<Diagnostic>& Diagnostics::entries() const noexcept { return entries_; }

namespace {

constexpr const char* kLifecycleMessage =
    "helix supports one active Context per process; destroy the current Context first";

std::atomic_bool& activeFlag()
{
    static std::atomic_bool flag{false};
    return flag;
}

class Lease {
public:
    Lease()
    {
        bool expected = false;
        if (!activeFlag().compare_exchange_strong(expected, true)) throw std::logic_error(kLifecycleMessage);
    }
    ~Lease() noexcept { activeFlag().store(false); }
    Lease(const Lease&) = delete;
    Lease& operator=(const Lease&) = delete;
};

void append(Diagnostics& to, const Diagnostics& from)
{
    for (const auto& d : from.entries()) to.add(d.code, d.message);
}

StatusCode status_from_hx(int rc)
{
    return static_cast<StatusCode>(rc - 1);
}

bool near(double a, double b) { return std::abs(a - b) <= 1.0e-12; }

// Compiled defaults of the reference (src/parameters.cu:11-31).
constexpr double kLegacyBeta = 3.0;
constexpr double kLegacyGamma = 1.0;
constexpr double kLegacyZeta = 0.01;
constexpr std::size_t kLegacyK = 2;
constexpr std::size_t kLegacyJMax = 3;

void validate_csr(const char* name, const SparseOperator& op, Diagnostics& d)
{
    auto add = [&](StatusCode c, const std::string& m) { d.add(c, std::string(name) + ": " + m); };
    if (op.rowOffsets.size() != op.rows + 1) {
        add(StatusCode::InvalidRowOffsets, "CSR rowOffsets size must equal rows + 1");
        return;
    }
    if (op.rowOffsets.front() != 0) add(StatusCode::InvalidRowOffsets, "CSR rowOffsets must start at zero");
    for (std::size_t i = 1; i < op.rowOffsets.size(); ++i)
        if (op.rowOffsets[i] < op.rowOffsets[i - 1]) {
            add(StatusCode::InvalidRowOffsets, "CSR rowOffsets must be monotonically nondecreasing");
            break;
        }
    if (op.columnIndices.size() != op.values.size())
        add(StatusCode::InvalidColumnValueSize, "CSR columnIndices and values must have identical sizes");
    if (op.rowOffsets.back() != op.columnIndices.size())
        add(StatusCode::InvalidRowOffsets, "CSR final row offset must equal the number of column entries");
    for (auto c : op.columnIndices)
        if (c >= op.cols) {
            add(StatusCode::InvalidColumnIndex, "CSR column index is outside operator dimensions");
            break;
        }
}

Diagnostics validate_context_options(const ContextOptions& o)
{
    Diagnostics d;
    if (o.backend == Backend::CpuReference)
        d.add(StatusCode::UnsupportedBackend, "Backend::CpuReference has no execution path; the B200 propagator runs on CUDA");
    if (o.allowConcurrentContexts) d.add(StatusCode::ConcurrentContextUnsupported, kLifecycleMessage);
    if (o.device < 0) d.add(StatusCode::InvalidRuntimeOption, "CUDA device index must be non-negative");
    if (o.integrationOrder <= 0 || o.integrationOrder > 8)
        d.add(StatusCode::InvalidRuntimeOption, "integrationOrder must be in 1..8");
    if (!(o.timeStep > 0.0)) d.add(StatusCode::InvalidRuntimeOption, "timeStep must be positive");
    return d;
}

Diagnostics validate_solver_options(const SolverOptions& o)
{
    Diagnostics d;
    if (o.timeStep < 0.0) d.add(StatusCode::InvalidRuntimeOption, "SolverOptions::timeStep must be non-negative");
    return d;
}

// The executable structure: H = diag(E) + sum_i h_i sx_i (real), each coupling
// V_j = diag(v_j) + sum_i w_ji sx_i (real).
struct LoweredCsr {
    std::vector<int32_t> ptr, col;
    std::vector<double> val;  // re, im interleaved
};

struct Lowered {
    uint32_t dim = 0;
    std::vector<double> hdiag, hflip;
    std::vector<std::vector<double>> vdiag, vflip;
    // operators outside the diagonal-plus-flip structure, passed on in CSR form
    bool h_is_csr = false;
    LoweredCsr hcsr;
    std::vector<LoweredCsr> vcsr;  // per coupling; empty ptr = diagonal-plus-flip form
};

LoweredCsr csr_of(const SparseOperator& op)
{
    LoweredCsr o;
    o.ptr.reserve(op.rowOffsets.size());
    for (std::size_t x : op.rowOffsets) o.ptr.push_back(static_cast<int32_t>(x));
    for (std::size_t c : op.columnIndices) o.col.push_back(static_cast<int32_t>(c));
    for (const std::complex<double>& v : op.values) {
        o.val.push_back(v.real());
        o.val.push_back(v.imag());
    }
    return o;
}

// Split a real CSR operator into its diagonal and per-spin flip weights;
// false if it has any other structure.
bool split_flip_operator(const SparseOperator& op, std::size_t d, int n, std::vector<double>& diag,
                         std::vector<double>& flip, std::string& why, const char* name)
{
    diag.assign(d, 0.0);
    flip.assign(n, 0.0);
    std::vector<int> count(n, 0);
    for (std::size_t r = 0; r < d; ++r)
        for (std::size_t p = op.rowOffsets[r]; p < op.rowOffsets[r + 1]; ++p) {
            const std::size_t c = op.columnIndices[p];
            const std::complex<double> v = op.values[p];
            if (v.imag() != 0.0) {
                why = std::string(name) + ": complex entries are outside the supported structure";
                return false;
            }
            if (c == r) {
                diag[r] += v.real();
                continue;
            }
            const std::size_t x = r ^ c;
            if ((x & (x - 1)) != 0) {
                why = std::string(name) + ": off-diagonal entries must be single-spin flips";
                return false;
            }
            int bit = 0;
            while ((std::size_t(1) << bit) != x) ++bit;
            if (count[bit] > 0 && flip[bit] != v.real()) {
                why = std::string(name) + ": the flip of one spin must carry one value";
                return false;
            }
            flip[bit] = v.real();
            ++count[bit];
        }
    for (int b = 0; b < n; ++b)
        if (count[b] != 0 && static_cast<std::size_t>(count[b]) != d) {
            why = std::string(name) + ": a spin flip must act on every basis state";
            return false;
        }
    return true;
}

// The reference's compiled spin-glass model (src/parameters.cu:11-18,
// src/initialize.cu:95-157, initialize_detail.h:38-157): d = 1024, diagonal H
// from the nearest-neighbour chain (J = 0.6) with projections +-1/2, one
// collective V = sum_i s_z(i) + sum_{i : 2^i in the sparse flip masks} sx(i)
// (mask 512 is absent from those masks).
Lowered legacy_model()
{
    const int n = 10;
    const std::size_t d = std::size_t(1) << n;
    Lowered L;
    L.dim = static_cast<uint32_t>(d);
    L.hdiag.assign(d, 0.0);
    L.hflip.assign(n, 0.0);
    std::vector<double> v(d, 0.0), w(n, 0.0);
    for (std::size_t state = 0; state < d; ++state) {
        double p[n];
        double total = 0.0;
        for (int s = 0; s < n; ++s) {
            p[s] = ((state >> s) & 1) ? 0.5 : -0.5;
            total += p[s];
        }
        v[state] = total;
        for (int j = 0; j < n; ++j)
            for (int k = 0; k < j; ++k)
                if (j - k == 1) total += 0.6 * p[j] * p[k];
        L.hdiag[state] = total;
    }
    for (int i = 0; i < n; ++i) w[i] = ((1 << i) <= 256) ? 1.0 : 0.0;
    L.vdiag.push_back(v);
    L.vflip.push_back(w);
    return L;
}

bool lower_system(const System& s, Lowered& out, std::string& why)
{
    const SparseOperator& H = s.hamiltonian;
    const std::size_t d = H.rows;
    if (d < 2 || (d & (d - 1)) != 0 || H.cols != d) {
        why = "Hilbert dimension must be a power of two >= 2";
        return false;
    }
    int n = 0;
    while ((std::size_t(1) << n) < d) ++n;
    out.dim = static_cast<uint32_t>(d);
    // H as diagonal plus uniform single-spin flips (the fused kernels), else in CSR
    auto flip_form = [&](std::string& why) {
    out.hdiag.assign(d, 0.0);
    out.hflip.assign(n, 0.0);
    std::vector<bool> seen(n, false);
    for (std::size_t r = 0; r < d; ++r)
        for (std::size_t p = H.rowOffsets[r]; p < H.rowOffsets[r + 1]; ++p) {
            const std::size_t c = H.columnIndices[p];
            const std::complex<double> v = H.values[p];
            if (v.imag() != 0.0) {
                why = "complex Hamiltonian entries are outside the fused path";
                return false;
            }
            if (c == r) {
                out.hdiag[r] += v.real();
                continue;
            }
            const std::size_t x = r ^ c;
            if ((x & (x - 1)) != 0) {
                why = "Hamiltonian off-diagonals must be single-spin flips";
                return false;
            }
            int bit = 0;
            while ((std::size_t(1) << bit) != x) ++bit;
            if (!seen[bit]) {
                out.hflip[bit] = v.real();
                seen[bit] = true;
            } else if (out.hflip[bit] != v.real()) {
                why = "transverse field must be uniform over the flips of one spin";
                return false;
            }
        }
    for (int b = 0; b < n; ++b)
        if (seen[b]) {
            // every row must carry the flip of spin b with the same value
            for (std::size_t r = 0; r < d; ++r) {
                bool found = false;
                for (std::size_t p = H.rowOffsets[r]; p < H.rowOffsets[r + 1]; ++p)
                    if (H.columnIndices[p] == (r ^ (std::size_t(1) << b))) found = true;
                if (!found) {
                    why = "transverse field must act on every basis state";
                    return false;
                }
            }
        }
    return true;
    };
    std::string why_h;
    out.h_is_csr = !flip_form(why_h);
    if (out.h_is_csr) out.hcsr = csr_of(H);
    out.vdiag.clear();
    out.vflip.clear();
    out.vcsr.clear();
    for (std::size_t k = 0; k < s.couplings.size(); ++k) {
        std::vector<double> v, w;
        const std::string name = "coupling[" + std::to_string(k) + "]";
        std::string why_v;
        if (split_flip_operator(s.couplings[k], d, n, v, w, why_v, name.c_str())) {
            out.vcsr.emplace_back();
        } else {
            v.assign(d, 0.0);
            w.assign(n, 0.0);
            out.vcsr.push_back(csr_of(s.couplings[k]));
        }
        out.vdiag.push_back(std::move(v));
        out.vflip.push_back(std::move(w));
    }
    if (out.vdiag.empty()) {
        why = "at least one coupling operator is required";
        return false;
    }
    return true;
}

}  // namespace

// ---------------------------------------------------------------------------
// Bath / HierarchySpec / System
// ---------------------------------------------------------------------------

Bath Bath::drude_lorentz_pade()
{
    Bath b;
    b.inverseTemperature = kLegacyBeta;
    b.damping = kLegacyGamma;
    b.couplingStrength = kLegacyZeta;
    b.padeTerms = kLegacyK;
    return b;
}

Bath Bath::drude_lorentz(double lambda, double gamma, double temperature, std::size_t padeTerms)
{
    Bath b;
    b.inverseTemperature = 1.0 / temperature;
    b.damping = gamma;
    b.couplingStrength = 2.0 * lambda / gamma;
    b.padeTerms = padeTerms;
    return b;
}

Bath Bath::user_exponents(std::vector<std::complex<double>> coefficients, std::vector<std::complex<double>> rates)
{
    Bath b;
    b.kind = Kind::UserExponents;
    b.exponentCoefficients = std::move(coefficients);
    b.exponentRates = std::move(rates);
    return b;
}

Diagnostics Bath::validate_supported() const
{
    Diagnostics d;
    if (kind == Kind::UserExponents) {
        if (exponentCoefficients.empty())
            d.add(StatusCode::BathExponentsInvalid, "User-provided bath exponent coefficients must not be empty");
        if (exponentRates.empty())
            d.add(StatusCode::BathExponentsInvalid, "User-provided bath exponent rates must not be empty");
        if (exponentCoefficients.size() != exponentRates.size())
            d.add(StatusCode::BathExponentsInvalid,
                  "User-provided bath exponent coefficients and rates must have equal sizes");
        for (std::size_t i = 0; i < exponentRates.size(); ++i)
            if (exponentRates[i].real() <= 0.0)
                d.add(StatusCode::BathExponentsInvalid,
                      "User-provided bath exponent rate " + std::to_string(i) + " must have a positive real part");
        if (d.ok())
            d.add(StatusCode::UnsupportedBath, "User-provided bath exponent sets are validation-only");
        return d;
    }
    if (!(inverseTemperature > 0.0)) d.add(StatusCode::UnsupportedBath, "inverse temperature must be positive");
    if (!(damping > 0.0)) d.add(StatusCode::UnsupportedBath, "bath damping must be positive");
    if (!std::isfinite(couplingStrength)) d.add(StatusCode::UnsupportedBath, "coupling strength must be finite");
    if (padeTerms > 32) d.add(StatusCode::UnsupportedBath, "at most 32 Pade terms are supported");
    if (!frequencies.empty() || !residues.empty()) {
        // explicit values must agree with the Pade decomposition the solver uses
        std::vector<double> poles(padeTerms), res(padeTerms);
        if (padeTerms > 0 && hx_psd(static_cast<uint32_t>(padeTerms), poles.data(), res.data()) != HX_OK) {
            d.add(StatusCode::UnsupportedBath, "Pade decomposition failed");
            return d;
        }
        if (!frequencies.empty()) {
            bool ok = frequencies.size() == padeTerms + 1 && near(frequencies[0], damping);
            for (std::size_t k = 1; ok && k <= padeTerms; ++k)
                ok = near(frequencies[k], poles[k - 1] / inverseTemperature);
            if (!ok) d.add(StatusCode::UnsupportedBath, "bath frequencies must match the Drude-Lorentz/Pade modes");
        }
        if (!residues.empty()) {
            bool ok = residues.size() == padeTerms;
            for (std::size_t k = 0; ok && k < padeTerms; ++k) ok = near(residues[k].real(), res[k]) && residues[k].imag() == 0.0;
            if (!ok) d.add(StatusCode::UnsupportedBath, "Pade residues must match the [K-1/K] decomposition");
        }
    }
    return d;
}

HierarchySpec HierarchySpec::compiled_default(Bath bath)
{
    HierarchySpec h;
    h.maxDepth = kLegacyJMax;
    h.exponentialTerms = kLegacyK + 1;
    h.baths.push_back(std::move(bath));
    return h;
}

Diagnostics HierarchySpec::validate_supported() const
{
    Diagnostics d;
    if (maxDepth < 1) d.add(StatusCode::UnsupportedHierarchy, "maxDepth must be at least 1");
    if (baths.empty()) {
        d.add(StatusCode::UnsupportedHierarchy, "at least one bath is required");
        return d;
    }
    for (const auto& b : baths) {
        if (exponentialTerms != 0 && b.kind == Bath::Kind::DrudeLorentzPade && exponentialTerms != b.padeTerms + 1)
            d.add(StatusCode::UnsupportedHierarchy, "exponentialTerms must equal padeTerms + 1 for every bath");
        for (const auto& e : b.validate_supported().entries())
            d.add(e.code, std::string("hierarchy bath: ") + e.message);
    }
    return d;
}

bool System::valid() const noexcept { return diagnostics.ok(); }

System System::from_sparse(SparseOperator hamiltonian, std::vector<SparseOperator> couplings)
{
    System s;
    s.kind = SystemKind::Sparse;
    s.hamiltonian = std::move(hamiltonian);
    s.couplings = std::move(couplings);
    validate_csr("hamiltonian", s.hamiltonian, s.diagnostics);
    if (s.hamiltonian.rows != s.hamiltonian.cols)
        s.diagnostics.add(StatusCode::InvalidDimension, "hamiltonian: system operator must be square");
    for (std::size_t i = 0; i < s.couplings.size(); ++i) {
        const std::string name = "coupling[" + std::to_string(i) + "]";
        validate_csr(name.c_str(), s.couplings[i], s.diagnostics);
        if (s.couplings[i].rows != s.hamiltonian.rows || s.couplings[i].cols != s.hamiltonian.cols)
            s.diagnostics.add(StatusCode::InvalidCouplingDimension,
                              name + ": coupling operator dimensions must match the system operator");
    }
    return s;
}

bool RunResult::ok() const noexcept { return diagnostics.ok(); }

// ---------------------------------------------------------------------------
// Context: device selection + lease; owns the hx_ctx of the bound problem.
// ---------------------------------------------------------------------------

class Context::Impl {
public:
    explicit Impl(ContextOptions options) : options_(options)
    {
        diagnostics_ = validate_context_options(options_);
        if (!diagnostics_.ok()) throw std::invalid_argument(diagnostics_.summary());
        lease_ = std::make_unique<Lease>();
        if (hx_select_device(options_.device) != HX_OK)
            throw std::runtime_error(std::string("Failed to select CUDA device: ") + hx_last_error());
    }
    ~Impl() noexcept { destroy(); }

    void bind(const Lowered& sys, const HierarchySpec& hier, double dt)
    {
        if (ctx_) return;
        std::vector<hx_bath> baths(sys.vdiag.size());
        std::vector<hx_csr> vcsr(sys.vdiag.size());
        hx_csr hcsr{};
        for (std::size_t j = 0; j < baths.size(); ++j) {
            const Bath& b = hier.baths.size() == 1 ? hier.baths[0] : hier.baths[j];
            baths[j].inverse_temperature = b.inverseTemperature;
            baths[j].damping = b.damping;
            baths[j].coupling_strength = b.couplingStrength;
            baths[j].pade_terms = static_cast<uint32_t>(b.padeTerms);
            baths[j].coupling_diag = sys.vdiag[j].data();
            baths[j].coupling_flip = sys.vflip.size() > j ? sys.vflip[j].data() : nullptr;
            if (sys.vcsr.size() > j && !sys.vcsr[j].ptr.empty()) {
                const LoweredCsr& o = sys.vcsr[j];
                vcsr[j] = hx_csr{o.ptr.data(), o.col.data(), o.val.data(), static_cast<uint32_t>(o.col.size())};
                baths[j].coupling_csr = &vcsr[j];
            }
        }
        hx_problem p{};
        p.dim = sys.dim;
        p.h_diag = sys.hdiag.data();
        p.h_flip = sys.hflip.data();
        if (sys.h_is_csr) {
            hcsr = hx_csr{sys.hcsr.ptr.data(), sys.hcsr.col.data(), sys.hcsr.val.data(),
                          static_cast<uint32_t>(sys.hcsr.col.size())};
            p.h_csr = &hcsr;
        }
        p.n_baths = static_cast<uint32_t>(baths.size());
        p.baths = baths.data();
        p.max_depth = static_cast<uint32_t>(hier.maxDepth);
        p.time_step = dt;
        p.integration_order = static_cast<uint32_t>(options_.integrationOrder);
        // Single-precision requests take the mixed path (complex64 hierarchy,
        // tier-0 ADO and observables in FP64) where it exists (128 <= d <= 1024,
        // diagonal couplings, at least two tiers below the top), else FP64.
        int rc = HX_ERR_UNSUPPORTED_PRECISION;
        mixed_ = false;
        if (options_.precision == Precision::Single) {
            p.precision = HX_PRECISION_MIXED;
            rc = hx_ctx_create(&p, &ctx_);
            mixed_ = rc == HX_OK;
            // an H given as CSR with many entries per row (16 or more on average) and outside the
            // diagonal-plus-flip form: single precision with the commutator on the tensor cores
            if (rc == HX_ERR_UNSUPPORTED_PRECISION && sys.h_is_csr && sys.hcsr.col.size() >= 16 * std::size_t(sys.dim)) {
                p.flags = HX_FLAG_FULL_STATE | HX_FLAG_DENSE_H;
                rc = hx_ctx_create(&p, &ctx_);
                mixed_ = rc == HX_OK;
                if (rc != HX_OK) {
                    p.flags = 0;
                    rc = HX_ERR_UNSUPPORTED_PRECISION;
                }
            }
        }
        if (rc == HX_ERR_UNSUPPORTED_PRECISION) {
            p.precision = HX_PRECISION_DOUBLE;
            rc = hx_ctx_create(&p, &ctx_);
        }
        if (rc != HX_OK) {
            lastCode_ = rc;
            throw std::runtime_error(hx_last_error());
        }
        dt_ = dt;
        dim_ = sys.dim;
    }

    void run_steps(std::size_t steps)
    {
        require();
        check(hx_ctx_step(ctx_, steps));
        check(hx_ctx_sync(ctx_));
    }

    void run_trace(std::size_t steps, std::vector<std::complex<double>>* rho, std::vector<double>* energy)
    {
        require();
        if (rho) rho->assign(steps * dim_ * dim_, {});
        if (energy) energy->assign(steps, 0.0);
        check(hx_ctx_step_trace(ctx_, steps, rho ? reinterpret_cast<double*>(rho->data()) : nullptr,
                                energy ? energy->data() : nullptr));
    }

    std::vector<std::complex<double>> reduced_density() const
    {
        require();
        std::vector<std::complex<double>> out(static_cast<std::size_t>(dim_) * dim_);
        check(hx_ctx_read_rho0(ctx_, reinterpret_cast<double*>(out.data()), 2 * out.size()));
        return out;
    }

    double energy() const
    {
        require();
        double e = 0, tr = 0, ti = 0;
        check(hx_ctx_observables(ctx_, &e, &tr, &ti));
        return e;
    }

    std::size_t hierarchy_size() const
    {
        hx_info info{};
        if (ctx_ && hx_ctx_info(ctx_, &info) == HX_OK) return static_cast<std::size_t>(info.hierarchy_size);
        return 0;
    }

    bool active() const noexcept { return ctx_ != nullptr; }

    void destroy() noexcept
    {
        if (ctx_) hx_ctx_destroy(ctx_);
        ctx_ = nullptr;
        lease_.reset();
    }

    const Diagnostics& diagnostics() const noexcept { return diagnostics_; }
    const ContextOptions& options() const noexcept { return options_; }
    double dt() const noexcept { return dt_; }
    uint32_t dim() const noexcept { return dim_; }
    bool mixed() const noexcept { return mixed_; }
    int lastCode() const noexcept { return lastCode_; }

private:
    void require() const
    {
        if (!ctx_) throw std::logic_error("Context has no bound problem");
    }
    void check(int rc) const
    {
        if (rc != HX_OK) {
            lastCode_ = rc;
            throw std::runtime_error(hx_last_error());
        }
    }

    ContextOptions options_;
    Diagnostics diagnostics_;
    std::unique_ptr<Lease> lease_;
    hx_ctx* ctx_ = nullptr;
    double dt_ = 0.0;
    uint32_t dim_ = 0;
    bool mixed_ = false;
    mutable int lastCode_ = HX_OK;
};

Context::Context(ContextOptions options) : impl_(std::make_unique<Impl>(options)) {}
Context::~Context() noexcept = default;
Context::Context(Context&&) noexcept = default;
Context& Context::operator=(Context&&) noexcept = default;

const Diagnostics& Context::diagnostics() const noexcept
{
    static const Diagnostics empty;
    return impl_ ? impl_->diagnostics() : empty;
}

bool Context::active() const noexcept { return impl_ && impl_->active(); }

void Context::run_steps(std::size_t steps)
{
    if (!impl_) throw std::logic_error("Cannot run a moved-from Context");
    impl_->run_steps(steps);
}

std::vector<std::complex<double>> Context::reduced_density() const
{
    if (!impl_) throw std::logic_error("Cannot read reduced density from a moved-from Context");
    return impl_->reduced_density();
}

void Context::destroy() noexcept
{
    if (impl_) impl_->destroy();
}

// ---------------------------------------------------------------------------
// HEOMSolver
// ---------------------------------------------------------------------------

HEOMSolver::HEOMSolver() = default;
HEOMSolver::HEOMSolver(ContextOptions options) : options_(options) {}
HEOMSolver::HEOMSolver(Context& context, System system, Bath bath, HierarchySpec hierarchy, SolverOptions options)
    : context_(&context), system_(std::move(system)), bath_(std::move(bath)), hierarchy_(std::move(hierarchy)),
      solverOptions_(options)
{
}

Diagnostics HEOMSolver::validate_options() const { return validate_context_options(options_); }

namespace {

Diagnostics validate_problem(const System& system, const HierarchySpec& hierarchy, const SolverOptions& options)
{
    Diagnostics d;
    append(d, system.diagnostics);
    append(d, hierarchy.validate_supported());
    append(d, validate_solver_options(options));
    if (system.kind == SystemKind::LegacySpinGlass) {
        if (hierarchy.baths.size() > 1)
            d.add(StatusCode::UnsupportedHierarchy, "the legacy spin-glass model has one collective bath");
    } else if (system.kind == SystemKind::Dense) {
        d.add(StatusCode::UnsupportedSystemKind, "dense systems are not executed; use System::from_sparse");
    } else if (d.ok()) {
        if (system.couplings.empty())
            d.add(StatusCode::UnsupportedExecution, "at least one coupling operator is required");
        else if (hierarchy.baths.size() != 1 && hierarchy.baths.size() != system.couplings.size())
            d.add(StatusCode::UnsupportedHierarchy,
                  "HierarchySpec::baths needs one bath per coupling operator (or one bath shared by all)");
    }
    return d;
}

}  // namespace

RunResult HEOMSolver::run_steps(std::size_t steps)
{
    RunResult result;
    if (!context_ || !context_->impl_) {
        result.diagnostics.add(StatusCode::InvalidRuntimeOption, "HEOMSolver::run_steps requires a Context-bound solver");
        return result;
    }
    HierarchySpec hier = hierarchy_;
    if (hier.baths.empty()) hier.baths.push_back(bath_);
    result.diagnostics = validate_problem(system_, hier, solverOptions_);
    if (!result.diagnostics.ok()) return result;
    Context::Impl& impl = *context_->impl_;
    const ContextOptions& copt = impl.options();
    try {
        Lowered low;
        std::string why;
        if (system_.kind == SystemKind::LegacySpinGlass) {
            low = legacy_model();
        } else if (!lower_system(system_, low, why)) {
            result.diagnostics.add(StatusCode::UnsupportedExecution, why);
            return result;
        }
        const double dt = solverOptions_.timeStep > 0.0 ? solverOptions_.timeStep : copt.timeStep;
        impl.bind(low, hier, dt);
        const std::size_t d = low.dim;
        const ResultMode mode = solverOptions_.resultMode;
        if (mode == ResultMode::FinalState) {
            impl.run_steps(steps);
            result.reduced_density = impl.reduced_density();
            result.reduced_density_shape = {1, d, d, MatrixStorageOrder::RowMajor};
            result.times.push_back(static_cast<double>(steps) * dt);
            result.energies.push_back(impl.energy());
        } else {
            std::vector<std::complex<double>> rho;
            impl.run_trace(steps, mode == ResultMode::Trajectory ? &rho : nullptr, &result.energies);
            for (std::size_t s = 1; s <= steps; ++s) result.times.push_back(static_cast<double>(s) * dt);
            if (mode == ResultMode::Trajectory) {
                result.reduced_density = std::move(rho);
                result.reduced_density_shape = {steps, d, d, MatrixStorageOrder::RowMajor};
            } else {
                result.reduced_density = impl.reduced_density();
                result.reduced_density_shape = {1, d, d, MatrixStorageOrder::RowMajor};
            }
        }
        result.diagnostics.backend = copt.backend;
        result.diagnostics.precision = impl.mixed() ? Precision::Single : Precision::Double;
        if (impl.mixed())
            result.diagnostics.warnings.push_back(
                "Precision::Single: hierarchy in complex64, tier-0 ADO and observables in double precision");
        else if (copt.precision == Precision::Single)
            result.diagnostics.warnings.push_back("Precision::Single requested; propagated in double precision");
        result.diagnostics.hilbertSize = d;
        result.diagnostics.hierarchySize = impl.hierarchy_size();
        result.diagnostics.steps = steps;
        result.diagnostics.timeStep = dt;
        result.diagnostics.integrationOrder = copt.integrationOrder;
        result.diagnostics.status = RunStatus::Success;
    } catch (const std::exception& e) {
        const int code = impl.lastCode();
        result.diagnostics.add(code > 0 ? status_from_hx(code) : StatusCode::InvalidRuntimeOption, e.what());
    }
    return result;
}

RunResult HEOMSolver::run(const System& system, const HierarchySpec& hierarchy, const SolverOptions& options) const
{
    RunResult result;
    result.diagnostics = validate_options();
    append(result.diagnostics, validate_problem(system, hierarchy, options));
    if (!result.diagnostics.ok()) return result;
    try {
        ContextOptions copt = options_;
        if (options.timeStep > 0.0) copt.timeStep = options.timeStep;
        Context context(copt);
        const Bath bath = hierarchy.baths.empty() ? Bath::drude_lorentz_pade() : hierarchy.baths.front();
        HEOMSolver bound(context, system, bath, hierarchy, options);
        result = bound.run_steps(options.steps);
        context.destroy();
    } catch (const std::exception& e) {
        result.diagnostics.add(StatusCode::InvalidRuntimeOption, e.what());
    }
    return result;
}

// ---------------------------------------------------------------------------
// examples
// ---------------------------------------------------------------------------

namespace examples {

System legacy_spin_glass_system()
{
    System s;
    s.kind = SystemKind::LegacySpinGlass;
    return s;
}

System transverse_ising_spin_glass(std::size_t spins, std::uint64_t seed, double h)
{
    const std::size_t d = std::size_t(1) << spins;
    std::vector<double> J(spins * spins, 0.0);
    hx_seeded_couplings(static_cast<uint32_t>(spins), seed, J.data());
    SparseOperator H;
    H.rows = H.cols = d;
    H.rowOffsets.push_back(0);
    for (std::size_t r = 0; r < d; ++r) {
        double e = 0.0;
        for (std::size_t i = 0; i < spins; ++i)
            for (std::size_t j = i + 1; j < spins; ++j) {
                const double si = ((r >> i) & 1) ? 1.0 : -1.0;
                const double sj = ((r >> j) & 1) ? 1.0 : -1.0;
                e += J[i * spins + j] * si * sj;
            }
        std::vector<std::pair<std::size_t, double>> row{{r, e}};
        if (h != 0.0)
            for (std::size_t i = 0; i < spins; ++i) row.push_back({r ^ (std::size_t(1) << i), h});
        std::sort(row.begin(), row.end());
        for (const auto& [c, v] : row) {
            H.columnIndices.push_back(c);
            H.values.push_back({v, 0.0});
        }
        H.rowOffsets.push_back(H.columnIndices.size());
    }
    std::vector<SparseOperator> V;
    for (std::size_t i = 0; i < spins; ++i) {
        SparseOperator op;
        op.rows = op.cols = d;
        for (std::size_t r = 0; r <= d; ++r) op.rowOffsets.push_back(r);
        for (std::size_t r = 0; r < d; ++r) {
            op.columnIndices.push_back(r);
            op.values.push_back({((r >> i) & 1) ? 1.0 : -1.0, 0.0});
        }
        V.push_back(std::move(op));
    }
    return System::from_sparse(std::move(H), std::move(V));
}

HierarchySpec spin_glass_hierarchy(std::size_t spins, double lambda, double gamma, double temperature,
                                   std::size_t padeTerms, std::size_t depth)
{
    HierarchySpec h;
    h.maxDepth = depth + 1;
    h.exponentialTerms = padeTerms + 1;
    for (std::size_t i = 0; i < spins; ++i) h.baths.push_back(Bath::drude_lorentz(lambda, gamma, temperature, padeTerms));
    return h;
}

}  // namespace examples

}  // namespace helix
