#pragma once
// helix:: public C++ API of helix_b200.
//
// Same shape and semantics as the reference's public header
// (HELIX include/helix/types.h:9-209): the same enums (append-only), value
// types, Diagnostics contract and HEOMSolver entry points, so code written
// against the reference compiles and runs unchanged.  Execution goes through
// the C ABI in <helix_b200.h> (libhelix_b200.so, sm_100a kernels).
//
// Differences from the reference (all additive):
//  - System::from_sparse systems execute when H = diagonal + single-spin
//    transverse flips and every coupling operator is diagonal; each coupling
//    operator has its own bath in HierarchySpec::baths (same order).
//  - Precision::Double executes; Precision::Single requests run in double
//    precision and say so in Diagnostics::warnings.
//  - ResultMode::ObservableTrace / Trajectory execute (per-step energy and,
//    for Trajectory, per-step reduced density).
//  - RunResult::energies (appended field): Tr(H rho_0) after each step for
//    the trace modes, or at the end for FinalState.

#include <complex>
#include <cstddef>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

namespace helix {

enum class Backend {
    LegacyCudaSparse,
    CudaSparse,
    CpuReference
};

enum class Precision {
    Single,
    Double
};

enum class SystemKind {
    Sparse,
    Dense,
    LegacySpinGlass
};

enum class ResultMode {
    FinalState,
    ObservableTrace,
    Trajectory
};

enum class MatrixStorageOrder {
    RowMajor
};

enum class RunStatus {
    NotStarted,
    Success,
    Failed
};

// Append-only: values never removed, reordered or reused.
enum class StatusCode {
    InvalidDimension,
    InvalidRowOffsets,
    InvalidColumnValueSize,
    InvalidColumnIndex,
    InvalidCouplingDimension,
    InvalidRuntimeOption,
    UnsupportedPrecision,
    UnsupportedBackend,
    UnsupportedSystemKind,
    UnsupportedExecution,
    UnsupportedBath,
    UnsupportedHierarchy,
    ConcurrentContextUnsupported,
    BathExponentsInvalid,
    CudaFailure,
    OutOfMemory,
    NonFiniteState,
    DeviceWaitTimeout
};

struct Diagnostic {
    StatusCode code;
    std::string message;
};

class Diagnostics {
public:
    Backend backend = Backend::LegacyCudaSparse;
    Precision precision = Precision::Single;
    std::size_t hilbertSize = 0;
    std::size_t hierarchySize = 0;
    std::size_t steps = 0;
    double timeStep = 0.0;
    int integrationOrder = 0;
    RunStatus status = RunStatus::NotStarted;
    std::vector<std::string> warnings;

    void add(StatusCode code, std::string message);
    bool ok() const noexcept;
    bool hasError(StatusCode code) const noexcept;
    std::string message(StatusCode code) const;
    std::string summary() const;
    const std::vector<Diagnostic>& entries() const noexcept;

private:
    std::vector<Diagnostic> entries_;
};

struct ContextOptions {
    Backend backend = Backend::LegacyCudaSparse;
    Precision precision = Precision::Single;
    bool allowConcurrentContexts = false;
    int device = 0;
    int integrationOrder = 4;
    double timeStep = 0.1;
};

struct SparseOperator {
    std::size_t rows = 0;
    std::size_t cols = 0;
    std::vector<std::size_t> rowOffsets;
    std::vector<std::size_t> columnIndices;
    std::vector<std::complex<double>> values;
};

struct Bath {
    enum class Kind {
        DrudeLorentzPade,
        UserExponents
    };

    Kind kind = Kind::DrudeLorentzPade;
    double inverseTemperature = 0.0;  // beta
    double damping = 0.0;             // gamma
    double couplingStrength = 0.0;    // zeta (reference units): lambda = zeta * gamma / 2
    std::size_t padeTerms = 0;        // K
    std::vector<std::complex<double>> residues;
    std::vector<double> frequencies;
    std::vector<std::complex<double>> exponentCoefficients;
    std::vector<std::complex<double>> exponentRates;

    // The reference's compiled bath: beta = 3, gamma = 1, zeta = 0.01, K = 2.
    static Bath drude_lorentz_pade();
    // Drude-Lorentz bath from the reorganisation energy lambda and temperature.
    static Bath drude_lorentz(double lambda, double gamma, double temperature, std::size_t padeTerms);
    static Bath user_exponents(std::vector<std::complex<double>> coefficients,
                               std::vector<std::complex<double>> rates);
    Diagnostics validate_supported() const;
};

struct HierarchySpec {
    std::size_t maxDepth = 0;          // exclusive bound on sum(n): depth L <=> maxDepth = L + 1
    std::size_t exponentialTerms = 0;  // per bath: padeTerms + 1
    std::vector<Bath> baths;

    static HierarchySpec compiled_default(Bath bath = Bath::drude_lorentz_pade());
    Diagnostics validate_supported() const;
};

struct SolverOptions {
    std::size_t steps = 0;
    double timeStep = 0.0;
    ResultMode resultMode = ResultMode::FinalState;
};

struct System {
    SystemKind kind = SystemKind::Sparse;
    SparseOperator hamiltonian;
    std::vector<SparseOperator> couplings;
    Diagnostics diagnostics;

    bool valid() const noexcept;
    static System from_sparse(SparseOperator hamiltonian, std::vector<SparseOperator> couplings = {});
};

struct ReducedDensityShape {
    std::size_t count = 0;
    std::size_t rows = 0;
    std::size_t cols = 0;
    MatrixStorageOrder storageOrder = MatrixStorageOrder::RowMajor;
};

struct RunResult {
    std::vector<double> times;
    std::vector<std::complex<double>> reduced_density;
    ReducedDensityShape reduced_density_shape;
    Diagnostics diagnostics;
    std::vector<double> energies;  // appended field

    bool ok() const noexcept;
};

class Context {
public:
    explicit Context(ContextOptions options = {});
    ~Context() noexcept;

    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    Context(Context&&) noexcept;
    Context& operator=(Context&&) noexcept;

    const Diagnostics& diagnostics() const noexcept;
    bool active() const noexcept;
    void run_steps(std::size_t steps);
    std::vector<std::complex<double>> reduced_density() const;
    void destroy() noexcept;

    class Impl;

private:
    std::unique_ptr<Impl> impl_;
    friend class HEOMSolver;
};

class HEOMSolver {
public:
    HEOMSolver();
    explicit HEOMSolver(ContextOptions options);
    HEOMSolver(Context& context, System system, Bath bath, HierarchySpec hierarchy, SolverOptions options = {});

    Diagnostics validate_options() const;
    RunResult run_steps(std::size_t steps);
    RunResult run(const System& system, const HierarchySpec& hierarchy, const SolverOptions& options) const;

private:
    ContextOptions options_;
    Context* context_ = nullptr;
    System system_;
    Bath bath_;
    HierarchySpec hierarchy_;
    SolverOptions solverOptions_;
};

const char* runtimeVersion() noexcept;

}  // namespace helix
