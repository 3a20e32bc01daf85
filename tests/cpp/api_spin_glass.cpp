// Drives the helix:: C++ API the way a reference user does
// (helix::HEOMSolver(options).run(system, hierarchy, solverOptions)) and
// prints the result as JSON for tests/test_cpp_api.py to check against the
// FP64 oracle.  Usage: api_spin_glass <spins> <seed> <h> <depth> <K> <steps> <dt> <mode>
//   mode: final | trace | trajectory | single | legacy | sparse-bad | sparse-general | dense-single
#include <helix/helix.h>

#include <algorithm>
#include <complex>
#include <cmath>
#include <cstdio>
#include <utility>
#include <vector>
#include <cstdlib>
#include <cstring>
#include <string>

int main(int argc, char** argv)
{
    if (argc < 9) return 2;
    const std::size_t spins = std::strtoul(argv[1], nullptr, 10);
    const std::uint64_t seed = std::strtoull(argv[2], nullptr, 10);
    const double h = std::atof(argv[3]);
    const std::size_t depth = std::strtoul(argv[4], nullptr, 10);
    const std::size_t K = std::strtoul(argv[5], nullptr, 10);
    const std::size_t steps = std::strtoul(argv[6], nullptr, 10);
    const double dt = std::atof(argv[7]);
    const std::string mode = argv[8];

    helix::ContextOptions options;
    options.precision = helix::Precision::Double;
    helix::System system = helix::examples::transverse_ising_spin_glass(spins, seed, h);
    helix::HierarchySpec hierarchy = helix::examples::spin_glass_hierarchy(spins, 0.1, 1.0, 1.0, K, depth);
    helix::SolverOptions solver;
    solver.steps = steps;
    solver.timeStep = dt;
    if (mode == "single") options.precision = helix::Precision::Single;
    if (mode == "trace") solver.resultMode = helix::ResultMode::ObservableTrace;
    if (mode == "trajectory") solver.resultMode = helix::ResultMode::Trajectory;
    if (mode == "legacy") {
        // the reference's example: compiled legacy system, bath and hierarchy
        system = helix::examples::legacy_spin_glass_system();
        hierarchy = helix::HierarchySpec::compiled_default(helix::Bath::drude_lorentz_pade());
        options = helix::ContextOptions{};
    }
    if (mode == "sparse-general") {
        // H plus the complex Hermitian two-spin term 0.05 i (|r><r^3| - |r^3><r|), r < r^3:
        // outside the diagonal-plus-flip form, so System::from_sparse runs on the CSR path
        const helix::SparseOperator& H0 = system.hamiltonian;
        helix::SparseOperator H = H0;
        H.rowOffsets.assign(1, 0);
        H.columnIndices.clear();
        H.values.clear();
        for (std::size_t r = 0; r < H0.rows; ++r) {
            std::vector<std::pair<std::size_t, std::complex<double>>> row;
            for (std::size_t p = H0.rowOffsets[r]; p < H0.rowOffsets[r + 1]; ++p)
                row.emplace_back(H0.columnIndices[p], H0.values[p]);
            const std::size_t s = r ^ 3u;
            row.emplace_back(s, std::complex<double>(0.0, r < s ? 0.05 : -0.05));
            std::sort(row.begin(), row.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
            for (const auto& e : row) {
                H.columnIndices.push_back(e.first);
                H.values.push_back(e.second);
            }
            H.rowOffsets.push_back(H.columnIndices.size());
        }
        system = helix::System::from_sparse(H, system.couplings);
    }
    if (mode == "dense-single") {
        // H plus a dense Hermitian term (every entry non-zero), single precision requested: the
        // mixed-precision path with the commutator on the tensor cores
        options.precision = helix::Precision::Single;
        const helix::SparseOperator& H0 = system.hamiltonian;
        const std::size_t d = H0.rows;
        std::vector<std::complex<double>> dense(d * d);
        for (std::size_t r = 0; r < d; ++r)
            for (std::size_t p = H0.rowOffsets[r]; p < H0.rowOffsets[r + 1]; ++p) dense[r * d + H0.columnIndices[p]] += H0.values[p];
        const double scale = 0.02 / std::sqrt(static_cast<double>(d));
        for (std::size_t r = 0; r < d; ++r)
            for (std::size_t c = 0; c < d; ++c) {
                const double a = 0.3 * r + 0.7 * c, b = 0.3 * c + 0.7 * r;
                dense[r * d + c] += scale * std::complex<double>(std::cos(a) + std::cos(b), std::sin(a) - std::sin(b));
            }
        helix::SparseOperator H;
        H.rows = H.cols = d;
        H.rowOffsets.assign(1, 0);
        for (std::size_t r = 0; r < d; ++r) {
            for (std::size_t c = 0; c < d; ++c) {
                H.columnIndices.push_back(c);
                H.values.push_back(dense[r * d + c]);
            }
            H.rowOffsets.push_back(H.columnIndices.size());
        }
        system = helix::System::from_sparse(H, system.couplings);
    }
    if (mode == "sparse-bad") {
        // a column index outside the operator: System::from_sparse validation must flag it
        helix::SparseOperator bad = system.couplings[0];
        bad.columnIndices[0] = 1u << 20;
        system = helix::System::from_sparse(system.hamiltonian, {bad});
    }

    const helix::RunResult result = helix::HEOMSolver(options).run(system, hierarchy, solver);
    std::printf("{\"ok\": %s, \"codes\": [", result.ok() ? "true" : "false");
    for (std::size_t i = 0; i < result.diagnostics.entries().size(); ++i)
        std::printf("%s%d", i ? ", " : "", static_cast<int>(result.diagnostics.entries()[i].code));
    std::printf("], \"hierarchy\": %zu, \"count\": %zu, \"rows\": %zu, \"times\": [",
                result.diagnostics.hierarchySize, result.reduced_density_shape.count,
                result.reduced_density_shape.rows);
    for (std::size_t i = 0; i < result.times.size(); ++i) std::printf("%s%.17g", i ? ", " : "", result.times[i]);
    std::printf("], \"energies\": [");
    for (std::size_t i = 0; i < result.energies.size(); ++i) std::printf("%s%.17g", i ? ", " : "", result.energies[i]);
    std::printf("], \"rho\": [");
    for (std::size_t i = 0; i < result.reduced_density.size(); ++i)
        std::printf("%s%.17g, %.17g", i ? ", " : "", result.reduced_density[i].real(), result.reduced_density[i].imag());
    std::printf("], \"warnings\": %zu, \"single\": %s}\n", result.diagnostics.warnings.size(),
                result.diagnostics.precision == helix::Precision::Single ? "true" : "false");
    return 0;
}
