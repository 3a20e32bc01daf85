#pragma once

#include <helix/types.h>

#include <cstdint>

namespace helix::examples {

// The reference's compiled spin-glass model (d = 1024, one collective bath).
System legacy_spin_glass_system();

// Transverse-field Ising spin glass H = sum_{i<j} J_ij sz_i sz_j + h sum_i sx_i
// with J_ij ~ N(0,1) from `seed` (splitmix64 + Box-Muller, i<j row-major pair
// order), as System::from_sparse(H, {sz_0, ..., sz_{n-1}}).
System transverse_ising_spin_glass(std::size_t spins, std::uint64_t seed, double h);

// One Drude-Lorentz bath per spin (lambda, gamma, temperature, K Pade terms),
// hierarchy depth L (maxDepth = L + 1).
HierarchySpec spin_glass_hierarchy(std::size_t spins, double lambda, double gamma, double temperature,
                                   std::size_t padeTerms, std::size_t depth);

}  // namespace helix::examples
