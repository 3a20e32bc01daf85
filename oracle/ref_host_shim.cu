// Host-only shim over the reference's own setup functions — TEST INFRASTRUCTURE.
//
// Compiled by oracle/build.py together with the reference sources
// src/psd/psd.cu and src/psd/eigenvalues.cu, straight from the reference tree,
// into oracle/_ref/libhelix_ref_host.so.  It exposes the reference's
// hierarchy-table builders (src/initialize_detail.h:159-269), its Pade
// decomposition (src/psd/psd.cu:12-113) and its legacy operator helpers
// (src/initialize_detail.h:38-157) through a C interface, so the tests can
// check the oracle and the CUDA table builder against the reference's code
// itself.  This file holds no reference code: it only calls it.

#include "initialize_detail.h"
#include "psd/psd.h"

#include <cstring>

extern "C" {

long long ref_hierarchy_size(int modes, int maxLevel)
{
    return initialize_detail::hierarchySizeFor(modes, maxLevel);
}

// rows: H*M ints, edges: H*2M ints.  Returns 0 on success.
int ref_hierarchy_tables(int modes, int maxLevel, int* rows, int* edges)
{
    const int count = initialize_detail::hierarchySizeFor(modes, maxLevel);
    host_vector<host_vector<int> > table = initialize_detail::buildHierarchyRows(modes, maxLevel);
    host_vector<host_vector<int> > edge(count, host_vector<int>(modes * 2));
    initialize_detail::buildHierarchyEdges(table, edge, count, modes);
    host_vector<int> flatRows = initialize_detail::flattenRows(table, modes);
    host_vector<int> flatEdges = initialize_detail::flattenRows(edge, modes * 2);
    for (size_t i = 0; i < flatRows.size(); ++i) rows[i] = flatRows[i];
    for (size_t i = 0; i < flatEdges.size(); ++i) edges[i] = flatEdges[i];
    return 0;
}

int ref_psd(int K, double* poles, double* residues)
{
    thrust::host_vector<double> p, r;
    double R = 0.0, T = 0.0;
    if (!getPsdPoleResidue(K, false, NMinus1_N, p, r, R, T)) return 1;
    for (int i = 0; i < K; ++i) {
        poles[i] = p[i];
        residues[i] = r[i];
    }
    return 0;
}

// Legacy diagonal Hamiltonian entry for one basis state (initialize.cu:139-142).
double ref_legacy_h_diagonal(int state, int spinCount, double coupling, int isSquare, double omega0)
{
    host_vector<double> couplings = initialize_detail::buildCouplingMatrix(spinCount, coupling, isSquare != 0);
    host_vector<double> projections = initialize_detail::spinProjections(state, spinCount, omega0);
    return initialize_detail::hamiltonianDiagonal(couplings, projections, spinCount);
}

double ref_legacy_projection_sum(int state, int spinCount, double omega0)
{
    host_vector<double> projections = initialize_detail::spinProjections(state, spinCount, omega0);
    return initialize_detail::sumProjections(projections);
}

int ref_sparse_flip_mask(int mask) { return initialize_detail::isSparseFlipMask(mask) ? 1 : 0; }

}  // extern "C"
