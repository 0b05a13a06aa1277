// mg_setup.h -- host construction of the lattice multigrid hierarchy that preconditions the
// field solve's CG on box meshes (meshes whose nodes sit on a regular lattice, such as the
// Kuhn boxes of scdat_kuhn_box_mesh).
//
// Level 0 is the Dirichlet-reduced Poisson matrix itself (HostPoisson).  Each coarser level
// keeps the lattice points of even index that are unknowns of the finer level; the
// prolongation P is trilinear interpolation on the lattice (weights 1, 1/2, 1/4, 1/8, dropped
// where the coarse point is not an unknown, so the correction vanishes on Dirichlet nodes),
// the restriction is P^T and the coarse operator the Galerkin product P^T A P.  Smoothing is
// damped Jacobi with weight 1.6 / (the Gershgorin bound of D^-1 A); the coarsest level (at
// most kMgCoarseMax rows) is solved by a dense inverse.
#pragma once

#include "mesh_setup.h"

#include <cstdint>
#include <string>
#include <vector>

namespace scdat {

constexpr int kMgCoarseMax = 1024;  // rows at which coarsening stops (dense coarsest solve)
constexpr int kMgMaxLevels = 12;

struct HostMgLevel {
    int R = 0;
    // operator of this level (levels >= 1; level 0 uses HostPoisson's arrays): off-diagonal
    // CSR with ascending columns, and the diagonal
    std::vector<int32_t> row_ptr, col;
    std::vector<double> val, diag;
    double omega = 0.8;  // damped-Jacobi weight
    // to the next coarser level (empty on the coarsest): P as CSR over this level's rows,
    // R = P^T as CSR over the coarser level's rows
    std::vector<int32_t> p_ptr, p_col, r_ptr, r_col;
    std::vector<float> p_w, r_w;
};

struct HostMg {
    std::vector<HostMgLevel> lv;     // lv[0] describes the fine level (R, omega, P, R)
    std::vector<double> coarse_inv;  // dense inverse of the coarsest operator, row-major
};

// Builds the hierarchy; returns an empty string on success, else why the mesh has none
// (its nodes are not on a regular lattice, or the lattice cannot be coarsened below
// kMgCoarseMax rows by halving).
std::string build_multigrid(const HostMesh& m, const HostPoisson& ps, HostMg& mg);

}  // namespace scdat
