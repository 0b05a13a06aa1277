// mesh_setup.h -- host-side preprocessing of a tetrahedral mesh for the device kernels:
// face neighbours, per-tet inverse Jacobians, the locate grid, the node graph and the
// Dirichlet-reduced edge-Laplacian (PoissonSolver.cpp:274-385, LinearSystem.cpp:37-58).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace scdat {

struct HostMesh {
    int64_t N = 0, T = 0;
    std::vector<double> xyz;      // [N*3]
    std::vector<int32_t> tet;     // [T*4]
    std::vector<int32_t> nbr;     // [T*4]
    std::vector<uint8_t> dirichlet;
    std::vector<double> eps_rel;  // [T] or empty
};

struct HostGeometry {
    std::vector<double> geom;   // [T*16] inverse Jacobian row-major, origin xyz, face neighbours + node ids (int32)
    std::vector<float> geomf;   // [T*12] FP32 inverse Jacobian, 3 unused
    double bmin[3], bmax[3];
    double max_edge = 0.0;
};

struct HostGrid {
    double gmin[3], ginv[3];
    int32_t gdim[3];
    double gdelta;
    std::vector<int32_t> bin_start, bin_tets;
};

struct HostGraph {
    std::vector<int32_t> ptr, col;  // node graph CSR, neighbours ascending, no self
};

struct HostPoisson {
    int R = 0;
    std::vector<int32_t> row_of_node;  // -1 for Dirichlet nodes
    std::vector<int32_t> row_node;
    std::vector<double> cv, diag, dinv;
    std::vector<float> diagf, dinvf;
    std::vector<int32_t> row_ptr, col;
    std::vector<double> val;
    std::vector<float> valf;
    std::vector<int32_t> lift_ptr, lift_node;
    std::vector<double> lift_val;
};

// Returns an empty string on success, else the reason.
std::string compute_face_neighbors(const HostMesh& m, std::vector<int32_t>& nbr);
std::string compute_geometry(const HostMesh& m, HostGeometry& g);
std::string build_locate_grid(const HostMesh& m, const HostGeometry& g, HostGrid& grid);
std::string build_node_graph(const HostMesh& m, HostGraph& gr);
std::string assemble_poisson(const HostMesh& m, const HostGraph& gr, HostPoisson& ps);

// 6-tet Kuhn box (node id = i + (nx+1)*(j + (ny+1)*k); hex cells x-fastest, minus the
// half-open body range; tets 6 per hex in permutation order (0,1,2),(0,2,1),(1,0,2),(1,2,0),
// (2,0,1),(2,1,0)).  Outer-face nodes Dirichlet at `wall`, body nodes Dirichlet at `bias`.
void build_kuhn_box(int nx, int ny, int nz, double h, const int* body_lo, const int* body_hi, double bias,
                    double wall, std::vector<double>& xyz, std::vector<int32_t>& tet, std::vector<uint8_t>& dirichlet,
                    std::vector<double>& phi, std::vector<int32_t>& hex_ijk);

}  // namespace scdat
