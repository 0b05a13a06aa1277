// mesh_setup.cpp -- host preprocessing (see mesh_setup.h).
#include "mesh_setup.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

namespace scdat {

namespace {
constexpr double kEps0 = 8.8541878128e-12;  // PoissonSolver.cpp:18

inline void node(const HostMesh& m, int64_t n, double p[3])
{
    p[0] = m.xyz[3 * n];
    p[1] = m.xyz[3 * n + 1];
    p[2] = m.xyz[3 * n + 2];
}
}  // namespace

std::string compute_face_neighbors(const HostMesh& m, std::vector<int32_t>& nbr)
{
    const int64_t T = m.T;
    nbr.assign((size_t)(4 * T), -1);
    struct Face {
        int32_t a, b, c;
        int64_t owner;  // tet*4 + local face
    };
    std::vector<Face> f((size_t)(4 * T));
    for (int64_t t = 0; t < T; ++t) {
        const int32_t* tn = &m.tet[4 * t];
        for (int k = 0; k < 4; ++k) {
            int32_t v[3], q = 0;
            for (int i = 0; i < 4; ++i)
                if (i != k) v[q++] = tn[i];
            std::sort(v, v + 3);
            f[4 * t + k] = Face{v[0], v[1], v[2], 4 * t + k};
        }
    }
    std::sort(f.begin(), f.end(), [](const Face& x, const Face& y) {
        if (x.a != y.a) return x.a < y.a;
        if (x.b != y.b) return x.b < y.b;
        if (x.c != y.c) return x.c < y.c;
        return x.owner < y.owner;
    });
    for (size_t i = 0; i + 1 < f.size(); ++i) {
        if (f[i].a == f[i + 1].a && f[i].b == f[i + 1].b && f[i].c == f[i + 1].c) {
            if (i + 2 < f.size() && f[i + 2].a == f[i].a && f[i + 2].b == f[i].b && f[i + 2].c == f[i].c)
                return "non-manifold mesh: a face is shared by more than two tets";
            nbr[f[i].owner] = (int32_t)(f[i + 1].owner / 4);
            nbr[f[i + 1].owner] = (int32_t)(f[i].owner / 4);
            ++i;
        }
    }
    return "";
}

std::string compute_geometry(const HostMesh& m, HostGeometry& g)
{
    const int64_t T = m.T;
    g.geom.assign((size_t)(16 * T), 0.0);
    g.geomf.assign((size_t)(12 * T), 0.0f);
    for (int a = 0; a < 3; ++a) {
        g.bmin[a] = std::numeric_limits<double>::infinity();
        g.bmax[a] = -std::numeric_limits<double>::infinity();
    }
    for (int64_t n = 0; n < m.N; ++n)
        for (int a = 0; a < 3; ++a) {
            g.bmin[a] = std::min(g.bmin[a], m.xyz[3 * n + a]);
            g.bmax[a] = std::max(g.bmax[a], m.xyz[3 * n + a]);
        }
    const double nan = std::numeric_limits<double>::quiet_NaN();
    double max_edge = 0.0;
    for (int64_t t = 0; t < T; ++t) {
        double p[4][3];
        for (int i = 0; i < 4; ++i) {
            int32_t id = m.tet[4 * t + i];
            if (id < 0 || id >= m.N) return "tet node index out of range";
            node(m, id, p[i]);
        }
        for (int i = 0; i < 4; ++i)
            for (int j = i + 1; j < 4; ++j) {
                double d = std::sqrt((p[i][0] - p[j][0]) * (p[i][0] - p[j][0]) + (p[i][1] - p[j][1]) * (p[i][1] - p[j][1]) +
                                     (p[i][2] - p[j][2]) * (p[i][2] - p[j][2]));
                max_edge = std::max(max_edge, d);
            }
        // J = [p1-p0, p2-p0, p3-p0] (columns); lambda_{1..3} = J^-1 (x - p0)
        double J[3][3];
        for (int c = 0; c < 3; ++c)
            for (int r = 0; r < 3; ++r) J[r][c] = p[c + 1][r] - p[0][r];
        // signed volume x6 as FieldInterpolator uses it (PICParticleAlgorithms.cpp:261-276)
        double v1[3] = {J[0][0], J[1][0], J[2][0]}, v2[3] = {J[0][1], J[1][1], J[2][1]},
               v3[3] = {J[0][2], J[1][2], J[2][2]};
        double cx = v2[1] * v3[2] - v2[2] * v3[1], cy = v2[2] * v3[0] - v2[0] * v3[2], cz = v2[0] * v3[1] - v2[1] * v3[0];
        double V6 = v1[0] * cx + v1[1] * cy + v1[2] * cz;
        double* G = &g.geom[16 * t];
        float* Gf = &g.geomf[12 * t];
        if (std::fabs(V6) < 1e-15) {  // degenerate: never contains a point
            for (int k = 0; k < 9; ++k) {
                G[k] = nan;
                Gf[k] = std::numeric_limits<float>::quiet_NaN();
            }
        } else {
            double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                         J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
            double id = 1.0 / det;
            double inv[3][3];
            inv[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) * id;
            inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
            inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
            inv[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) * id;
            inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
            inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
            inv[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) * id;
            inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
            inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) {
                    G[3 * r + c] = inv[r][c];
                    Gf[3 * r + c] = (float)inv[r][c];
                }
        }
        G[9] = p[0][0];
        G[10] = p[0][1];
        G[11] = p[0][2];
        // words 12..15 hold the 4 face neighbours and the 4 node ids as int32
        int32_t ids[8];
        for (int k = 0; k < 4; ++k) {
            ids[k] = m.nbr.empty() ? -1 : m.nbr[4 * t + k];
            ids[4 + k] = m.tet[4 * t + k];
        }
        std::memcpy(&G[12], ids, sizeof(ids));
    }
    g.max_edge = max_edge;
    return "";
}

std::string build_locate_grid(const HostMesh& m, const HostGeometry& g, HostGrid& grid)
{
    const int64_t T = m.T;
    double ext[3];
    double vol = 1.0;
    for (int a = 0; a < 3; ++a) {
        ext[a] = std::max(g.bmax[a] - g.bmin[a], 1e-300);
        vol *= ext[a];
    }
    // bins about the size of a group of 6 tets (one hex of a Kuhn box)
    double bs = std::cbrt(vol * 6.0 / (double)std::max<int64_t>(T, 1));
    int64_t total = 1;
    for (int a = 0; a < 3; ++a) {
        int d = (int)std::ceil(ext[a] / bs - 1e-9);
        d = std::max(1, std::min(d, 2048));
        grid.gdim[a] = d;
        grid.gmin[a] = g.bmin[a];
        grid.ginv[a] = (double)d / ext[a];
        total *= d;
    }
    if (total > (int64_t)1 << 30) return "locate grid too large";
    grid.gdelta = 2e-8 * g.max_edge + 1e-300;
    std::vector<int32_t> cnt((size_t)total + 1, 0);
    auto range = [&](int64_t t, int lo[3], int hi[3]) {
        for (int a = 0; a < 3; ++a) {
            double mn = 1e300, mx = -1e300;
            for (int i = 0; i < 4; ++i) {
                double c = m.xyz[3 * (int64_t)m.tet[4 * t + i] + a];
                mn = std::min(mn, c);
                mx = std::max(mx, c);
            }
            int l = (int)std::floor((mn - grid.gmin[a]) * grid.ginv[a]);
            int h = (int)std::floor((mx - grid.gmin[a]) * grid.ginv[a]);
            lo[a] = std::max(0, std::min(l, grid.gdim[a] - 1));
            hi[a] = std::max(0, std::min(h, grid.gdim[a] - 1));
        }
    };
    int lo[3], hi[3];
    for (int64_t t = 0; t < T; ++t) {
        range(t, lo, hi);
        for (int k = lo[2]; k <= hi[2]; ++k)
            for (int j = lo[1]; j <= hi[1]; ++j)
                for (int i = lo[0]; i <= hi[0]; ++i) cnt[1 + i + grid.gdim[0] * ((int64_t)j + grid.gdim[1] * (int64_t)k)]++;
    }
    for (int64_t b = 0; b < total; ++b) {
        if ((int64_t)cnt[b + 1] + cnt[b] > 0x7fffffffLL) return "locate grid index overflow";
        cnt[b + 1] += cnt[b];
    }
    grid.bin_start = cnt;
    grid.bin_tets.assign((size_t)cnt[total], 0);
    std::vector<int32_t> cur(cnt.begin(), cnt.end() - 1);
    for (int64_t t = 0; t < T; ++t) {  // ascending tet id inside every bin
        range(t, lo, hi);
        for (int k = lo[2]; k <= hi[2]; ++k)
            for (int j = lo[1]; j <= hi[1]; ++j)
                for (int i = lo[0]; i <= hi[0]; ++i)
                    grid.bin_tets[cur[i + grid.gdim[0] * ((int64_t)j + grid.gdim[1] * (int64_t)k)]++] = (int32_t)t;
    }
    return "";
}

std::string build_node_graph(const HostMesh& m, HostGraph& gr)
{
    const int64_t N = m.N, T = m.T;
    std::vector<int64_t> deg((size_t)N + 1, 0);
    for (int64_t t = 0; t < T; ++t)
        for (int i = 0; i < 4; ++i) deg[1 + m.tet[4 * t + i]] += 3;
    for (int64_t n = 0; n < N; ++n) deg[n + 1] += deg[n];
    std::vector<int32_t> tmp((size_t)deg[N]);
    std::vector<int64_t> cur(deg.begin(), deg.end() - 1);
    for (int64_t t = 0; t < T; ++t)
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j)
                if (i != j) tmp[cur[m.tet[4 * t + i]]++] = m.tet[4 * t + j];
    gr.ptr.assign((size_t)N + 1, 0);
    gr.col.clear();
    gr.col.reserve((size_t)(deg[N] / 4 + 16));
    for (int64_t n = 0; n < N; ++n) {
        auto b = tmp.begin() + deg[n], e = tmp.begin() + deg[n + 1];
        std::sort(b, e);
        auto u = std::unique(b, e);
        for (auto it = b; it != u; ++it)
            if (*it != n) gr.col.push_back(*it);
        if (gr.col.size() > 0x7fffffffULL) return "node graph too large";
        gr.ptr[n + 1] = (int32_t)gr.col.size();
    }
    return "";
}

std::string assemble_poisson(const HostMesh& m, const HostGraph& gr, HostPoisson& ps)
{
    const int64_t N = m.N, T = m.T;
    // full matrix in graph layout, accumulated element by element in element order like
    // the dense LinearSystem (PoissonSolver.cpp:264-269, 274-329)
    std::vector<double> off(gr.col.size(), 0.0), diag((size_t)N, 0.0), cv((size_t)N, 0.0);
    auto find = [&](int32_t i, int32_t j) -> int64_t {
        auto b = gr.col.begin() + gr.ptr[i], e = gr.col.begin() + gr.ptr[i + 1];
        auto it = std::lower_bound(b, e, j);
        return (it != e && *it == j) ? (int64_t)(it - gr.col.begin()) : -1;
    };
    for (int64_t t = 0; t < T; ++t) {
        const int32_t* tn = &m.tet[4 * t];
        double p[4][3];
        for (int i = 0; i < 4; ++i) node(m, tn[i], p[i]);
        // TetrahedronElement::getVolume (MeshAlgorithms.cpp:29-54) + elementMeasure (PoissonSolver.cpp:31-38)
        double ax = p[1][0] - p[0][0], ay = p[1][1] - p[0][1], az = p[1][2] - p[0][2];
        double bx = p[2][0] - p[0][0], by = p[2][1] - p[0][1], bz = p[2][2] - p[0][2];
        double cx = p[3][0] - p[0][0], cy = p[3][1] - p[0][1], cz = p[3][2] - p[0][2];
        double det = ax * (by * cz - bz * cy) - ay * (bx * cz - bz * cx) + az * (bx * cy - by * cx);
        double vol = std::fabs(det) / 6.0;
        double meas = std::max(std::fabs(vol), 1.0e-12);
        // resolvePermittivity (PoissonSolver.cpp:21-29) of the tet's material
        double epsr = m.eps_rel.empty() ? 1.0 : m.eps_rel[t];
        double eps = epsr <= 0.0 ? kEps0 : (epsr < 1.0e-8 ? epsr : epsr * kEps0);
        double es = meas / 6.0;
        for (int i = 0; i < 4; ++i) {
            for (int j = i + 1; j < 4; ++j) {
                double dx = p[i][0] - p[j][0], dy = p[i][1] - p[j][1], dz = p[i][2] - p[j][2];
                double d = std::max(std::sqrt(dx * dx + dy * dy + dz * dz), 1.0e-12);
                double w = eps * es / (d * d);
                diag[tn[i]] += w;
                diag[tn[j]] += w;
                int64_t eij = find(tn[i], tn[j]), eji = find(tn[j], tn[i]);
                if (eij < 0 || eji < 0) return "node graph inconsistent with tets";
                off[eij] += -w;
                off[eji] += -w;
            }
        }
        for (int i = 0; i < 4; ++i) cv[tn[i]] += meas / 4.0;
    }
    ps.row_of_node.assign((size_t)N, -1);
    ps.row_node.clear();
    for (int64_t n = 0; n < N; ++n)
        if (!m.dirichlet[n]) {
            ps.row_of_node[n] = (int32_t)ps.row_node.size();
            ps.row_node.push_back((int32_t)n);
        }
    ps.R = (int)ps.row_node.size();
    ps.cv.resize(ps.R);
    ps.diag.resize(ps.R);
    ps.dinv.resize(ps.R);
    ps.diagf.resize(ps.R);
    ps.dinvf.resize(ps.R);
    ps.row_ptr.assign((size_t)ps.R + 1, 0);
    ps.lift_ptr.assign((size_t)ps.R + 1, 0);
    ps.col.clear();
    ps.val.clear();
    ps.valf.clear();
    ps.lift_node.clear();
    ps.lift_val.clear();
    for (int r = 0; r < ps.R; ++r) {
        int32_t n = ps.row_node[r];
        ps.cv[r] = cv[n];
        ps.diag[r] = diag[n];
        if (!(diag[n] > 0.0)) return "interior node with no positive diagonal (isolated node not marked Dirichlet)";
        ps.dinv[r] = 1.0 / diag[n];
        ps.diagf[r] = (float)ps.diag[r];
        ps.dinvf[r] = (float)ps.dinv[r];
        for (int32_t e = gr.ptr[n]; e < gr.ptr[n + 1]; ++e) {
            int32_t j = gr.col[e];
            if (m.dirichlet[j]) {
                ps.lift_node.push_back(j);
                ps.lift_val.push_back(off[e]);
            } else {
                ps.col.push_back(ps.row_of_node[j]);
                ps.val.push_back(off[e]);
                ps.valf.push_back((float)off[e]);
            }
        }
        ps.row_ptr[r + 1] = (int32_t)ps.col.size();
        ps.lift_ptr[r + 1] = (int32_t)ps.lift_node.size();
    }
    return "";
}

void build_kuhn_box(int nx, int ny, int nz, double h, const int* body_lo, const int* body_hi, double bias,
                    double wall, std::vector<double>& xyz, std::vector<int32_t>& tet, std::vector<uint8_t>& dirichlet,
                    std::vector<double>& phi, std::vector<int32_t>& hex_ijk)
{
    static const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    const int64_t N = (int64_t)(nx + 1) * (ny + 1) * (nz + 1);
    xyz.resize((size_t)(3 * N));
    dirichlet.assign((size_t)N, 0);
    phi.assign((size_t)N, 0.0);
    auto nid = [&](int64_t i, int64_t j, int64_t k) { return i + (int64_t)(nx + 1) * (j + (int64_t)(ny + 1) * k); };
    const bool has_body = body_lo && body_hi;
    for (int k = 0; k <= nz; ++k)
        for (int j = 0; j <= ny; ++j)
            for (int i = 0; i <= nx; ++i) {
                int64_t n = nid(i, j, k);
                xyz[3 * n] = i * h;
                xyz[3 * n + 1] = j * h;
                xyz[3 * n + 2] = k * h;
                if (i == 0 || i == nx || j == 0 || j == ny || k == 0 || k == nz) {
                    dirichlet[n] = 1;
                    phi[n] = wall;
                }
                if (has_body && i >= body_lo[0] && i <= body_hi[0] && j >= body_lo[1] && j <= body_hi[1] &&
                    k >= body_lo[2] && k <= body_hi[2]) {
                    dirichlet[n] = 1;
                    phi[n] = bias;
                }
            }
    hex_ijk.clear();
    tet.clear();
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                if (has_body && i >= body_lo[0] && i < body_hi[0] && j >= body_lo[1] && j < body_hi[1] &&
                    k >= body_lo[2] && k < body_hi[2])
                    continue;
                hex_ijk.push_back(i);
                hex_ijk.push_back(j);
                hex_ijk.push_back(k);
                for (int p = 0; p < 6; ++p) {
                    int c[3] = {0, 0, 0};
                    tet.push_back((int32_t)nid(i, j, k));
                    for (int s = 0; s < 3; ++s) {
                        c[perms[p][s]] += 1;
                        tet.push_back((int32_t)nid(i + c[0], j + c[1], k + c[2]));
                    }
                }
            }
}

}  // namespace scdat
