// mg_setup.cpp -- the lattice multigrid hierarchy (see mg_setup.h).
#include "mg_setup.h"

#include <algorithm>
#include <cmath>
#include <thread>

namespace scdat {

namespace {

// Distinct coordinate values along one axis, if they are equally spaced.
bool lattice_axis(const std::vector<double>& xyz, int a, double tol, double& v0, double& h, int& n)
{
    std::vector<double> v;
    v.reserve(xyz.size() / 3);
    for (size_t i = a; i < xyz.size(); i += 3) v.push_back(xyz[i]);
    std::sort(v.begin(), v.end());
    std::vector<double> u;
    for (double x : v)
        if (u.empty() || x - u.back() > tol) u.push_back(x);
    n = (int)u.size();
    v0 = u[0];
    if (n < 2) return false;
    h = (u.back() - u[0]) / (n - 1);
    for (int k = 0; k < n; ++k)
        if (std::fabs(u[k] - (v0 + k * h)) > tol) return false;
    return h > 0.0;
}

struct Lattice {
    int n[3];                    // points per axis on this level
    std::vector<int64_t> point;  // lattice index of each row of the level
};

// Gershgorin bound of D^-1 A for a level given as diag + off-diagonal CSR.
double gershgorin(int R, const std::vector<int32_t>& ptr, const std::vector<double>& val, const std::vector<double>& d)
{
    double g = 0.0;
    for (int r = 0; r < R; ++r) {
        double s = std::fabs(d[r]);
        for (int32_t e = ptr[r]; e < ptr[r + 1]; ++e) s += std::fabs(val[e]);
        g = std::max(g, s / d[r]);
    }
    return g;
}

// Dense inverse of an SPD matrix by Cholesky: A = L L^T, A^-1 = L^-T L^-1.
bool spd_inverse(int n, std::vector<double>& a)
{
    std::vector<double> L((size_t)n * n, 0.0);
    for (int j = 0; j < n; ++j) {
        double s = a[(size_t)j * n + j];
        for (int k = 0; k < j; ++k) s -= L[(size_t)j * n + k] * L[(size_t)j * n + k];
        if (!(s > 0.0)) return false;
        const double ljj = std::sqrt(s);
        L[(size_t)j * n + j] = ljj;
        for (int i = j + 1; i < n; ++i) {
            double t = a[(size_t)i * n + j];
            for (int k = 0; k < j; ++k) t -= L[(size_t)i * n + k] * L[(size_t)j * n + k];
            L[(size_t)i * n + j] = t / ljj;
        }
    }
    // M = L^-1 (lower triangular), column by column
    std::vector<double> M((size_t)n * n, 0.0);
    for (int j = 0; j < n; ++j) {
        M[(size_t)j * n + j] = 1.0 / L[(size_t)j * n + j];
        for (int i = j + 1; i < n; ++i) {
            double t = 0.0;
            for (int k = j; k < i; ++k) t -= L[(size_t)i * n + k] * M[(size_t)k * n + j];
            M[(size_t)i * n + j] = t / L[(size_t)i * n + i];
        }
    }
    // A^-1 = M^T M
    for (int i = 0; i < n; ++i)
        for (int j = 0; j <= i; ++j) {
            double t = 0.0;
            for (int k = i; k < n; ++k) t += M[(size_t)k * n + i] * M[(size_t)k * n + j];
            a[(size_t)i * n + j] = t;
            a[(size_t)j * n + i] = t;
        }
    return true;
}

template <typename F>
void parallel_rows(int n, F&& f)
{
    const int nt = std::max(1, std::min<int>((int)std::thread::hardware_concurrency(), 32));
    if (nt == 1 || n < 4096) {
        f(0, n);
        return;
    }
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t) {
        const int a = (int)((int64_t)n * t / nt), b = (int)((int64_t)n * (t + 1) / nt);
        th.emplace_back([&f, a, b] { f(a, b); });
    }
    for (auto& x : th) x.join();
}

}  // namespace

std::string build_multigrid(const HostMesh& m, const HostPoisson& ps, HostMg& mg)
{
    mg = HostMg{};
    if (ps.R == 0) return "no interior rows";
    // the node lattice
    double ext = 0.0;
    for (int a = 0; a < 3; ++a) {
        double lo = m.xyz[a], hi = m.xyz[a];
        for (size_t i = a; i < m.xyz.size(); i += 3) {
            lo = std::min(lo, m.xyz[i]);
            hi = std::max(hi, m.xyz[i]);
        }
        ext = std::max(ext, hi - lo);
    }
    const double tol = 1e-9 * std::max(ext, 1e-300);
    double v0[3], h[3];
    Lattice fine;
    for (int a = 0; a < 3; ++a)
        if (!lattice_axis(m.xyz, a, tol, v0[a], h[a], fine.n[a])) return "mesh nodes are not on a regular lattice";
    const int64_t npts = (int64_t)fine.n[0] * fine.n[1] * fine.n[2];
    if (npts > ((int64_t)1 << 31)) return "lattice too large";
    std::vector<int32_t> row_at((size_t)npts, -1);  // lattice point -> row of the level
    fine.point.resize(ps.R);
    for (int r = 0; r < ps.R; ++r) {
        const int32_t nd = ps.row_node[r];
        int64_t idx = 0, mul = 1;
        for (int a = 0; a < 3; ++a) {
            const double q = (m.xyz[3 * (size_t)nd + a] - v0[a]) / h[a];
            const int64_t i = (int64_t)std::llround(q);
            if (std::fabs(q - (double)i) * h[a] > tol || i < 0 || i >= fine.n[a])
                return "mesh nodes are not on a regular lattice";
            idx += i * mul;
            mul *= fine.n[a];
        }
        if (row_at[idx] >= 0) return "two nodes on one lattice point";
        row_at[idx] = r;
        fine.point[r] = idx;
    }
    // the current level's operator in the common layout (level 0: HostPoisson's arrays)
    std::vector<int32_t> A_ptr = ps.row_ptr, A_col = ps.col;
    std::vector<double> A_val = ps.val, A_diag = ps.diag;
    Lattice cur = fine;
    int R = ps.R;
    for (int level = 0;; ++level) {
        HostMgLevel L;
        L.R = R;
        if (level > 0) {
            L.row_ptr = A_ptr;
            L.col = A_col;
            L.val = A_val;
            L.diag = A_diag;
        }
        const double g = gershgorin(R, A_ptr, A_val, A_diag);
        L.omega = g > 0.0 ? std::min(1.0, 1.6 / g) : 0.8;
        bool halvable = true;
        for (int a = 0; a < 3; ++a) halvable = halvable && cur.n[a] >= 3 && (cur.n[a] - 1) % 2 == 0;
        if (R <= kMgCoarseMax || !halvable || level + 1 >= kMgMaxLevels) {
            if (R > kMgCoarseMax) return "lattice cannot be coarsened below " + std::to_string(kMgCoarseMax) + " rows";
            // dense inverse of the coarsest operator
            std::vector<double> a((size_t)R * R, 0.0);
            for (int r = 0; r < R; ++r) {
                a[(size_t)r * R + r] = A_diag[r];
                for (int32_t e = A_ptr[r]; e < A_ptr[r + 1]; ++e) a[(size_t)r * R + A_col[e]] += A_val[e];
            }
            if (!spd_inverse(R, a)) return "coarsest operator is not positive definite";
            mg.coarse_inv = std::move(a);
            mg.lv.push_back(std::move(L));
            return "";
        }
        // coarse lattice and its unknowns: even points whose fine point is an unknown, in
        // ascending coarse lattice index
        Lattice crs;
        for (int a = 0; a < 3; ++a) crs.n[a] = (cur.n[a] - 1) / 2 + 1;
        const int64_t cpts = (int64_t)crs.n[0] * crs.n[1] * crs.n[2];
        std::vector<int32_t> crow((size_t)cpts, -1);
        int Rc = 0;
        {
            std::vector<int32_t> fine_row_at((size_t)((int64_t)cur.n[0] * cur.n[1] * cur.n[2]), -1);
            for (int r = 0; r < R; ++r) fine_row_at[cur.point[r]] = r;
            for (int64_t c = 0; c < cpts; ++c) {
                const int64_t ci = c % crs.n[0], cj = (c / crs.n[0]) % crs.n[1], ck = c / ((int64_t)crs.n[0] * crs.n[1]);
                const int64_t f = 2 * ci + (int64_t)cur.n[0] * (2 * cj + (int64_t)cur.n[1] * 2 * ck);
                if (fine_row_at[f] >= 0) crow[c] = Rc++;
            }
            crs.point.resize(Rc);
            for (int64_t c = 0; c < cpts; ++c)
                if (crow[c] >= 0) crs.point[crow[c]] = c;
        }
        if (Rc == 0) return "coarse level has no unknowns";
        // P: trilinear weights of each fine row
        L.p_ptr.assign((size_t)R + 1, 0);
        for (int r = 0; r < R; ++r) {
            const int64_t p = cur.point[r];
            const int64_t ii[3] = {p % cur.n[0], (p / cur.n[0]) % cur.n[1], p / ((int64_t)cur.n[0] * cur.n[1])};
            int64_t cc[3][2];
            float ww[3][2];
            int nc[3];
            for (int a = 0; a < 3; ++a) {
                if (ii[a] % 2 == 0) {
                    nc[a] = 1;
                    cc[a][0] = ii[a] / 2;
                    ww[a][0] = 1.0f;
                } else {
                    nc[a] = 2;
                    cc[a][0] = (ii[a] - 1) / 2;
                    cc[a][1] = (ii[a] + 1) / 2;
                    ww[a][0] = ww[a][1] = 0.5f;
                }
            }
            struct E {
                int32_t c;
                float w;
            } ent[8];
            int ne = 0;
            for (int z = 0; z < nc[2]; ++z)
                for (int y = 0; y < nc[1]; ++y)
                    for (int x = 0; x < nc[0]; ++x) {
                        const int64_t c = cc[0][x] + (int64_t)crs.n[0] * (cc[1][y] + (int64_t)crs.n[1] * cc[2][z]);
                        if (crow[c] >= 0) ent[ne++] = E{crow[c], ww[0][x] * ww[1][y] * ww[2][z]};
                    }
            std::sort(ent, ent + ne, [](const E& a, const E& b) { return a.c < b.c; });
            for (int k = 0; k < ne; ++k) {
                L.p_col.push_back(ent[k].c);
                L.p_w.push_back(ent[k].w);
            }
            L.p_ptr[r + 1] = (int32_t)L.p_col.size();
        }
        // R = P^T (fine rows ascending within each coarse row)
        L.r_ptr.assign((size_t)Rc + 1, 0);
        for (int32_t c : L.p_col) ++L.r_ptr[c + 1];
        for (int c = 0; c < Rc; ++c) L.r_ptr[c + 1] += L.r_ptr[c];
        L.r_col.resize(L.p_col.size());
        L.r_w.resize(L.p_col.size());
        {
            std::vector<int32_t> fill(L.r_ptr.begin(), L.r_ptr.end() - 1);
            for (int r = 0; r < R; ++r)
                for (int32_t e = L.p_ptr[r]; e < L.p_ptr[r + 1]; ++e) {
                    const int32_t c = L.p_col[e];
                    L.r_col[fill[c]] = r;
                    L.r_w[fill[c]] = L.p_w[e];
                    ++fill[c];
                }
        }
        // Galerkin product P^T A P, one coarse row at a time:
        // Ac[c, :] = sum_{f in R[c]} w_fc * sum_{j in A[f, :]} A_fj * P[j, :]
        std::vector<std::vector<int32_t>> rcol((size_t)Rc);
        std::vector<std::vector<double>> rval((size_t)Rc);
        std::vector<double> cdiag((size_t)Rc, 0.0);
        parallel_rows(Rc, [&](int c0, int c1) {
            std::vector<double> acc((size_t)Rc, 0.0);
            std::vector<char> seen((size_t)Rc, 0);
            std::vector<int32_t> touched;
            for (int c = c0; c < c1; ++c) {
                touched.clear();
                for (int32_t e = L.r_ptr[c]; e < L.r_ptr[c + 1]; ++e) {
                    const int32_t f = L.r_col[e];
                    const double wf = L.r_w[e];
                    auto add_col = [&](int32_t j, double a) {
                        for (int32_t q = L.p_ptr[j]; q < L.p_ptr[j + 1]; ++q) {
                            const int32_t c2 = L.p_col[q];
                            if (!seen[c2]) {
                                seen[c2] = 1;
                                touched.push_back(c2);
                            }
                            acc[c2] += wf * a * (double)L.p_w[q];
                        }
                    };
                    add_col(f, A_diag[f]);
                    for (int32_t k = A_ptr[f]; k < A_ptr[f + 1]; ++k) add_col(A_col[k], A_val[k]);
                }
                std::sort(touched.begin(), touched.end());
                for (int32_t c2 : touched) {
                    const double v = acc[c2];
                    if (c2 == c)
                        cdiag[c] = v;
                    else if (v != 0.0) {
                        rcol[c].push_back(c2);
                        rval[c].push_back(v);
                    }
                    acc[c2] = 0.0;
                    seen[c2] = 0;
                }
            }
        });
        mg.lv.push_back(std::move(L));
        // the coarse level becomes the current one
        A_ptr.assign((size_t)Rc + 1, 0);
        A_col.clear();
        A_val.clear();
        for (int c = 0; c < Rc; ++c) {
            A_col.insert(A_col.end(), rcol[c].begin(), rcol[c].end());
            A_val.insert(A_val.end(), rval[c].begin(), rval[c].end());
            A_ptr[c + 1] = (int32_t)A_col.size();
            if (!(cdiag[c] > 0.0)) return "coarse operator has a non-positive diagonal";
        }
        A_diag = std::move(cdiag);
        cur = std::move(crs);
        R = Rc;
    }
}

}  // namespace scdat
