// maille_oracle.cpp -- CPU FP64 restatement of the reference's linear-elastic solve path.
//
// TEST INFRASTRUCTURE ONLY. This file is the oracle: tests/, __graft_entry__.smoke() and the
// cpu_baseline / reference legs of bench.py load it as the checker and as the timed CPU
// baseline. The product library (maille_b200/) never links, loads or calls it.
//
// The reference (timothee-faget/maille, pure Rust, single-threaded) cannot be compiled in this
// image (no cargo/rustc), so this is a single-threaded C++17 restatement that keeps the
// reference's order of floating-point operations: it is compiled with -ffp-contract=off (Rust
// never fuses a*b+c), sums are left folds like Rust's Iterator::sum, and `dot` keeps the
// reference's 8-lane combine order. Every function cites the reference file:line it follows
// (paths relative to the reference project root, crate maille-core unless stated).
//
// Parity pin: the oracle is checked against the reference's own known-answer tests (analytic
// patch test, uniaxial traction, hydrostatic cube with face pressure, face-load KATs, element
// invariants, the iterative.rs / solve.rs unit tests and the examples/cube fixture), restated in
// tests/test_oracle_kats.py.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <optional>
#include <vector>

namespace {

using std::size_t;
using Vec = std::vector<double>;
using IVec = std::vector<size_t>;
constexpr size_t NONE = std::numeric_limits<size_t>::max();

// --- constants -------------------------------------------------------------------------------

// src/iterative.rs:9-14
constexpr double TOLERANCE = 1e-12;
constexpr size_t MAX_ITERATIONS = 10000;
constexpr double SHIFTS[6] = {0.0, 1e-3, 1e-2, 1e-1, 1.0, 10.0};
// src/solve.rs:185
constexpr size_t ITERATIVE_FROM = 100000;

// status codes shared with the tests (mirror of MailleError on this path, src/error.rs:224-229)
enum Status : int { OK = 0, SINGULAR = 1, NOT_CONVERGED = 2, INVALID = 3 };
// Inside the quasi-static Newton loop only: an inner PCG that hit its cap
// (MailleError::IterativeNotConverged, error.rs:226-229), which advance (model.rs:839-842) does
// not answer with a cut, unlike Newton's NotConverged; reported to callers as NOT_CONVERGED.
constexpr int ITERATIVE_NOT_CONVERGED = 4;

// --- quadrature: src/quadrature.rs ------------------------------------------------------------

struct TetGP { double xi, eta, zeta, w; };
struct TriGP { double xi, eta, w; };

// TETRA_1, quadrature.rs:100-105
const TetGP TETRA_1[1] = {{0.25, 0.25, 0.25, 1.0 / 6.0}};
// TET_A / TET_B and TETRA_4, quadrature.rs:108-138
constexpr double TET_A = 0.5854101966249685;
constexpr double TET_B = 0.1381966011250105;
const TetGP TETRA_4[4] = {{TET_B, TET_B, TET_B, 1.0 / 24.0},
                          {TET_A, TET_B, TET_B, 1.0 / 24.0},
                          {TET_B, TET_A, TET_B, 1.0 / 24.0},
                          {TET_B, TET_B, TET_A, 1.0 / 24.0}};
// TRIANGLE_3, quadrature.rs:19-35
const TriGP TRIANGLE_3[3] = {{1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0},
                             {2.0 / 3.0, 1.0 / 6.0, 1.0 / 6.0},
                             {1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0}};
// TRIANGLE_6 (Dunavant), quadrature.rs:38-54
constexpr double T6A = 0.445948490915965;
constexpr double T6WA = 0.223381589678011 / 2.0;
constexpr double T6B = 0.091576213509771;
constexpr double T6WB = 0.109951743655322 / 2.0;
const TriGP TRIANGLE_6[6] = {{T6A, T6A, T6WA},
                             {1.0 - 2.0 * T6A, T6A, T6WA},
                             {T6A, 1.0 - 2.0 * T6A, T6WA},
                             {T6B, T6B, T6WB},
                             {1.0 - 2.0 * T6B, T6B, T6WB},
                             {T6B, 1.0 - 2.0 * T6B, T6WB}};

// --- shape functions: src/shape.rs -----------------------------------------------------------

// TET_FACES, shape.rs:129 ; TET10_EDGES, shape.rs:135
const int TET_FACES[4][3] = {{0, 1, 2}, {0, 3, 1}, {1, 3, 2}, {2, 3, 0}};
const int TET10_EDGES[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};

// tet_barycentric + tet4 + tet10, shape.rs:95-153. n: values, dn: [npe][3] derivatives.
void tet_shape(int npe, double xi, double eta, double zeta, double* n, double (*dn)[3]) {
    const double l[4] = {1.0 - xi - eta - zeta, xi, eta, zeta};
    const double dl[4][3] = {{-1.0, -1.0, -1.0}, {1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};
    if (npe == 4) {
        for (int i = 0; i < 4; ++i) {
            n[i] = l[i];
            for (int c = 0; c < 3; ++c) dn[i][c] = dl[i][c];
        }
        return;
    }
    for (int i = 0; i < 4; ++i) {
        n[i] = l[i] * (2.0 * l[i] - 1.0);
        for (int c = 0; c < 3; ++c) dn[i][c] = (4.0 * l[i] - 1.0) * dl[i][c];
    }
    for (int k = 0; k < 6; ++k) {
        const int a = TET10_EDGES[k][0], b = TET10_EDGES[k][1];
        n[4 + k] = 4.0 * l[a] * l[b];
        for (int c = 0; c < 3; ++c) dn[4 + k][c] = 4.0 * (l[a] * dl[b][c] + l[b] * dl[a][c]);
    }
}

// tri3 / tri6 values, shape.rs:11-48
void tri_values(int nn, double xi, double eta, double* n) {
    if (nn == 3) {
        n[0] = 1.0 - xi - eta;
        n[1] = xi;
        n[2] = eta;
        return;
    }
    const double l1 = 1.0 - xi - eta, l2 = xi, l3 = eta;
    n[0] = l1 * (2.0 * l1 - 1.0);
    n[1] = l2 * (2.0 * l2 - 1.0);
    n[2] = l3 * (2.0 * l3 - 1.0);
    n[3] = 4.0 * l1 * l2;
    n[4] = 4.0 * l2 * l3;
    n[5] = 4.0 * l3 * l1;
}

// Mapping3d::new, shape.rs:164-190: det J by cofactors and dN/dx = J^-1 dN/dxi.
double mapping3d(int npe, const double (*coords)[3], const double (*dn)[3], double (*dn_dx)[3]) {
    double j[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int k = 0; k < npe; ++k)
        for (int i = 0; i < 3; ++i)
            for (int r = 0; r < 3; ++r) j[i][r] += dn[k][i] * coords[k][r];
    auto cof = [&](int r, int c) {
        const int r1 = (r + 1) % 3, r2 = (r + 2) % 3, c1 = (c + 1) % 3, c2 = (c + 2) % 3;
        return j[r1][c1] * j[r2][c2] - j[r1][c2] * j[r2][c1];
    };
    double det = 0.0;
    det = j[0][0] * cof(0, 0);
    det = det + j[0][1] * cof(0, 1);
    det = det + j[0][2] * cof(0, 2);
    double inv[3][3];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) inv[r][c] = cof(c, r) / det;
    for (int k = 0; k < npe; ++k)
        for (int r = 0; r < 3; ++r) {
            double s = inv[r][0] * dn[k][0];
            s = s + inv[r][1] * dn[k][1];
            s = s + inv[r][2] * dn[k][2];
            dn_dx[k][r] = s;
        }
    return det;
}

// --- element kernels: src/element.rs ---------------------------------------------------------

// solid_d, element.rs:193-206 (Voigt xx, yy, zz, yz, xz, xy; engineering shears)
void solid_d(double young, double nu, double d[6][6]) {
    const double c = young / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double g = young / (2.0 * (1.0 + nu));
    for (int i = 0; i < 6; ++i)
        for (int k = 0; k < 6; ++k) d[i][k] = 0.0;
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) d[i][k] = (i == k) ? c * (1.0 - nu) : c * nu;
    for (int i = 3; i < 6; ++i) d[i][i] = g;
}

// solid_strain_displacement, element.rs:209-220: column 3k+c of B (6 rows).
void b_columns(int npe, const double (*g)[3], double (*b)[6]) {
    for (int k = 0; k < npe; ++k) {
        const double gx = g[k][0], gy = g[k][1], gz = g[k][2];
        const double c0[6] = {gx, 0.0, 0.0, 0.0, gz, gy};
        const double c1[6] = {0.0, gy, 0.0, gz, 0.0, gx};
        const double c2[6] = {0.0, 0.0, gz, gy, gx, 0.0};
        for (int r = 0; r < 6; ++r) {
            b[3 * k][r] = c0[r];
            b[3 * k + 1][r] = c1[r];
            b[3 * k + 2][r] = c2[r];
        }
    }
}

// Rule of SolidKernel::tet4 / ::tet10, assembly.rs:212-229
int rule_of(int npe, const TetGP** rule) {
    if (npe == 4) {
        *rule = TETRA_1;
        return 1;
    }
    *rule = TETRA_4;
    return 4;
}

// solid_stiffness, element.rs:223-243. ke is m x m row-major, ke[j*m+i].
void solid_stiffness(int npe, const double (*coords)[3], const double d[6][6], double* ke) {
    const int m = 3 * npe;
    std::fill(ke, ke + m * m, 0.0);
    const TetGP* rule;
    const int ng = rule_of(npe, &rule);
    double n[10], dn[10][3], dn_dx[10][3], b[30][6];
    for (int gp = 0; gp < ng; ++gp) {
        tet_shape(npe, rule[gp].xi, rule[gp].eta, rule[gp].zeta, n, dn);
        const double det = mapping3d(npe, coords, dn, dn_dx);
        b_columns(npe, dn_dx, b);
        const double factor = rule[gp].w * std::fabs(det);
        for (int i = 0; i < m; ++i) {
            double db[6];
            for (int r = 0; r < 6; ++r) {
                double s = d[r][0] * b[i][0];
                for (int c = 1; c < 6; ++c) s = s + d[r][c] * b[i][c];
                db[r] = s;
            }
            for (int jj = 0; jj < m; ++jj) {
                double s = b[jj][0] * db[0];
                for (int r = 1; r < 6; ++r) s = s + b[jj][r] * db[r];
                ke[jj * m + i] += factor * s;
            }
        }
    }
}

// solid_stresses, element.rs:270-302 (no thermal strain on this path: strain_e empty, e = 0).
// out per Gauss point: x, y, z, sxx, syy, szz, txy, tyz, txz (field order of results.rs:6-20).
void solid_stresses(int npe, const double (*coords)[3], const double d[6][6], const double* u_e,
                    double* out) {
    const TetGP* rule;
    const int ng = rule_of(npe, &rule);
    const int m = 3 * npe;
    double n[10], dn[10][3], dn_dx[10][3], b[30][6];
    for (int gp = 0; gp < ng; ++gp) {
        tet_shape(npe, rule[gp].xi, rule[gp].eta, rule[gp].zeta, n, dn);
        mapping3d(npe, coords, dn, dn_dx);
        b_columns(npe, dn_dx, b);
        double eps[6], sigma[6];
        for (int r = 0; r < 6; ++r) {
            double s = b[0][r] * u_e[0];
            for (int k = 1; k < m; ++k) s = s + b[k][r] * u_e[k];
            eps[r] = s - 0.0;
        }
        for (int r = 0; r < 6; ++r) {
            double s = d[r][0] * eps[0];
            for (int c = 1; c < 6; ++c) s = s + d[r][c] * eps[c];
            sigma[r] = s;
        }
        double at[3];
        for (int k = 0; k < 3; ++k) {
            double s = n[0] * coords[0][k];
            for (int i = 1; i < npe; ++i) s = s + n[i] * coords[i][k];
            at[k] = s;
        }
        double* o = out + 9 * gp;
        o[0] = at[0];
        o[1] = at[1];
        o[2] = at[2];
        o[3] = sigma[0];
        o[4] = sigma[1];
        o[5] = sigma[2];
        o[6] = sigma[5];  // tau_xy
        o[7] = sigma[3];  // tau_yz
        o[8] = sigma[4];  // tau_xz
    }
}

// Stress::von_mises, results.rs:24-32 (s in the layout written by solid_stresses)
double von_mises(const double* s) {
    const double a = s[3], b = s[4], c = s[5];
    const double shear = s[6] * s[6] + s[7] * s[7] + s[8] * s[8];
    const double v = a * a + b * b + c * c - a * b - b * c - c * a + 3.0 * shear;
    return std::sqrt(v > 0.0 ? v : 0.0);
}

// --- face pressure: src/assembly.rs:527-593 (tet branch 556-585), 650-674; mesh.rs:184-198 -----

int face_positions(int npe, int face, int* pos) {
    if (face < 0 || face > 3) return 0;
    const int a = TET_FACES[face][0], b = TET_FACES[face][1], c = TET_FACES[face][2];
    pos[0] = a;
    pos[1] = b;
    pos[2] = c;
    if (npe == 4) return 3;
    auto mid = [](int p, int q) {
        for (int k = 0; k < 6; ++k)
            if ((TET10_EDGES[k][0] == p && TET10_EDGES[k][1] == q) ||
                (TET10_EDGES[k][0] == q && TET10_EDGES[k][1] == p))
                return 4 + k;
        return 4;
    };
    pos[3] = mid(a, b);
    pos[4] = mid(b, c);
    pos[5] = mid(c, a);
    return 6;
}

// forces[3*k + c] for the k-th face node, positions in pos. Returns the number of face nodes.
int face_pressure(int npe, const double (*ecoords)[3], int face, double value, int* pos,
                  double* forces) {
    const int nn = face_positions(npe, face, pos);
    if (nn == 0) return 0;
    double c[6][3];
    for (int k = 0; k < nn; ++k)
        for (int q = 0; q < 3; ++q) c[k][q] = ecoords[pos[k]][q];
    double u[3], v[3];
    for (int k = 0; k < 3; ++k) {
        u[k] = c[1][k] - c[0][k];
        v[k] = c[2][k] - c[0][k];
    }
    const double cross[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2],
                             u[0] * v[1] - u[1] * v[0]};
    double sq = cross[0] * cross[0];
    sq = sq + cross[1] * cross[1];
    sq = sq + cross[2] * cross[2];
    const double twice_area = std::sqrt(sq);
    const TriGP* rule = (nn == 3) ? TRIANGLE_3 : TRIANGLE_6;
    const int np = (nn == 3) ? 3 : 6;
    double outward[3];
    for (int k = 0; k < 3; ++k)
        outward[k] = (c[0][k] + c[1][k] + c[2][k]) / 3.0 -
                     (ecoords[0][k] + ecoords[1][k] + ecoords[2][k] + ecoords[3][k]) / 4.0;
    double dot = cross[0] * outward[0];
    dot = dot + cross[1] * outward[1];
    dot = dot + cross[2] * outward[2];
    const double sign = dot < 0.0 ? -1.0 : 1.0;
    double normal[3];
    for (int k = 0; k < 3; ++k) normal[k] = sign * cross[k] / twice_area;
    for (int k = 0; k < 3 * nn; ++k) forces[k] = 0.0;
    for (int g = 0; g < np; ++g) {
        const double w = rule[g].w * twice_area;
        double nv[6];
        tri_values(nn, rule[g].xi, rule[g].eta, nv);
        for (int a = 0; a < nn; ++a)
            for (int q = 0; q < 3; ++q) forces[3 * a + q] -= value * w * nv[a] * normal[q];
    }
    return nn;
}

// --- sparse machinery: src/solve.rs, src/iterative.rs -----------------------------------------

// dot, solve.rs:100-110: 8 partial sums, fixed combine, sequential tail.
double dot(const double* a, const double* b, size_t n) {
    const size_t full = n / 8 * 8;
    double tail = 0.0;
    for (size_t k = full; k < n; ++k) tail = tail + a[k] * b[k];
    double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (size_t k = 0; k < full; k += 8)
        for (int l = 0; l < 8; ++l) s[l] += a[k + l] * b[k + l];
    return ((s[0] + s[1]) + (s[2] + s[3])) + ((s[4] + s[5]) + (s[6] + s[7])) + tail;
}

// Graph (CSR adjacency), iterative.rs:19-76
struct Graph {
    IVec offsets, targets;
    size_t len() const { return offsets.size() - 1; }
    size_t degree(size_t v) const { return offsets[v + 1] - offsets[v]; }
};

// Graph::from_elements, iterative.rs:38-76 (element lists given as CSR: eoff/eidx)
Graph graph_from_elements(size_t n, const IVec& eoff, const IVec& eidx) {
    const size_t ne = eoff.size() - 1;
    IVec incident(n + 1, 0);
    for (size_t e = 0; e < ne; ++e)
        for (size_t p = eoff[e]; p < eoff[e + 1]; ++p) incident[eidx[p] + 1] += 1;
    for (size_t v = 0; v < n; ++v) incident[v + 1] += incident[v];
    IVec cursor = incident;
    IVec of_vertex(incident[n]);
    for (size_t e = 0; e < ne; ++e)
        for (size_t p = eoff[e]; p < eoff[e + 1]; ++p) of_vertex[cursor[eidx[p]]++] = e;
    Graph g;
    g.offsets.reserve(n + 1);
    g.offsets.push_back(0);
    IVec mark(n, NONE);
    for (size_t v = 0; v < n; ++v) {
        mark[v] = v;
        for (size_t q = incident[v]; q < incident[v + 1]; ++q) {
            const size_t e = of_vertex[q];
            for (size_t p = eoff[e]; p < eoff[e + 1]; ++p) {
                const size_t w = eidx[p];
                if (mark[w] != v) {
                    mark[w] = v;
                    g.targets.push_back(w);
                }
            }
        }
        g.offsets.push_back(g.targets.size());
    }
    return g;
}

// bfs_levels, solve.rs:248-270
std::vector<IVec> bfs_levels(const Graph& g, size_t start, const std::vector<char>& excluded) {
    std::vector<char> seen = excluded;
    seen[start] = 1;
    std::vector<IVec> levels{IVec{start}};
    for (;;) {
        IVec next;
        for (size_t v : levels.back())
            for (size_t p = g.offsets[v]; p < g.offsets[v + 1]; ++p) {
                const size_t w = g.targets[p];
                if (!seen[w]) {
                    seen[w] = 1;
                    next.push_back(w);
                }
            }
        if (next.empty()) return levels;
        levels.push_back(std::move(next));
    }
}

// reverse_cuthill_mckee, solve.rs:200-245 (order[new] = old)
IVec reverse_cuthill_mckee(const Graph& g) {
    const size_t n = g.len();
    std::vector<char> visited(n, 0);
    IVec order;
    order.reserve(n);
    size_t scan_from = 0;  // every vertex before it is visited (same first minimum as a full scan)
    for (;;) {
        while (scan_from < n && visited[scan_from]) ++scan_from;
        size_t seed = NONE;
        for (size_t v = scan_from; v < n; ++v)
            if (!visited[v] && (seed == NONE || g.degree(v) < g.degree(seed))) seed = v;
        if (seed == NONE) break;
        size_t start = seed;
        auto levels = bfs_levels(g, start, visited);
        for (;;) {
            const IVec& last = levels.back();
            size_t far = NONE;
            for (size_t v : last)
                if (far == NONE || g.degree(v) < g.degree(far)) far = v;
            if (far == NONE) break;
            auto far_levels = bfs_levels(g, far, visited);
            if (far_levels.size() <= levels.size()) break;
            start = far;
            levels = std::move(far_levels);
        }
        const size_t first = order.size();
        visited[start] = 1;
        order.push_back(start);
        size_t head = first;
        while (head < order.size()) {
            const size_t v = order[head++];
            IVec next;
            for (size_t p = g.offsets[v]; p < g.offsets[v + 1]; ++p)
                if (!visited[g.targets[p]]) next.push_back(g.targets[p]);
            std::stable_sort(next.begin(), next.end(),
                             [&](size_t a, size_t b) { return g.degree(a) < g.degree(b); });
            for (size_t w : next)
                if (!visited[w]) {
                    visited[w] = 1;
                    order.push_back(w);
                }
        }
    }
    std::reverse(order.begin(), order.end());
    return order;
}

// Csr: lower triangle incl. diagonal, columns ascending, diagonal last. iterative.rs:82-189
struct Csr {
    IVec offsets, cols;
    Vec values;
    size_t n() const { return offsets.size() - 1; }

    // Csr::zeros, iterative.rs:91-114
    static Csr zeros(const Graph& g, const IVec& order, const IVec& rank) {
        Csr m;
        m.offsets.reserve(order.size() + 1);
        m.offsets.push_back(0);
        for (size_t r = 0; r < order.size(); ++r) {
            const size_t v = order[r];
            const size_t start = m.cols.size();
            for (size_t p = g.offsets[v]; p < g.offsets[v + 1]; ++p) {
                const size_t c = rank[g.targets[p]];
                if (c < r) m.cols.push_back(c);
            }
            std::sort(m.cols.begin() + start, m.cols.end());
            m.cols.push_back(r);
            m.offsets.push_back(m.cols.size());
        }
        m.values.assign(m.cols.size(), 0.0);
        return m;
    }

    // Csr::add, iterative.rs:121-128. Returns false when the entry is outside the profile.
    bool add(size_t i, size_t j, double v) {
        if (j > i) std::swap(i, j);
        auto b = cols.begin() + offsets[i], e = cols.begin() + offsets[i + 1];
        auto it = std::lower_bound(b, e, j);
        if (it == e || *it != j) return false;
        values[it - cols.begin()] += v;
        return true;
    }

    // Csr::multiply, iterative.rs:131-142
    void multiply(const double* x, double* y) const {
        const size_t nn = n();
        std::fill(y, y + nn, 0.0);
        for (size_t i = 0; i < nn; ++i) {
            const size_t start = offsets[i], diag = offsets[i + 1] - 1;
            double s = values[diag] * x[i];
            for (size_t p = start; p < diag; ++p) {
                s += values[p] * x[cols[p]];
                y[cols[p]] += values[p] * x[i];
            }
            y[i] += s;
        }
    }

    // Csr::incomplete_cholesky, iterative.rs:146-170
    std::optional<Vec> incomplete_cholesky(double shift) const {
        const size_t nn = n();
        Vec l(values.size(), 0.0), w(nn, 0.0);
        for (size_t i = 0; i < nn; ++i) {
            const size_t start = offsets[i], diag = offsets[i + 1] - 1;
            for (size_t p = start; p < diag; ++p) {
                const size_t j = cols[p];
                const size_t js = offsets[j], jd = offsets[j + 1] - 1;
                double s = 0.0;
                for (size_t q = js; q < jd; ++q) s = s + l[q] * w[cols[q]];
                l[p] = (values[p] - s) / l[jd];
                w[j] = l[p];
            }
            double squares = 0.0;
            for (size_t p = start; p < diag; ++p) squares = squares + l[p] * l[p];
            const double pivot = values[diag] * (1.0 + shift) - squares;
            if (std::isnan(pivot) || pivot <= 1e-12 * values[diag]) return std::nullopt;
            l[diag] = std::sqrt(pivot);
            for (size_t p = start; p < diag; ++p) w[cols[p]] = 0.0;
        }
        return l;
    }

    // Csr::precondition, iterative.rs:173-188
    void precondition(const Vec& l, const double* r, double* z) const {
        const size_t nn = n();
        std::copy(r, r + nn, z);
        for (size_t i = 0; i < nn; ++i) {
            const size_t start = offsets[i], diag = offsets[i + 1] - 1;
            double s = 0.0;
            for (size_t p = start; p < diag; ++p) s = s + l[p] * z[cols[p]];
            z[i] = (z[i] - s) / l[diag];
        }
        for (size_t i = nn; i-- > 0;) {
            const size_t start = offsets[i], diag = offsets[i + 1] - 1;
            z[i] /= l[diag];
            for (size_t p = start; p < diag; ++p) z[cols[p]] -= l[p] * z[i];
        }
    }
};

struct SolveStats {
    size_t iterations = 0;
    double rel_residual = 0.0;
    double shift = 0.0;
};

// Pcg::new + Pcg::solve, iterative.rs:201-248. tol replaces the TOLERANCE constant (default 1e-12).
int pcg_solve(const Csr& a, const Vec& b, double tol, size_t max_iter, Vec& x, SolveStats& st,
              const Vec* l_given = nullptr) {
    Vec l;
    if (l_given) {
        l = *l_given;
    } else {
        bool ok = false;
        for (double shift : SHIFTS) {
            auto got = a.incomplete_cholesky(shift);
            if (got) {
                l = std::move(*got);
                st.shift = shift;
                ok = true;
                break;
            }
        }
        if (!ok) return SINGULAR;
    }
    const size_t n = b.size();
    auto norm = [n](const Vec& v) { return std::sqrt(dot(v.data(), v.data(), n)); };
    const double b_norm = norm(b);
    x.assign(n, 0.0);
    st.iterations = 0;
    if (b_norm == 0.0) {
        st.rel_residual = 0.0;
        return OK;
    }
    Vec r = b, z(n), p(n), ap(n);
    a.precondition(l, r.data(), z.data());
    p = z;
    double rz = dot(r.data(), z.data(), n);
    for (size_t it = 0; it < max_iter; ++it) {
        a.multiply(p.data(), ap.data());
        const double curvature = dot(p.data(), ap.data(), n);
        if (std::isnan(curvature) || curvature <= 0.0) {
            st.iterations = it + 1;
            return SINGULAR;
        }
        const double alpha = rz / curvature;
        for (size_t k = 0; k < n; ++k) {
            x[k] += alpha * p[k];
            r[k] -= alpha * ap[k];
        }
        const double rn = norm(r);
        st.iterations = it + 1;
        st.rel_residual = rn / b_norm;
        if (rn <= tol * b_norm) return OK;
        a.precondition(l, r.data(), z.data());
        const double rz_next = dot(r.data(), z.data(), n);
        const double beta = rz_next / rz;
        rz = rz_next;
        for (size_t k = 0; k < n; ++k) p[k] = z[k] + beta * p[k];
    }
    st.rel_residual = norm(r) / b_norm;
    return NOT_CONVERGED;
}

// SkylineMatrix + Cholesky, solve.rs:10-139 (the direct solver, kept as a second oracle)
struct Skyline {
    IVec first, start;
    Vec data;
    explicit Skyline(IVec f) : first(std::move(f)) {
        start.assign(first.size() + 1, 0);
        for (size_t i = 0; i < first.size(); ++i) start[i + 1] = start[i] + i + 1 - first[i];
        data.assign(start.back(), 0.0);
    }
    size_t n() const { return first.size(); }
    double get(size_t i, size_t j) const {
        if (j > i) std::swap(i, j);
        return j < first[i] ? 0.0 : data[start[i] + j - first[i]];
    }
    void add(size_t i, size_t j, double v) {
        if (j > i) std::swap(i, j);
        data[start[i] + j - first[i]] += v;
    }
    // factorize, solve.rs:70-94
    int factorize() {
        const size_t nn = n();
        double max_diag = 0.0;
        for (size_t i = 0; i < nn; ++i) max_diag = std::fmax(max_diag, get(i, i));
        const double tol = 1e-12 * max_diag;
        for (size_t i = 0; i < nn; ++i) {
            const size_t fi = first[i];
            for (size_t j = fi; j <= i; ++j) {
                const size_t k0 = std::max(fi, first[j]);
                const size_t ri = start[i] - fi, rj = start[j] - first[j];
                const double s = dot(&data[ri + k0], &data[rj + k0], j - k0);
                const double a = data[ri + j] - s;
                if (i == j) {
                    if (std::isnan(a) || a <= tol) return SINGULAR;
                    data[ri + j] = std::sqrt(a);
                } else {
                    data[ri + j] = a / data[rj + j];
                }
            }
        }
        return OK;
    }
    // Cholesky::solve, solve.rs:118-138
    Vec solve(const Vec& b) const {
        Vec x = b;
        const size_t nn = n();
        for (size_t i = 0; i < nn; ++i) {
            const size_t fi = first[i];
            const double* row = &data[start[i]];
            double s = 0.0;
            for (size_t k = fi; k < i; ++k) s = s + row[k - fi] * x[k];
            x[i] = (x[i] - s) / row[i - fi];
        }
        for (size_t i = nn; i-- > 0;) {
            const size_t fi = first[i];
            const double* row = &data[start[i]];
            x[i] /= row[i - fi];
            for (size_t k = fi; k < i; ++k) x[k] -= row[k - fi] * x[i];
        }
        return x;
    }
};

double now_ms() {
    return std::chrono::duration<double, std::milli>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

// Element matrix of element e of a solid mesh (element_stiffness, assembly.rs:64-79, Tet branch)
struct SolidMesh {
    size_t n_nodes, n_elems;
    int npe;
    const double* coords;
    const int64_t* conn;
    const double* young;
    const double* poisson;
    void elem_coords(size_t e, double (*c)[3]) const {
        for (int a = 0; a < npe; ++a)
            for (int k = 0; k < 3; ++k) c[a][k] = coords[3 * conn[e * npe + a] + k];
    }
    void stiffness(size_t e, double* ke) const {
        double c[10][3], d[6][6];
        elem_coords(e, c);
        solid_d(young[e], poisson[e], d);
        solid_stiffness(npe, c, d, ke);
    }
};

// --- large strain: src/finite_strain.rs, model.rs:720-1022 -------------------------------------

// lame, finite_strain.rs:30-35
void lame(double young, double nu, double& lambda, double& mu) {
    lambda = young * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    mu = young / (2.0 * (1.0 + nu));
}

// mul / transpose / det / inverse, finite_strain.rs:89-117 (sums are left folds)
void mul3(const double a[3][3], const double b[3][3], double o[3][3]) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = a[i][0] * b[0][j];
            s = s + a[i][1] * b[1][j];
            s = s + a[i][2] * b[2][j];
            o[i][j] = s;
        }
}
double det3(const double a[3][3]) {
    return a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
           a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
}
void inv3(const double a[3][3], double o[3][3]) {
    const double d = det3(a);
    auto cof = [&](int i, int j) {
        const int r0 = (i + 1) % 3, r1 = (i + 2) % 3, c0 = (j + 1) % 3, c1 = (j + 2) % 3;
        return a[r0][c0] * a[r1][c1] - a[r0][c1] * a[r1][c0];
    };
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) o[i][j] = cof(j, i) / d;
}

// large_strain_response (finite_strain.rs:119-214) with LargeStrainLaw::NeoHookean
// (finite_strain.rs:40-86) on a Tet4 (solid_gauss with TETRA_1, element.rs:338-357): internal
// force fe [12], tangent ke [12 x 12] row-major, and the derivatives of fe with respect to mu and
// lambda at fixed u (dS/dmu = I - C^-1, dS/dlambda = ln J C^-1 from the same law; the reference
// has no gradients). Returns false when J <= 0 makes the law non-finite.
bool neo_hookean_tet4(const double c[4][3], double lambda, double mu, const double* ue, double* fe, double* ke,
                      double* dfe_dmu, double* dfe_dlambda) {
    double n[10], dn[10][3], dn_dx[10][3];
    const TetGP& gp = TETRA_1[0];
    tet_shape(4, gp.xi, gp.eta, gp.zeta, n, dn);
    const double weight = gp.w * std::fabs(mapping3d(4, c, dn, dn_dx));
    double f[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int a = 0; a < 4; ++a)
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) f[i][j] += ue[3 * a + i] * dn_dx[a][j];
    double ft[3][3], cc[3][3], inv[3][3], s[3][3], pk1[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) ft[i][j] = f[j][i];
    mul3(ft, f, cc);
    const double log_j = std::log(det3(f));
    inv3(cc, inv);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) s[i][j] = mu * ((i == j ? 1.0 : 0.0) - inv[i][j]) + lambda * log_j * inv[i][j];
    mul3(f, s, pk1);
    static thread_local double mod[3][3][3][3], A[3][3][3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k)
                for (int l = 0; l < 3; ++l)
                    mod[i][j][k][l] = lambda * inv[i][j] * inv[k][l] +
                                      (mu - lambda * log_j) * (inv[i][k] * inv[j][l] + inv[i][l] * inv[j][k]);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k)
                for (int l = 0; l < 3; ++l) {
                    double material = 0.0;
                    for (int ii = 0; ii < 3; ++ii)
                        for (int kk = 0; kk < 3; ++kk) material += f[i][ii] * mod[ii][j][kk][l] * f[k][kk];
                    const double geometric = i == k ? s[j][l] : 0.0;
                    A[i][j][k][l] = geometric + material;
                }
    std::fill(fe, fe + 12, 0.0);
    std::fill(ke, ke + 144, 0.0);
    for (int na = 0; na < 4; ++na) {
        const double* ga = dn_dx[na];
        for (int i = 0; i < 3; ++i) {
            const int row = 3 * na + i;
            double fr = pk1[i][0] * ga[0];
            fr = fr + pk1[i][1] * ga[1];
            fr = fr + pk1[i][2] * ga[2];
            fe[row] += weight * fr;
            for (int nb = 0; nb < 4; ++nb) {
                const double* gb = dn_dx[nb];
                for (int k = 0; k < 3; ++k) {
                    double v = 0.0;
                    for (int j = 0; j < 3; ++j)
                        for (int l = 0; l < 3; ++l) v += ga[j] * A[i][j][k][l] * gb[l];
                    ke[row * 12 + 3 * nb + k] += weight * v;
                }
            }
        }
    }
    if (dfe_dmu || dfe_dlambda) {
        double ds_mu[3][3], ds_la[3][3], dp_mu[3][3], dp_la[3][3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                ds_mu[i][j] = (i == j ? 1.0 : 0.0) - inv[i][j];
                ds_la[i][j] = log_j * inv[i][j];
            }
        mul3(f, ds_mu, dp_mu);
        mul3(f, ds_la, dp_la);
        for (int na = 0; na < 4; ++na)
            for (int i = 0; i < 3; ++i) {
                const double* ga = dn_dx[na];
                if (dfe_dmu) dfe_dmu[3 * na + i] = weight * (dp_mu[i][0] * ga[0] + dp_mu[i][1] * ga[1] + dp_mu[i][2] * ga[2]);
                if (dfe_dlambda)
                    dfe_dlambda[3 * na + i] = weight * (dp_la[i][0] * ga[0] + dp_la[i][1] * ga[1] + dp_la[i][2] * ga[2]);
            }
    }
    return std::isfinite(log_j);
}

// The topology part of FreeSystem::new (model.rs:1449-1466): free numbering, RCM rank and the
// lower CSR profile. The reference rebuilds it at every Newton iteration (model.rs:1011) from
// the same pattern; it is built once here, with the same result.
struct FreeTopology {
    IVec free, rank;
    size_t count = 0;
    Csr pattern;
};

FreeTopology free_topology(size_t n_elems, const int64_t* conn, const uint8_t* fixed, size_t n) {
    FreeTopology t;
    t.free.assign(n, NONE);
    for (size_t g = 0; g < n; ++g)
        if (!fixed[g]) t.free[g] = t.count++;
    IVec eoff(n_elems + 1, 0), eidx;
    for (size_t e = 0; e < n_elems; ++e) {
        for (int l = 0; l < 12; ++l) {
            const size_t g = 3 * (size_t)conn[e * 4 + l / 3] + l % 3;
            if (t.free[g] != NONE) eidx.push_back(t.free[g]);
        }
        eoff[e + 1] = eidx.size();
    }
    Graph graph = graph_from_elements(t.count, eoff, eidx);
    IVec order = reverse_cuthill_mckee(graph);
    t.rank.assign(t.count, 0);
    for (size_t r = 0; r < t.count; ++r) t.rank[order[r]] = r;
    t.pattern = Csr::zeros(graph, order, t.rank);
    return t;
}

struct LargeStrainMesh {
    size_t n_nodes, n_elems;
    const double* coords;
    const int64_t* conn;
    Vec lambda, mu;  // per element, from lame(E, nu) as large_strain_law does (assembly.rs:55-61)
    void coords_of(size_t e, double c[4][3]) const {
        for (int a = 0; a < 4; ++a)
            for (int k = 0; k < 3; ++k) c[a][k] = coords[3 * conn[e * 4 + a] + k];
    }
};

// FreeSystem::new (values) + FreeSystem::solve (model.rs:1442-1516) with the iterative factor:
// K_ff x_f = f_f - K_fc u_c, written into u at free DOFs. `tangents` holds 144 values per element.
int free_solve(const FreeTopology& t, const LargeStrainMesh& m, const Vec& tangents, const Vec& f, Vec& u,
               double pcg_tol, size_t pcg_max, size_t& pcg_iters) {
    Csr k = t.pattern;
    std::fill(k.values.begin(), k.values.end(), 0.0);
    Vec coupling(t.count, 0.0);
    for (size_t e = 0; e < m.n_elems; ++e) {
        const double* ke = &tangents[e * 144];
        for (int r = 0; r < 12; ++r) {
            const size_t gi = 3 * (size_t)m.conn[e * 4 + r / 3] + r % 3;
            const size_t a = t.free[gi];
            if (a == NONE) continue;
            for (int c = 0; c < 12; ++c) {
                const size_t gj = 3 * (size_t)m.conn[e * 4 + c / 3] + c % 3;
                const size_t b = t.free[gj];
                if (b != NONE) {
                    if (t.rank[b] <= t.rank[a]) k.add(t.rank[a], t.rank[b], ke[r * 12 + c]);
                } else {
                    coupling[t.rank[a]] += ke[r * 12 + c] * u[gj];
                }
            }
        }
    }
    Vec rhs(t.count);
    for (size_t q = 0; q < t.count; ++q) rhs[q] = -coupling[q];
    for (size_t g = 0; g < t.free.size(); ++g)
        if (t.free[g] != NONE) rhs[t.rank[t.free[g]]] += f[g];
    Vec x;
    SolveStats st;
    const int status = pcg_solve(k, rhs, pcg_tol, pcg_max, x, st);
    pcg_iters += st.iterations;
    if (status != OK) return status;
    for (size_t g = 0; g < t.free.size(); ++g)
        if (t.free[g] != NONE) u[g] = x[t.rank[t.free[g]]];
    return OK;
}

// Element responses at u: internal force (internal_force, model.rs:1241-1249) and tangents.
bool responses(const LargeStrainMesh& m, const Vec& u, Vec& internal, Vec& tangents) {
    internal.assign(3 * m.n_nodes, 0.0);
    tangents.resize(m.n_elems * 144);
    bool finite = true;
    for (size_t e = 0; e < m.n_elems; ++e) {
        double c[4][3], ue[12], fe[12];
        m.coords_of(e, c);
        for (int l = 0; l < 12; ++l) ue[l] = u[3 * (size_t)m.conn[e * 4 + l / 3] + l % 3];
        finite = neo_hookean_tet4(c, m.lambda[e], m.mu[e], ue, fe, &tangents[e * 144], nullptr, nullptr) && finite;
        for (int l = 0; l < 12; ++l) internal[3 * (size_t)m.conn[e * 4 + l / 3] + l % 3] += fe[l];
    }
    return finite;
}

constexpr double NEWTON_TOLERANCE = 1e-8;  // model.rs:1220
constexpr size_t NEWTON_ITERATIONS = 25;   // model.rs:1222
constexpr int MAX_CUTS = 5;                // model.rs:1224

struct QuasiStatic {
    const LargeStrainMesh& m;
    const FreeTopology& t;
    const uint8_t* fixed;
    const double* imposed;
    const double* loads;
    double newton_tol, pcg_tol;
    size_t newton_max, pcg_max;
    size_t pcg_iters = 0, newton_total = 0;
    Vec u;
    double scale = 0.0;

    // equilibrium, model.rs:923-1022 (no contacts, no follower pressures): Newton-Raphson to
    // F_int(u) = lambda F with imposed values lambda * imposed. Returns the status; on success
    // `reactions` = F_int - lambda F at fixed DOFs and `iterations` = residuals computed.
    int equilibrium(Vec& uu, double lam, double& sc, Vec& reactions, size_t& iterations) {
        const size_t n = uu.size();
        Vec internal, tangents, residual(n), external(n);
        size_t count = 0;
        for (;;) {
            responses(m, uu, internal, tangents);
            for (size_t g = 0; g < n; ++g) {
                external[g] = lam * (loads ? loads[g] : 0.0);
                residual[g] = internal[g] - external[g];
            }
            double ni = 0.0, ne = 0.0, nf = 0.0;
            for (size_t g = 0; g < n; ++g) {
                ni += internal[g] * internal[g];
                ne += external[g] * external[g];
                if (!fixed[g]) nf += residual[g] * residual[g];
            }
            sc = std::max(std::max(sc, std::sqrt(ni)), std::sqrt(ne));
            const double free = std::sqrt(nf);
            const double relative = sc > 0.0 ? free / sc : free;
            if (!std::isfinite(relative)) return NOT_CONVERGED;
            ++count;
            ++newton_total;
            if (count > 1 && relative <= newton_tol) {
                reactions.assign(n, 0.0);
                for (size_t g = 0; g < n; ++g)
                    if (fixed[g]) reactions[g] = residual[g];
                iterations = count;
                return OK;
            }
            if (count > newton_max) return NOT_CONVERGED;
            Vec du(n, 0.0), minus(n);
            for (size_t g = 0; g < n; ++g) {
                if (fixed[g]) du[g] = lam * imposed[g] - uu[g];
                minus[g] = -residual[g];
            }
            const int st = free_solve(t, m, tangents, minus, du, pcg_tol, pcg_max, pcg_iters);
            if (st == NOT_CONVERGED) return ITERATIVE_NOT_CONVERGED;
            if (st != OK) return st;
            for (size_t g = 0; g < n; ++g) uu[g] += du[g];
        }
    }

    // advance, model.rs:820-870: Newton from the committed state, halving the interval up to
    // MAX_CUTS times when Newton fails or meets a non-positive-definite tangent (NotConverged or
    // Singular, model.rs:839-842); an inner PCG at its cap is passed up without a cut.
    int advance(double t0, double t1, int cuts, Vec& reactions, size_t& iterations, int& cut_count) {
        Vec trial = u;
        double sc = scale;
        const int st = equilibrium(trial, t1, sc, reactions, iterations);  // amplitude lambda(t) = t
        if (st == OK) {
            u = trial;
            scale = sc;
            return OK;
        }
        if ((st == NOT_CONVERGED || st == SINGULAR) && cuts < MAX_CUTS) {
            const double middle = (t0 + t1) / 2.0;
            ++cut_count;
            const int a = advance(t0, middle, cuts + 1, reactions, iterations, cut_count);
            if (a != OK) return a;
            return advance(middle, t1, cuts + 1, reactions, iterations, cut_count);
        }
        return st;
    }
};

// --- transient heat conduction: model.rs:621-706 (solve_step_with), assembly.rs:386-484 and
// 485-626 (thermal element matrices, sources, convection), element.rs:338-357 and 451-506 -----

// TETRA_14, quadrature.rs:140-177: the published 14-point degree-5 rule on the reference
// tetrahedron (weights sum to 1/6), points in the reference's order: two orbits of 4 points
// (a, a, a) and their permutations with 1 - 3a, one orbit of 6 points on the edge midlines.
constexpr double T14_A1 = 0.09273525031089142, T14_W1 = 0.01224884051939372;
constexpr double T14_A2 = 0.3108859192633008, T14_W2 = 0.01878132095300283;
constexpr double T14_B = 0.04550370412564851, T14_W3 = 0.00709100346284674;
struct Tetra14 {
    TetGP p[14];
    Tetra14() {
        int k = 0;
        auto orbit4 = [&](double a, double w) {  // (a, a, a) and its three moves to 1 - 3a
            const double c = 1.0 - 3.0 * a;
            p[k++] = {a, a, a, w};
            p[k++] = {c, a, a, w};
            p[k++] = {a, c, a, w};
            p[k++] = {a, a, c, w};
        };
        orbit4(T14_A1, T14_W1);
        orbit4(T14_A2, T14_W2);
        const double b = T14_B, d = 0.5 - T14_B;  // the six (b, b, d) permutations
        p[k++] = {b, b, d, T14_W3};
        p[k++] = {b, d, b, T14_W3};
        p[k++] = {d, b, b, T14_W3};
        p[k++] = {d, d, b, T14_W3};
        p[k++] = {d, b, d, T14_W3};
        p[k++] = {b, d, d, T14_W3};
    }
};
const Tetra14 TETRA_14;

// GaussData of solid_gauss, element.rs:338-357: weight w |det J|, N, dN/dx, position sum N x.
struct GaussData {
    double w;
    double n[10];
    double g[10][3];
    double at[3];
};

int solid_gauss(int npe, const double (*c)[3], const TetGP* rule, int ng, GaussData* out) {
    double dn[10][3];
    for (int gp = 0; gp < ng; ++gp) {
        GaussData& d = out[gp];
        tet_shape(npe, rule[gp].xi, rule[gp].eta, rule[gp].zeta, d.n, dn);
        const double det = mapping3d(npe, c, dn, d.g);
        d.w = rule[gp].w * std::fabs(det);
        for (int k = 0; k < 3; ++k) {
            double s = d.n[0] * c[0][k];
            for (int a = 1; a < npe; ++a) s = s + d.n[a] * c[a][k];
            d.at[k] = s;
        }
    }
    return ng;
}

// conduction, element.rs:451-463: K = sum_g w k grad N grad N^T (npe x npe row-major)
void conduction(int npe, const GaussData* p, int ng, double k, double* ke) {
    std::fill(ke, ke + npe * npe, 0.0);
    for (int gp = 0; gp < ng; ++gp)
        for (int a = 0; a < npe; ++a)
            for (int b = 0; b < npe; ++b) {
                const double* ga = p[gp].g[a];
                const double* gb = p[gp].g[b];
                double s = ga[0] * gb[0];
                s = s + ga[1] * gb[1];
                s = s + ga[2] * gb[2];
                ke[a * npe + b] += p[gp].w * k * s;
            }
}

// capacity, element.rs:465-477: C = sum_g w rho_c N N^T, on a rule exact for N N^T
// (element_capacity, assembly.rs:413-433: TETRA_4 for Tet4, TETRA_14 for Tet10)
void capacity(int npe, const GaussData* p, int ng, double rho_c, double* ce) {
    std::fill(ce, ce + npe * npe, 0.0);
    for (int gp = 0; gp < ng; ++gp)
        for (int a = 0; a < npe; ++a)
            for (int b = 0; b < npe; ++b) ce[a * npe + b] += p[gp].w * rho_c * p[gp].n[a] * p[gp].n[b];
}

// FaceConvection of face_convection, assembly.rs:486-509 and 595-626: matrix = h int N N^T dS,
// load = h T_inf int N dS over the face rule of face_rule (the geometry of face_pressure above).
struct Convection {
    int nn = 0;
    int pos[6];
    double matrix[36];
    double load[6];
};

bool face_convection(int npe, const double (*ecoords)[3], int face, double film, double sink, Convection& out) {
    const int nn = face_positions(npe, face, out.pos);
    if (nn == 0) return false;
    out.nn = nn;
    double c[6][3];
    for (int k = 0; k < nn; ++k)
        for (int q = 0; q < 3; ++q) c[k][q] = ecoords[out.pos[k]][q];
    double u[3], v[3];
    for (int k = 0; k < 3; ++k) {
        u[k] = c[1][k] - c[0][k];
        v[k] = c[2][k] - c[0][k];
    }
    const double cross[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2],
                             u[0] * v[1] - u[1] * v[0]};
    double sq = cross[0] * cross[0];
    sq = sq + cross[1] * cross[1];
    sq = sq + cross[2] * cross[2];
    const double twice_area = std::sqrt(sq);
    const TriGP* rule = (nn == 3) ? TRIANGLE_3 : TRIANGLE_6;
    const int np = (nn == 3) ? 3 : 6;
    std::fill(out.matrix, out.matrix + 36, 0.0);
    std::fill(out.load, out.load + 6, 0.0);
    for (int g = 0; g < np; ++g) {
        const double w = rule[g].w * twice_area;
        double nv[6];
        tri_values(nn, rule[g].xi, rule[g].eta, nv);
        for (int a = 0; a < nn; ++a) {
            out.load[a] += film * sink * w * nv[a];
            for (int b = 0; b < nn; ++b) out.matrix[a * nn + b] += film * w * nv[a] * nv[b];
        }
    }
    return true;
}

// heat_fluxes, element.rs:480-506: per Gauss point x, y, z, qx, qy, qz with q = -k grad T
void heat_fluxes(int npe, const GaussData* p, int ng, double k, const double* t_e, double* out) {
    for (int gp = 0; gp < ng; ++gp) {
        double* o = out + 6 * gp;
        for (int c = 0; c < 3; ++c) o[c] = p[gp].at[c];
        for (int c = 0; c < 3; ++c) {
            double s = p[gp].g[0][c] * t_e[0];
            for (int a = 1; a < npe; ++a) s = s + p[gp].g[a][c] * t_e[a];
            o[3 + c] = -k * s;
        }
    }
}

}  // namespace

// ============================================================================================
// C ABI used by the tests and bench (ctypes). Everything below is test infrastructure.
// ============================================================================================
extern "C" {

// element_stiffness of one Tet4/Tet10 (coords npe x 3), ke: (3npe)^2 row-major
void oracle_element_stiffness(int npe, const double* coords, double young, double nu, double* ke) {
    double d[6][6];
    solid_d(young, nu, d);
    solid_stiffness(npe, reinterpret_cast<const double(*)[3]>(coords), d, ke);
}

// element_stresses of one element: out ngp x 9 (x, y, z, sxx, syy, szz, txy, tyz, txz)
void oracle_element_stresses(int npe, const double* coords, double young, double nu,
                             const double* u_e, double* out) {
    double d[6][6];
    solid_d(young, nu, d);
    solid_stresses(npe, reinterpret_cast<const double(*)[3]>(coords), d, u_e, out);
}

double oracle_von_mises(const double* s9) { return von_mises(s9); }

// face_pressure of one element: positions (<=6) and forces (3 per face node). Returns node count.
int oracle_face_pressure(int npe, const double* coords, int face, double value, int* positions,
                         double* forces) {
    return face_pressure(npe, reinterpret_cast<const double(*)[3]>(coords), face, value, positions,
                         forces);
}

double oracle_dot(const double* a, const double* b, int64_t n) { return dot(a, b, (size_t)n); }

// Graph::from_elements. Call with out_targets = NULL to get the target count.
int64_t oracle_graph_from_elements(int64_t n, int64_t n_el, const int64_t* eoff,
                                   const int64_t* eidx, int64_t* out_offsets,
                                   int64_t* out_targets) {
    IVec o(eoff, eoff + n_el + 1), ix(eidx, eidx + eoff[n_el]);
    Graph g = graph_from_elements((size_t)n, o, ix);
    if (out_offsets)
        for (size_t v = 0; v <= (size_t)n; ++v) out_offsets[v] = (int64_t)g.offsets[v];
    if (out_targets)
        for (size_t p = 0; p < g.targets.size(); ++p) out_targets[p] = (int64_t)g.targets[p];
    return (int64_t)g.targets.size();
}

// reverse_cuthill_mckee on a CSR adjacency
void oracle_rcm(int64_t n, const int64_t* offsets, const int64_t* targets, int64_t* order) {
    Graph g;
    g.offsets.assign(offsets, offsets + n + 1);
    g.targets.assign(targets, targets + offsets[n]);
    IVec o = reverse_cuthill_mckee(g);
    for (size_t k = 0; k < o.size(); ++k) order[k] = (int64_t)o[k];
}

// A Csr built on `graph` in numbering `order` (identity when order == NULL), filled with
// triplets (Csr::add in the renumbered indices ti, tj). mode 0: Pcg::new + Pcg::solve(b) -> x;
// mode 1: incomplete_cholesky(0) + precondition(b) -> x; mode 2: multiply(b) -> x.
// Returns the status (0 OK, 1 SINGULAR, 2 NOT_CONVERGED, 3 outside profile).
int oracle_csr_run(int64_t n, const int64_t* offsets, const int64_t* targets, const int64_t* order,
                   int64_t nt, const int64_t* ti, const int64_t* tj, const double* tv,
                   const double* b, int mode, double tol, double* x, int64_t* iterations) {
    Graph g;
    g.offsets.assign(offsets, offsets + n + 1);
    g.targets.assign(targets, targets + offsets[n]);
    IVec ord(n), rank(n);
    for (int64_t k = 0; k < n; ++k) ord[k] = order ? (size_t)order[k] : (size_t)k;
    for (int64_t k = 0; k < n; ++k) rank[ord[k]] = (size_t)k;
    Csr a = Csr::zeros(g, ord, rank);
    for (int64_t t = 0; t < nt; ++t)
        if (!a.add((size_t)ti[t], (size_t)tj[t], tv[t])) return INVALID;
    Vec bb(b, b + n), xx(n);
    if (mode == 2) {
        a.multiply(bb.data(), xx.data());
    } else if (mode == 1) {
        auto l = a.incomplete_cholesky(0.0);
        if (!l) return SINGULAR;
        a.precondition(*l, bb.data(), xx.data());
    } else {
        SolveStats st;
        int s = pcg_solve(a, bb, tol, MAX_ITERATIONS, xx, st);
        if (iterations) *iterations = (int64_t)st.iterations;
        if (s != OK) return s;
    }
    std::copy(xx.begin(), xx.end(), x);
    return OK;
}

// Model::solve for a linear static Tet4/Tet10 model (model.rs:548-610 with assemble 1070-1147,
// FreeSystem::new/solve 1442-1516, product 1353-1369, element_stresses 304-312).
//   loads: nodal load vector (3 n_nodes; the sum of the model's Loads at their DOFs)
//   pressures: (element, face, value) triples added through face_pressure + add_load
//   solver: 0 Auto, 1 Direct, 2 Iterative (SolverKind, solve.rs:170-195)
//   tol: PCG relative-residual tolerance (the reference's constant is 1e-12; 0 selects it)
//   dof_order: optional permutation of the free DOFs (order[new] = old free index) that replaces
//              RCM; NULL keeps reverse_cuthill_mckee. Used to check the GPU ordering's factor.
//   out: u, reactions (3 n_nodes), gauss (n_elems*ngp*9), vm (n_elems*ngp), f_out (3 n_nodes),
//        info[0..7] = iterations, rel_residual, shift, free dofs, nnz(L), ms setup, ms factor, ms pcg
int oracle_model_solve(int64_t n_nodes, const double* coords, int npe, int64_t n_elems,
                       const int64_t* conn, const double* young, const double* poisson,
                       const uint8_t* fixed, const double* imposed, const double* loads,
                       int64_t n_press, const int64_t* p_elem, const int32_t* p_face,
                       const double* p_value, int solver, double tol, int64_t max_iter,
                       const int64_t* dof_order, double* u, double* reactions, double* gauss,
                       double* vm, double* f_out, double* info) {
    if (tol <= 0.0) tol = TOLERANCE;
    if (max_iter <= 0) max_iter = (int64_t)MAX_ITERATIONS;
    const double t0 = now_ms();
    SolidMesh mesh{(size_t)n_nodes, (size_t)n_elems, npe, coords, conn, young, poisson};
    const size_t n = 3 * (size_t)n_nodes;
    const int m = 3 * npe;
    // assemble, model.rs:1070-1147: element DOFs (element_dofs, assembly.rs:20-32), loads,
    // pressures, imposed/fixed
    Vec f(n, 0.0);
    for (size_t g = 0; g < n; ++g) f[g] += loads ? loads[g] : 0.0;
    for (int64_t k = 0; k < n_press; ++k) {
        const size_t e = (size_t)p_elem[k];
        double c[10][3], forces[18];
        int pos[6];
        mesh.elem_coords(e, c);
        const int nn = face_pressure(npe, c, p_face[k], p_value[k], pos, forces);
        for (int a = 0; a < nn; ++a)
            for (int q = 0; q < 3; ++q)
                f[3 * (size_t)conn[e * npe + pos[a]] + q] += forces[3 * a + q];
    }
    auto dof = [&](size_t e, int l) { return 3 * (size_t)conn[e * npe + l / 3] + l % 3; };
    Vec uu(n);
    for (size_t g = 0; g < n; ++g) uu[g] = fixed[g] ? imposed[g] : 0.0;

    // FreeSystem::new, model.rs:1442-1499
    IVec free(n, NONE);
    size_t count = 0;
    for (size_t g = 0; g < n; ++g)
        if (!fixed[g]) free[g] = count++;
    IVec eoff(mesh.n_elems + 1, 0), eidx;
    for (size_t e = 0; e < mesh.n_elems; ++e) {
        for (int l = 0; l < m; ++l)
            if (free[dof(e, l)] != NONE) eidx.push_back(free[dof(e, l)]);
        eoff[e + 1] = eidx.size();
    }
    Graph graph = graph_from_elements(count, eoff, eidx);
    IVec order;
    if (dof_order) {
        order.assign(count, 0);
        for (size_t k = 0; k < count; ++k) order[k] = (size_t)dof_order[k];
    } else {
        order = reverse_cuthill_mckee(graph);
    }
    IVec rank(count);
    for (size_t r = 0; r < count; ++r) rank[order[r]] = r;
    const bool iterative = solver == 2 || (solver == 0 && count >= ITERATIVE_FROM);
    Csr csr;
    std::optional<Skyline> sky;
    if (iterative) {
        csr = Csr::zeros(graph, order, rank);
    } else {
        IVec first(count);
        for (size_t a = 0; a < count; ++a) first[a] = a;
        for (size_t a = 0; a < count; ++a)
            for (size_t p = graph.offsets[a]; p < graph.offsets[a + 1]; ++p)
                first[rank[a]] = std::min(first[rank[a]], rank[graph.targets[p]]);
        sky.emplace(first);
    }
    graph = Graph{};
    Vec coupling(count, 0.0);
    Vec ke((size_t)m * m);
    for (size_t e = 0; e < mesh.n_elems; ++e) {
        mesh.stiffness(e, ke.data());
        for (int r = 0; r < m; ++r) {
            const size_t a = free[dof(e, r)];
            if (a == NONE) continue;
            for (int c = 0; c < m; ++c) {
                const size_t b = free[dof(e, c)];
                const double k = ke[(size_t)r * m + c];
                if (b != NONE) {
                    if (rank[b] <= rank[a]) {
                        if (iterative)
                            csr.add(rank[a], rank[b], k);
                        else
                            sky->add(rank[a], rank[b], k);
                    }
                } else {
                    coupling[rank[a]] += k * uu[dof(e, c)];
                }
            }
        }
    }
    const double t1 = now_ms();
    // FreeSystem::solve, model.rs:1502-1516
    Vec rhs(count);
    for (size_t k = 0; k < count; ++k) rhs[k] = -coupling[k];
    for (size_t g = 0; g < n; ++g)
        if (free[g] != NONE) rhs[rank[free[g]]] += f[g];
    Vec x;
    SolveStats st;
    int status = OK;
    double t2 = t1;
    if (iterative) {
        Vec l;
        bool ok = false;
        for (double shift : SHIFTS) {
            auto got = csr.incomplete_cholesky(shift);
            if (got) {
                l = std::move(*got);
                st.shift = shift;
                ok = true;
                break;
            }
        }
        t2 = now_ms();
        if (!ok)
            status = SINGULAR;
        else
            status = pcg_solve(csr, rhs, tol, (size_t)max_iter, x, st, &l);
    } else {
        status = sky->factorize();
        t2 = now_ms();
        if (status == OK) x = sky->solve(rhs);
    }
    const double t3 = now_ms();
    if (info) {
        info[0] = (double)st.iterations;
        info[1] = st.rel_residual;
        info[2] = st.shift;
        info[3] = (double)count;
        info[4] = iterative ? (double)csr.cols.size() : (double)sky->data.size();
        info[5] = t1 - t0;
        info[6] = t2 - t1;
        info[7] = t3 - t2;
    }
    if (f_out) std::copy(f.begin(), f.end(), f_out);
    if (status != OK) return status;
    for (size_t g = 0; g < n; ++g)
        if (free[g] != NONE) uu[g] = x[rank[free[g]]];
    std::copy(uu.begin(), uu.end(), u);

    // reactions = product(dofs, matrix, u, fixed) - f on fixed DOFs, model.rs:586-593, 1353-1369
    if (reactions) {
        Vec y(n, 0.0);
        for (size_t e = 0; e < mesh.n_elems; ++e) {
            bool any = false;
            for (int l = 0; l < m; ++l) any = any || fixed[dof(e, l)];
            if (!any) continue;
            mesh.stiffness(e, ke.data());
            for (int r = 0; r < m; ++r) {
                const size_t g = dof(e, r);
                if (!fixed[g]) continue;
                double s = 0.0;
                for (int c = 0; c < m; ++c) s = s + ke[(size_t)r * m + c] * uu[dof(e, c)];
                y[g] += s;
            }
        }
        for (size_t g = 0; g < n; ++g)
            if (fixed[g]) y[g] -= f[g];
        std::copy(y.begin(), y.end(), reactions);
    }
    // Gauss-point stresses and von Mises, element_stresses, assembly.rs:304-312
    if (gauss) {
        const int ng = npe == 4 ? 1 : 4;
        for (size_t e = 0; e < mesh.n_elems; ++e) {
            double c[10][3], d[6][6], ue[30];
            mesh.elem_coords(e, c);
            solid_d(young[e], poisson[e], d);
            for (int l = 0; l < m; ++l) ue[l] = uu[dof(e, l)];
            double* o = gauss + e * ng * 9;
            solid_stresses(npe, c, d, ue, o);
            if (vm)
                for (int gp = 0; gp < ng; ++gp) vm[e * ng + gp] = von_mises(o + 9 * gp);
        }
    }
    return OK;
}

// Energy v^T K v = sum_e v_e^T K_e v_e of a displacement-like vector v (3 n_nodes), with the
// element matrices of element_stiffness (assembly.rs:64-79). Used to measure energy-norm errors.
double oracle_energy(int64_t n_nodes, const double* coords, int npe, int64_t n_elems,
                     const int64_t* conn, const double* young, const double* poisson,
                     const double* v) {
    SolidMesh mesh{(size_t)n_nodes, (size_t)n_elems, npe, coords, conn, young, poisson};
    const int m = 3 * npe;
    Vec ke((size_t)m * m);
    double total = 0.0;
    for (size_t e = 0; e < mesh.n_elems; ++e) {
        mesh.stiffness(e, ke.data());
        double ve[30];
        for (int l = 0; l < m; ++l) ve[l] = v[3 * (size_t)conn[e * npe + l / 3] + l % 3];
        for (int r = 0; r < m; ++r) {
            double s = 0.0;
            for (int c = 0; c < m; ++c) s += ke[(size_t)r * m + c] * ve[c];
            total += ve[r] * s;
        }
    }
    return total;
}

// Per element a_e^T K_e b_e (K_e from solid_stiffness, element.rs:223-243). With a = lambda (the
// adjoint solution) and b = u it gives the adjoint sensitivity dJ/dE_e = -lambda_e^T K_e u_e / E_e,
// since K_e is linear in E_e; the reference has no gradients, so this is the oracle's restatement
// of that formula on top of its own element matrices.
void oracle_element_bilinear(int64_t n_nodes, const double* coords, int npe, int64_t n_elems,
                             const int64_t* conn, const double* young, const double* poisson,
                             const double* a, const double* b, double* out) {
    SolidMesh mesh{(size_t)n_nodes, (size_t)n_elems, npe, coords, conn, young, poisson};
    const int m = 3 * npe;
    Vec ke((size_t)m * m);
    for (size_t e = 0; e < mesh.n_elems; ++e) {
        mesh.stiffness(e, ke.data());
        double ae[30], be[30];
        for (int l = 0; l < m; ++l) {
            const size_t d = 3 * (size_t)conn[e * npe + l / 3] + l % 3;
            ae[l] = a[d];
            be[l] = b[d];
        }
        double total = 0.0;
        for (int r = 0; r < m; ++r) {
            double s = 0.0;
            for (int c = 0; c < m; ++c) s += ke[(size_t)r * m + c] * be[c];
            total += ae[r] * s;
        }
        out[e] = total;
    }
}

// nodal_stresses / smooth, results.rs:137-230: Gauss values extrapolated to the element nodes
// (TET4_EXTRAPOLATION 98, TET10_EXTRAPOLATION 118-132) and averaged. gauss: n_elems*ngp*9 as
// written above; out: n_nodes*6 (sxx, syy, szz, txy, tyz, txz).
void oracle_nodal_stresses(int64_t n_nodes, int npe, int64_t n_elems, const int64_t* conn,
                           const double* gauss, double* out) {
    const double V = 1.9270509831248424, M = 0.8090169943749475, O = -0.30901699437494745;
    const double T10[10][4] = {{V, O, O, O}, {O, V, O, O}, {O, O, V, O}, {O, O, O, V},
                               {M, M, O, O}, {O, M, M, O}, {M, O, M, O}, {M, O, O, M},
                               {O, M, O, M}, {O, O, M, M}};
    const int ng = npe == 4 ? 1 : 4;
    Vec sum((size_t)n_nodes * 6, 0.0);
    std::vector<size_t> count((size_t)n_nodes, 0);
    for (int64_t e = 0; e < n_elems; ++e) {
        for (int a = 0; a < npe; ++a) {
            const size_t nd = (size_t)conn[e * npe + a];
            for (int g = 0; g < ng; ++g) {
                const double w = npe == 4 ? 1.0 : T10[a][g];
                const double* p = gauss + (e * ng + g) * 9 + 3;
                for (int c = 0; c < 6; ++c) sum[nd * 6 + c] += w * p[c];
            }
            count[nd] += 1;
        }
    }
    for (int64_t k = 0; k < n_nodes; ++k)
        for (int c = 0; c < 6; ++c)
            out[k * 6 + c] = sum[k * 6 + c] / (double)std::max<size_t>(count[k], 1);
}


// Model::solve_quasi_static (model.rs:720-806) of a neo-Hookean Tet4 model in large strain
// (Kinematics::Large, Step::quasi_static(1, increments), linear amplitude (0,0)-(1,1), loads and
// imposed values scaled by lambda(t) = t), with IC(0)-PCG inner solves to pcg_tol. Per increment:
// the converged displacements (the checkpoints, [increments][3 n_nodes]), the reactions
// F_int - lambda F at fixed DOFs ([increments][3 n_nodes]), the Newton iterations of the last
// equilibrium and the cuts. info: [0] total Newton iterations, [1] total PCG iterations, [2] the
// cuts of the increment the run stopped at (the last one on success), [3] that increment.
int oracle_large_strain_run(int64_t n_nodes, const double* coords, int64_t n_elems, const int64_t* conn,
                            const double* young, const double* poisson, const uint8_t* fixed,
                            const double* imposed, const double* loads, int increments, double newton_tol,
                            int newton_max, double pcg_tol, int64_t pcg_max, double* u_hist, double* r_hist,
                            int32_t* newton_iters, int32_t* cuts, double* info) {
    LargeStrainMesh m{(size_t)n_nodes, (size_t)n_elems, coords, conn, {}, {}};
    m.lambda.resize(m.n_elems);
    m.mu.resize(m.n_elems);
    for (size_t e = 0; e < m.n_elems; ++e) lame(young[e], poisson[e], m.lambda[e], m.mu[e]);
    const size_t n = 3 * (size_t)n_nodes;
    FreeTopology t = free_topology(m.n_elems, conn, fixed, n);
    QuasiStatic qs{m, t, fixed, imposed, loads, newton_tol > 0 ? newton_tol : NEWTON_TOLERANCE,
                   pcg_tol > 0 ? pcg_tol : TOLERANCE, newton_max > 0 ? (size_t)newton_max : NEWTON_ITERATIONS,
                   pcg_max > 0 ? (size_t)pcg_max : MAX_ITERATIONS, 0, 0, Vec(n, 0.0), 0.0};
    const double dt = 1.0 / increments;
    for (int inc = 1; inc <= increments; ++inc) {
        const double time = inc * dt;
        Vec reactions;
        size_t iterations = 0;
        int cut_count = 0;
        const int st = qs.advance(time - dt, time, 0, reactions, iterations, cut_count);
        if (info) {
            info[0] = (double)qs.newton_total;
            info[1] = (double)qs.pcg_iters;
            info[2] = (double)cut_count;
            info[3] = (double)inc;
        }
        if (st == ITERATIVE_NOT_CONVERGED) return NOT_CONVERGED;
        if (st != OK) return st;
        std::copy(qs.u.begin(), qs.u.end(), u_hist + (size_t)(inc - 1) * n);
        std::copy(reactions.begin(), reactions.end(), r_hist + (size_t)(inc - 1) * n);
        newton_iters[inc - 1] = (int32_t)iterations;
        cuts[inc - 1] = cut_count;
    }
    if (info) {
        info[0] = (double)qs.newton_total;
        info[1] = (double)qs.pcg_iters;
    }
    return OK;
}

// Adjoint of increment reactions: for J = sum_k dJdR[k] . R_k (R_k the reactions of increment k,
// weights read at fixed DOFs), dJ/dmu_e and dJ/dlambda_e (per element Lame parameters of the
// neo-Hookean law). Reverse pass over the checkpoints u_hist: at each increment with a nonzero
// weight g the tangent at u_k is recomputed, K_ff m_f = -K_fc g_c is solved with the same
// IC(0)-PCG, and w = (g_c, m_f) gives dJ_k/dp_e = w_e . dfe/dp_e. The reference has no
// gradients: this restates the adjoint on its equilibrium equations.
int oracle_large_strain_gradient(int64_t n_nodes, const double* coords, int64_t n_elems, const int64_t* conn,
                                 const double* young, const double* poisson, const uint8_t* fixed,
                                 int increments, const double* u_hist, const double* dJdR, double pcg_tol,
                                 int64_t pcg_max, double* dJdmu, double* dJdlambda) {
    LargeStrainMesh m{(size_t)n_nodes, (size_t)n_elems, coords, conn, {}, {}};
    m.lambda.resize(m.n_elems);
    m.mu.resize(m.n_elems);
    for (size_t e = 0; e < m.n_elems; ++e) lame(young[e], poisson[e], m.lambda[e], m.mu[e]);
    const size_t n = 3 * (size_t)n_nodes;
    FreeTopology t = free_topology(m.n_elems, conn, fixed, n);
    std::fill(dJdmu, dJdmu + n_elems, 0.0);
    if (dJdlambda) std::fill(dJdlambda, dJdlambda + n_elems, 0.0);
    size_t pcg_iters = 0;
    for (int k = increments - 1; k >= 0; --k) {
        const double* g = dJdR + (size_t)k * n;
        bool any = false;
        for (size_t q = 0; q < n; ++q) any = any || (fixed[q] && g[q] != 0.0);
        if (!any) continue;
        Vec uk(u_hist + (size_t)k * n, u_hist + (size_t)(k + 1) * n), internal, tangents;
        responses(m, uk, internal, tangents);
        Vec w(n, 0.0), zero(n, 0.0);
        for (size_t q = 0; q < n; ++q)
            if (fixed[q]) w[q] = g[q];
        const int st = free_solve(t, m, tangents, zero, w, pcg_tol > 0 ? pcg_tol : TOLERANCE,
                                  pcg_max > 0 ? (size_t)pcg_max : MAX_ITERATIONS, pcg_iters);
        if (st != OK) return st;
        for (size_t e = 0; e < m.n_elems; ++e) {
            double c[4][3], ue[12], fe[12], ke[144], dmu[12], dla[12];
            m.coords_of(e, c);
            for (int l = 0; l < 12; ++l) ue[l] = uk[3 * (size_t)conn[e * 4 + l / 3] + l % 3];
            neo_hookean_tet4(c, m.lambda[e], m.mu[e], ue, fe, ke, dmu, dla);
            double sm = 0.0, sl = 0.0;
            for (int l = 0; l < 12; ++l) {
                const double wl = w[3 * (size_t)conn[e * 4 + l / 3] + l % 3];
                sm += wl * dmu[l];
                sl += wl * dla[l];
            }
            dJdmu[e] += sm;
            if (dJdlambda) dJdlambda[e] += sl;
        }
    }
    return OK;
}

// One neo-Hookean Tet4 response (for element-level tests): fe [12], ke [144], dfe/dmu, dfe/dlambda.
int oracle_neo_hookean_tet4(const double* coords12, double lambda, double mu, const double* ue, double* fe,
                            double* ke, double* dfe_dmu, double* dfe_dlambda) {
    double c[4][3];
    for (int a = 0; a < 4; ++a)
        for (int k = 0; k < 3; ++k) c[a][k] = coords12[3 * a + k];
    return neo_hookean_tet4(c, lambda, mu, ue, fe, ke, dfe_dmu, dfe_dlambda) ? OK : INVALID;
}

// Model::solve_step (model.rs:621-706) of a Tet4/Tet10 thermal model on the CPU: the theta-method
// (C/dt + theta K) T_{n+1} = (C/dt - (1 - theta) K) T_n + F with K = conduction + convection,
// one factorisation (FreeSystem::new) reused by every increment, reactions
// R = (left T_{n+1} - right T_n - F) on imposed nodes and heat fluxes per increment.
//   per node: fixed, imposed, loads (nodal heat loads Load{dof: T}); per element: conductivity,
//   rho_c (density x specific heat); sources (element, value) (HeatSource, element_heat_source);
//   convection (element, face, film, sink) (Convection, face_convection).
//   initial: T at t = 0 (imposed values replace it at fixed nodes). solver: 0 Auto, 1 Direct,
//   2 Iterative. tol: PCG tolerance (0 selects 1e-12).
//   out: temps / reactions [(increments + 1) n_nodes], fluxes [(increments + 1) n_elems ngp 6]
//   (x, y, z, qx, qy, qz), f_out [n_nodes] the assembled F, iterations [increments],
//   info[0..7] = total PCG iterations, largest final relative residual, shift, free nodes,
//   nnz(L), ms setup, ms factor, ms increments.
// With rho_c = 0, theta = 1 and one increment the left matrix is K and the carried vector is
// zero: that run is the steady solve (Model::solve with Analysis::Thermal, model.rs:548-610).
int oracle_thermal_transient(int64_t n_nodes, const double* coords, int npe, int64_t n_elems,
                             const int64_t* conn, const double* conductivity, const double* rho_c,
                             const uint8_t* fixed, const double* imposed, const double* loads,
                             int64_t n_src, const int64_t* s_elem, const double* s_value,
                             int64_t n_conv, const int64_t* c_elem, const int32_t* c_face,
                             const double* c_film, const double* c_sink, const double* initial,
                             double dt, double theta, int64_t increments, int solver, double tol,
                             int64_t max_iter, double* temps, double* reactions, double* fluxes,
                             double* f_out, int64_t* iterations, double* info) {
    if (tol <= 0.0) tol = TOLERANCE;
    if (max_iter <= 0) max_iter = (int64_t)MAX_ITERATIONS;
    if (npe != 4 && npe != 10) return INVALID;
    const double t0 = now_ms();
    const size_t n = (size_t)n_nodes, ne = (size_t)n_elems;
    auto node = [&](size_t e, int a) { return (size_t)conn[e * npe + a]; };
    auto elem_coords = [&](size_t e, double (*c)[3]) {
        for (int a = 0; a < npe; ++a)
            for (int k = 0; k < 3; ++k) c[a][k] = coords[3 * node(e, a) + k];
    };
    const TetGP* rule;
    const int ng = rule_of(npe, &rule);
    const TetGP* crule = npe == 4 ? TETRA_4 : TETRA_14.p;
    const int cng = npe == 4 ? 4 : 14;

    // assemble, model.rs:1070-1147 (thermal: one DOF per node)
    std::vector<std::vector<Convection>> faces(ne);
    for (int64_t k = 0; k < n_conv; ++k) {
        const int64_t e = c_elem[k];
        if (e < 0 || e >= n_elems) continue;
        double c[10][3];
        elem_coords((size_t)e, c);
        Convection cv;
        if (face_convection(npe, c, c_face[k], c_film[k], c_sink[k], cv)) faces[(size_t)e].push_back(cv);
    }
    Vec f(n, 0.0);
    for (size_t g = 0; g < n; ++g) f[g] += loads ? loads[g] : 0.0;
    GaussData gd[14];
    for (int64_t k = 0; k < n_src; ++k) {
        const size_t e = (size_t)s_elem[k];
        double c[10][3];
        elem_coords(e, c);
        solid_gauss(npe, c, rule, ng, gd);
        double fs[10] = {0};
        for (int gp = 0; gp < ng; ++gp)
            for (int a = 0; a < npe; ++a) fs[a] += gd[gp].w * gd[gp].n[a] * s_value[k];
        for (int a = 0; a < npe; ++a) f[node(e, a)] += fs[a];
    }
    for (size_t e = 0; e < ne; ++e)
        for (const Convection& cv : faces[e])
            for (int a = 0; a < cv.nn; ++a) f[node(e, cv.pos[a])] += cv.load[a];

    // left / right element matrices, model.rs:646-663
    const int m = npe;
    Vec left(ne * m * m), right(ne * m * m), kk(m * m), cc(m * m);
    for (size_t e = 0; e < ne; ++e) {
        double c[10][3];
        elem_coords(e, c);
        solid_gauss(npe, c, rule, ng, gd);
        conduction(npe, gd, ng, conductivity[e], kk.data());
        for (const Convection& cv : faces[e])
            for (int a = 0; a < cv.nn; ++a)
                for (int b = 0; b < cv.nn; ++b) kk[cv.pos[a] * m + cv.pos[b]] += cv.matrix[a * cv.nn + b];
        solid_gauss(npe, c, crule, cng, gd);
        capacity(npe, gd, cng, rho_c[e], cc.data());
        for (int q = 0; q < m * m; ++q) {
            left[e * m * m + q] = cc[q] / dt + theta * kk[q];
            right[e * m * m + q] = cc[q] / dt + (theta - 1.0) * kk[q];
        }
    }
    Vec t(initial, initial + n);
    for (size_t g = 0; g < n; ++g)
        if (fixed[g]) t[g] = imposed[g];

    // FreeSystem::new, model.rs:1442-1499, on the left matrix
    IVec free(n, NONE);
    size_t count = 0;
    for (size_t g = 0; g < n; ++g)
        if (!fixed[g]) free[g] = count++;
    IVec eoff(ne + 1, 0), eidx;
    for (size_t e = 0; e < ne; ++e) {
        for (int a = 0; a < m; ++a)
            if (free[node(e, a)] != NONE) eidx.push_back(free[node(e, a)]);
        eoff[e + 1] = eidx.size();
    }
    Graph graph = graph_from_elements(count, eoff, eidx);
    IVec order = reverse_cuthill_mckee(graph);
    IVec rank(count);
    for (size_t r = 0; r < count; ++r) rank[order[r]] = r;
    const bool iterative = solver == 2 || (solver == 0 && count >= ITERATIVE_FROM);
    Csr csr;
    std::optional<Skyline> sky;
    if (iterative) {
        csr = Csr::zeros(graph, order, rank);
    } else {
        IVec first(count);
        for (size_t a = 0; a < count; ++a) first[a] = a;
        for (size_t a = 0; a < count; ++a)
            for (size_t p = graph.offsets[a]; p < graph.offsets[a + 1]; ++p)
                first[rank[a]] = std::min(first[rank[a]], rank[graph.targets[p]]);
        sky.emplace(first);
    }
    graph = Graph{};
    Vec coupling(count, 0.0);
    for (size_t e = 0; e < ne; ++e)
        for (int r = 0; r < m; ++r) {
            const size_t a = free[node(e, r)];
            if (a == NONE) continue;
            for (int c = 0; c < m; ++c) {
                const size_t b = free[node(e, c)];
                const double k = left[e * m * m + r * m + c];
                if (b != NONE) {
                    if (rank[b] <= rank[a]) {
                        if (iterative) csr.add(rank[a], rank[b], k);
                        else sky->add(rank[a], rank[b], k);
                    }
                } else {
                    coupling[rank[a]] += k * t[node(e, c)];
                }
            }
        }
    const double t1 = now_ms();
    Vec l;
    SolveStats st;
    if (iterative) {
        bool ok = false;
        for (double shift : SHIFTS) {
            auto got = csr.incomplete_cholesky(shift);
            if (got) {
                l = std::move(*got);
                st.shift = shift;
                ok = true;
                break;
            }
        }
        if (!ok) return SINGULAR;
    } else if (sky->factorize() != OK) {
        return SINGULAR;
    }
    const double t2 = now_ms();

    // product, model.rs:1353-1369: (sum_e M_e x_e) on the rows `rows` (nullptr = every row)
    auto product = [&](const Vec& mats, const Vec& x, const uint8_t* rows, Vec& y) {
        std::fill(y.begin(), y.end(), 0.0);
        for (size_t e = 0; e < ne; ++e) {
            bool any = rows == nullptr;
            for (int a = 0; a < m && !any; ++a) any = rows[node(e, a)] != 0;
            if (!any) continue;
            for (int r = 0; r < m; ++r) {
                const size_t g = node(e, r);
                if (rows && !rows[g]) continue;
                const double* row = &mats[e * m * m + r * m];
                double s = row[0] * x[node(e, 0)];
                for (int c = 1; c < m; ++c) s = s + row[c] * x[node(e, c)];
                y[g] += s;
            }
        }
    };
    auto write_fluxes = [&](const Vec& temp, double* out) {
        if (!out) return;
        for (size_t e = 0; e < ne; ++e) {
            double c[10][3], te[10];
            elem_coords(e, c);
            solid_gauss(npe, c, rule, ng, gd);
            for (int a = 0; a < m; ++a) te[a] = temp[node(e, a)];
            heat_fluxes(npe, gd, ng, conductivity[e], te, out + e * ng * 6);
        }
    };
    if (temps) std::copy(t.begin(), t.end(), temps);
    if (reactions) std::fill(reactions, reactions + n, 0.0);
    write_fluxes(t, fluxes);
    int64_t total = 0;
    double worst = 0.0;
    Vec carried(n), rhs(n), y(n), b(count), x;
    for (int64_t s = 1; s <= increments; ++s) {
        product(right, t, nullptr, carried);
        for (size_t g = 0; g < n; ++g) rhs[g] = carried[g] + f[g];
        // FreeSystem::solve, model.rs:1502-1516
        for (size_t k = 0; k < count; ++k) b[k] = -coupling[k];
        for (size_t g = 0; g < n; ++g)
            if (free[g] != NONE) b[rank[free[g]]] += rhs[g];
        if (iterative) {
            SolveStats ss;
            const int status = pcg_solve(csr, b, tol, (size_t)max_iter, x, ss, &l);
            total += (int64_t)ss.iterations;
            worst = std::max(worst, ss.rel_residual);
            if (iterations) iterations[s - 1] = (int64_t)ss.iterations;
            if (status != OK) {
                if (info) info[0] = (double)total;
                return status;
            }
        } else {
            x = sky->solve(b);
            if (iterations) iterations[s - 1] = 0;
        }
        for (size_t g = 0; g < n; ++g)
            if (free[g] != NONE) t[g] = x[rank[free[g]]];
        if (temps) std::copy(t.begin(), t.end(), temps + (size_t)s * n);
        if (reactions) {
            product(left, t, fixed, y);
            for (size_t g = 0; g < n; ++g)
                if (fixed[g]) y[g] -= rhs[g];
            std::copy(y.begin(), y.end(), reactions + (size_t)s * n);
        }
        if (fluxes) write_fluxes(t, fluxes + (size_t)s * ne * ng * 6);
    }
    const double t3 = now_ms();
    if (f_out) std::copy(f.begin(), f.end(), f_out);
    if (info) {
        info[0] = (double)total;
        info[1] = worst;
        info[2] = st.shift;
        info[3] = (double)count;
        info[4] = iterative ? (double)csr.cols.size() : (double)sky->data.size();
        info[5] = t1 - t0;
        info[6] = t2 - t1;
        info[7] = t3 - t2;
    }
    return OK;
}

// TETRA_14 points (xi, eta, zeta, w) x 14, for the quadrature known-answer test
void oracle_tetra14(double* out) {
    for (int k = 0; k < 14; ++k) {
        out[4 * k] = TETRA_14.p[k].xi;
        out[4 * k + 1] = TETRA_14.p[k].eta;
        out[4 * k + 2] = TETRA_14.p[k].zeta;
        out[4 * k + 3] = TETRA_14.p[k].w;
    }
}

// Element conduction K_e and capacity C_e (npe x npe each) of one element (coords npe x 3)
void oracle_thermal_element(int npe, const double* coords, double k, double rho_c, double* ke, double* ce) {
    const double (*c)[3] = reinterpret_cast<const double (*)[3]>(coords);
    GaussData gd[14];
    const TetGP* rule;
    const int ng = rule_of(npe, &rule);
    solid_gauss(npe, c, rule, ng, gd);
    conduction(npe, gd, ng, k, ke);
    solid_gauss(npe, c, npe == 4 ? TETRA_4 : TETRA_14.p, npe == 4 ? 4 : 14, gd);
    capacity(npe, gd, npe == 4 ? 4 : 14, rho_c, ce);
}

}  // extern "C"
