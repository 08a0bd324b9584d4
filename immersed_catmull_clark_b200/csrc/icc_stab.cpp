// Cut-cell stabilisation terms of the immersed solve, built on the host as triplets over the
// operator's DOF numbering.  They touch only the faces next to cut cells (O(surface) entries), so
// the device adds them to the volume operator as a sparse term (icc_op_set_extra_triplets) rather
// than as another matrix-free kernel.
//
//   * ghost penalty (rust/src/immersed.rs:224-370): for every interior face between two active
//     cells of which at least one is cut, gamma E h^(2p-1) int_F [d_n^p u] . [d_n^p v] per
//     component; on the box grid the face integral is the outer product of the jump of the p-th
//     normal derivative (4 functions across the face for p = 2) times the 1-D element mass
//     matrices of the two tangential directions;
//   * legacy springs (rust/src/immersed.rs:156-222), the MATLAB heuristic the reference keeps for
//     parity with its fixture.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "icc_internal.h"

namespace icc {
namespace {

constexpr int8_t kInside = 1, kCut = -1;   // cell status (rust/src/immersed.rs:22-24)

bool active(int8_t s) { return s == kInside || s == kCut; }

// Open uniform knots of degree 2 on [0, 1] with n elements (rust/src/iga/quadrature.rs:51-64).
std::vector<double> knots2(int n) {
    std::vector<double> t = {0.0, 0.0, 0.0};
    for (int i = 1; i < n; ++i) t.push_back(double(i) / double(n));
    t.insert(t.end(), {1.0, 1.0, 1.0});
    return t;
}

// Second parametric derivative of the three quadratics that live on knot span s (t_s <= x <
// t_{s+1}), functions s-2, s-1, s in that order.  It is constant on the span: differentiating
// N_{i,2} twice leaves the degree-0 indicator of span s weighted by the knot differences
// (terms with a zero difference vanish with their function).
void second_derivs(const std::vector<double> &t, int s, double d2[3]) {
    auto inv = [](double a) { return a > 0.0 ? 1.0 / a : 0.0; };
    const double h0 = t[s + 1] - t[s];                 // the span itself, > 0
    const double a = inv((t[s + 1] - t[s - 1]) * h0);  // N_{s-1,1}' / (t_{s+1} - t_{s-1}) part
    const double b = inv((t[s + 2] - t[s]) * h0);      // N_{s,1}' / (t_{s+2} - t_s) part
    d2[0] = 2.0 * a;
    d2[1] = -2.0 * (a + b);
    d2[2] = 2.0 * b;
}

struct Triplets {
    std::vector<int64_t> r, c;
    std::vector<double> v;
    void push(int64_t i, int64_t j, double x) {
        r.push_back(i);
        c.push_back(j);
        v.push_back(x);
    }
};

int export_triplets(const Triplets &t, int64_t *rows, int64_t *cols, double *vals, int64_t capacity, int64_t *count) {
    *count = int64_t(t.v.size());
    if (!rows && !cols && !vals) return ICC_OK;   // size query
    if (!rows || !cols || !vals) return set_error(ICC_BAD_ARG, "stabilization: rows, cols and vals must all be given");
    if (capacity < *count) return set_error(ICC_BAD_ARG, "stabilization: capacity smaller than the triplet count");
    std::memcpy(rows, t.r.data(), t.r.size() * sizeof(int64_t));
    std::memcpy(cols, t.c.data(), t.c.size() * sizeof(int64_t));
    std::memcpy(vals, t.v.data(), t.v.size() * sizeof(double));
    return ICC_OK;
}

void ghost_penalty(const Space &s, const int8_t *status, double gamma, double young, Triplets &out) {
    const int64_t n[3] = {s.nel_dir[0], s.nel_dir[1], s.nel_dir[2]};
    double h[3];
    for (int d = 0; d < 3; ++d) h[d] = s.len[d] / double(n[d]);
    const double hc = (h[0] + h[1] + h[2]) / 3.0;
    const double coef = gamma * young * std::pow(hc, 3.0);   // h^(2p - 1), p = 2
    // jumps of the second physical derivative across break k of each direction: functions
    // k-1 .. k+2 (the left element's k-1 .. k+1 and the right element's k .. k+2)
    std::vector<std::array<double, 4>> jump[3];
    for (int d = 0; d < 3; ++d) {
        const std::vector<double> t = knots2(int(n[d]));
        const double l2 = s.len[d] * s.len[d];
        jump[d].assign(size_t(n[d]), {0.0, 0.0, 0.0, 0.0});
        for (int64_t k = 1; k < n[d]; ++k) {
            double dl[3], dr[3];
            second_derivs(t, int(k - 1) + 2, dl);   // left element k-1: span k+1 of the knot vector
            second_derivs(t, int(k) + 2, dr);       // right element k
            std::array<double, 4> j;
            for (int q = 0; q < 4; ++q) {
                const double r = q >= 1 ? dr[q - 1] : 0.0;
                const double l = q <= 2 ? dl[q] : 0.0;
                j[size_t(q)] = (r - l) / l2;
            }
            jump[d][size_t(k)] = j;
        }
    }
    for (int d = 0; d < 3; ++d) {
        const int ta = d == 0 ? 1 : 0, tb = d == 2 ? 1 : 2;   // tangential directions, increasing
        const int64_t stride = d == 0 ? 1 : (d == 1 ? n[0] : n[0] * n[1]);
        for (int64_t e2 = 0; e2 < s.nel; ++e2) {
            const int64_t ix[3] = {e2 % n[0], (e2 / n[0]) % n[1], e2 / (n[0] * n[1])};
            if (ix[d] == 0) continue;
            const int64_t e1 = e2 - stride;
            if (!(active(status[e1]) && active(status[e2]) && (status[e1] == kCut || status[e2] == kCut))) continue;
            const std::array<double, 4> &jv = jump[d][size_t(ix[d])];
            const Mat1d &ma = s.mats1d[ta][size_t(s.type1d[ta][size_t(ix[ta])])];
            const Mat1d &mb = s.mats1d[tb][size_t(s.type1d[tb][size_t(ix[tb])])];
            // local functions: 4 along the normal (first k-1), 3 along each tangential direction
            // (first = the element index); local index a = (a0 + sz0 (a1 + sz1 a2)) over the
            // directions in increasing order, the normal one of size 4
            int sz[3] = {3, 3, 3};
            sz[d] = 4;
            int64_t first[3] = {ix[0], ix[1], ix[2]};
            first[d] = ix[d] - 1;
            const int nloc = sz[0] * sz[1] * sz[2];
            int loc[36][3];
            int64_t gidx[36];
            for (int a = 0; a < nloc; ++a) {
                loc[a][0] = a % sz[0];
                loc[a][1] = (a / sz[0]) % sz[1];
                loc[a][2] = a / (sz[0] * sz[1]);
                gidx[a] = (first[0] + loc[a][0]) + s.ncp[0] * ((first[1] + loc[a][1]) + s.ncp[1] * (first[2] + loc[a][2]));
            }
            for (int a = 0; a < nloc; ++a)
                for (int b = 0; b < nloc; ++b) {
                    double v = coef * jv[size_t(loc[a][d])] * jv[size_t(loc[b][d])];
                    v *= ma.k[0][loc[a][ta]][loc[b][ta]];
                    v *= mb.k[0][loc[a][tb]][loc[b][tb]];
                    if (v == 0.0) continue;
                    for (int c = 0; c < 3; ++c) out.push(c * s.nsc + gidx[a], c * s.nsc + gidx[b], v);
                }
        }
    }
}

void legacy_springs(const Space &s, const int8_t *status, double gamma, Triplets &out) {
    const int64_t n[3] = {s.nel_dir[0], s.nel_dir[1], s.nel_dir[2]};
    const double alpha = gamma * (((s.len[0] / double(n[0]) + s.len[1] / double(n[1])) + s.len[2] / double(n[2])) / 3.0);
    // faces in the order of the reference: direction x, y, z; within one, i slowest, k fastest
    std::vector<std::pair<int64_t, int64_t>> faces;
    const int64_t dir[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    auto lin = [&](int64_t i, int64_t j, int64_t k) { return i + n[0] * (j + n[1] * k); };
    for (const auto &dd : dir)
        for (int64_t i = 0; i < n[0] - dd[0]; ++i)
            for (int64_t j = 0; j < n[1] - dd[1]; ++j)
                for (int64_t k = 0; k < n[2] - dd[2]; ++k) {
                    const int64_t e1 = lin(i, j, k), e2 = lin(i + dd[0], j + dd[1], k + dd[2]);
                    if (active(status[e1]) && active(status[e2]) && (status[e1] == kCut || status[e2] == kCut))
                        faces.emplace_back(e1, e2);
                }
    // a cell's scalar control points (distinct and sorted: the 27 of its 3 x 3 x 3 block)
    auto cps = [&](int64_t e) {
        const int64_t ex = e % n[0], ey = (e / n[0]) % n[1], ez = e / (n[0] * n[1]);
        std::vector<int64_t> v;
        for (int az = 0; az < 3; ++az)
            for (int ay = 0; ay < 3; ++ay)
                for (int ax = 0; ax < 3; ++ax) v.push_back((ex + ax) + s.ncp[0] * ((ey + ay) + s.ncp[1] * (ez + az)));
        std::sort(v.begin(), v.end());
        return v;
    };
    for (const auto &f : faces) {
        const std::vector<int64_t> g1 = cps(f.first), g2 = cps(f.second);
        std::vector<int64_t> common, only1, only2;
        std::set_intersection(g1.begin(), g1.end(), g2.begin(), g2.end(), std::back_inserter(common));
        std::set_difference(g1.begin(), g1.end(), g2.begin(), g2.end(), std::back_inserter(only1));
        std::set_difference(g2.begin(), g2.end(), g1.begin(), g1.end(), std::back_inserter(only2));
        for (int c = 0; c < 3; ++c) {
            const int64_t off = c * s.nsc;
            const size_t m = common.size();
            if (m > 0) {
                // the block on the shared points: a diagonal entry alpha/m (delta - 1/m) for every
                // (i, j) pair of the shared set, written on row = column = shared point i
                const double mf = double(m);
                for (size_t q = 0; q < m * m; ++q) {
                    const size_t i = q % m, j = q / m;
                    out.push(off + common[i], off + common[i], (alpha / mf) * ((i == j ? 1.0 : 0.0) - 1.0 / mf));
                }
            }
            // springs between the non-shared points, paired in sorted order
            const size_t np = std::min(only1.size(), only2.size());
            for (size_t k = 0; k < np; ++k) {
                const int64_t p1 = off + only1[k], p2 = off + only2[k];
                out.push(p1, p1, alpha);
                out.push(p2, p2, alpha);
                out.push(p1, p2, -alpha);
                out.push(p2, p1, -alpha);
            }
        }
    }
}

}  // namespace
}  // namespace icc

using icc::set_error;

extern "C" {

int icc_ghost_penalty(const icc_space *sp, const int8_t *status, double gamma, double young, int64_t *rows,
                      int64_t *cols, double *vals, int64_t capacity, int64_t *count) {
    if (!sp || !status || !count) return set_error(ICC_BAD_ARG, "icc_ghost_penalty: null argument");
    icc::Triplets t;
    icc::ghost_penalty(sp->s, status, gamma, young, t);
    return icc::export_triplets(t, rows, cols, vals, capacity, count);
}

int icc_legacy_stabilization(const icc_space *sp, const int8_t *status, double gamma, int64_t *rows, int64_t *cols,
                             double *vals, int64_t capacity, int64_t *count) {
    if (!sp || !status || !count) return set_error(ICC_BAD_ARG, "icc_legacy_stabilization: null argument");
    icc::Triplets t;
    icc::legacy_springs(sp->s, status, gamma, t);
    return icc::export_triplets(t, rows, cols, vals, capacity, count);
}

}  // extern "C"
