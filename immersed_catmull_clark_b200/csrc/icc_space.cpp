// Host-side set-up of the p = 2 tensor-product B-spline space and its exact elasticity element
// matrices.  This is the library's own implementation of the reference's discretisation layer
// (rust/src/iga/quadrature.rs, basis.rs, space.rs, elasticity.rs), restricted to the hot path:
// 3-D boxes, degree 2, maximal regularity, 3 Gauss points per direction.  The arithmetic keeps
// the reference's association order so the element matrices are bit-identical to its own.
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include "icc_internal.h"

namespace icc {

namespace {

// Gauss-Legendre nodes/weights by Newton iteration from the Tricomi guess
// (rust/src/iga/quadrature.rs:5-47).
void gauss_rule(int n, double *x, double *w) {
    auto legendre = [n](double z, double &p, double &dp) {
        double a = 1.0, b = z;
        for (int k = 2; k <= n; ++k) {
            double kf = double(k);
            double c = ((2.0 * kf - 1.0) * z * b - (kf - 1.0) * a) / kf;
            a = b;
            b = c;
        }
        dp = double(n) * (z * b - a) / (z * z - 1.0);
        p = b;
    };
    for (int i = 0; i < n; ++i) {
        double z = std::cos(M_PI * (double(i) + 0.75) / (double(n) + 0.5));
        double dp = 0.0, p, d;
        for (int it = 0; it < 100; ++it) {
            legendre(z, p, d);
            dp = d;
            double dz = p / d;
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        legendre(z, p, d);
        if (d != 0.0) dp = d;
        x[i] = -z;
        w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
}

// Values and derivatives of the 3 quadratic B-splines that are nonzero at x
// (Cox-de Boor, rust/src/iga/basis.rs:20-72, specialised to p = 2).  Returns the first index.
int quadratic_basis(const std::vector<double> &kn, double x, double v[3], double dv[3]) {
    const int p = 2;
    const int nk = int(kn.size());
    const int ndof = nk - p - 1;
    int cnt = 0;
    while (cnt < nk && kn[cnt] <= x) ++cnt;
    int s = cnt > 0 ? cnt - 1 : 0;
    s = s < p ? p : (s > ndof - 1 ? ndof - 1 : s);
    double b[3] = {1.0, 0.0, 0.0}, prev[3] = {0, 0, 0};
    for (int k = 1; k <= p; ++k) {
        if (k == p) std::memcpy(prev, b, sizeof(prev));
        double nb[3] = {0, 0, 0};
        for (int r = 0; r <= k; ++r) {
            int i = s + r - k;
            double val = 0.0;
            if (r > 0) {
                double d = kn[i + k] - kn[i];
                if (d > 0.0) val += (x - kn[i]) / d * b[r - 1];
            }
            if (r < k) {
                double d = kn[i + k + 1] - kn[i + 1];
                if (d > 0.0) val += (kn[i + k + 1] - x) / d * b[r];
            }
            nb[r] = val;
        }
        std::memcpy(b, nb, sizeof(b));
    }
    for (int r = 0; r <= p; ++r) {
        int i = s + r - p;
        double val = 0.0;
        if (r > 0) {
            double d = kn[i + p] - kn[i];
            if (d > 0.0) val += prev[r - 1] / d;
        }
        if (r < p) {
            double d = kn[i + p + 1] - kn[i + 1];
            if (d > 0.0) val -= prev[r] / d;
        }
        v[r] = b[r];
        dv[r] = double(p) * val;
    }
    return s - p;
}

// One direction: the 1-D element matrices M00, M10, M01, M11 of every element and their grouping
// into 1-D types (rust/src/iga/elasticity.rs:37-85).
struct Dir1d {
    std::vector<Mat1d> distinct;   // distinct 1-D matrix quadruples, first-appearance order
    std::vector<int> type_of;      // 1-D type of every element
    std::vector<int> first_cp;     // first control point of every element
    std::vector<std::array<double, 9>> basis;  // basis values of each distinct type (Space::basis1d)
};

Dir1d build_direction(int nel, double length) {
    std::vector<double> kn;
    for (int i = 0; i < 3; ++i) kn.push_back(0.0);
    for (int i = 1; i < nel; ++i) kn.push_back(double(i) / double(nel));  // multiplicity p - (p-1) = 1
    for (int i = 0; i < 3; ++i) kn.push_back(1.0);
    // breaks = unique knots; for this knot vector they are i/nel
    std::vector<double> br;
    for (double k : kn)
        if (br.empty() || k != br.back()) br.push_back(k);
    double xg[3], wg[3];
    gauss_rule(3, xg, wg);
    Dir1d out;
    std::vector<Mat1d> per((size_t)nel);
    double scale = 0.0;
    for (int e = 0; e < nel; ++e) {
        double a = br[e], b = br[e + 1];
        double v[3], dv[3];
        out.first_cp.push_back(quadratic_basis(kn, 0.5 * (a + b), v, dv));
        double h = b - a;
        Mat1d m;
        std::memset(&m, 0, sizeof(m));
        for (int q = 0; q < 3; ++q) {
            double x = a + 0.5 * (xg[q] + 1.0) * h;
            double qw = 0.5 * wg[q] * h;
            quadratic_basis(kn, x, v, dv);
            double w = qw * length;
            for (int i = 0; i < 3; ++i) {
                double ni = v[i], di = dv[i] / length;
                for (int j = 0; j < 3; ++j) {
                    double nj = v[j], dj = dv[j] / length;
                    m.k[0][i][j] += w * ni * nj;
                    m.k[1][i][j] += w * di * nj;
                    m.k[2][i][j] += w * ni * dj;
                    m.k[3][i][j] += w * di * dj;
                }
            }
        }
        for (int k = 0; k < 4; ++k)
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) scale = std::fmax(scale, std::fabs(m.k[k][i][j]));
        per[size_t(e)] = m;
    }
    std::map<std::vector<long long>, int> seen;
    for (int e = 0; e < nel; ++e) {
        std::vector<long long> key;
        key.reserve(36);
        for (int k = 0; k < 4; ++k)
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) key.push_back((long long)std::round(per[e].k[k][i][j] / scale * 1e12));
        auto it = seen.find(key);
        int t;
        if (it == seen.end()) {
            t = int(out.distinct.size());
            seen.emplace(key, t);
            out.distinct.push_back(per[e]);
            std::array<double, 9> bv;
            const double a = br[e], h = br[e + 1] - br[e];
            for (int q = 0; q < 3; ++q) {
                double v[3], dv[3];
                quadratic_basis(kn, a + 0.5 * (xg[q] + 1.0) * h, v, dv);
                for (int i = 0; i < 3; ++i) bv[3 * i + q] = v[i];
            }
            out.basis.push_back(bv);
        } else {
            t = it->second;
        }
        out.type_of.push_back(t);
    }
    return out;
}

}  // namespace

bool Space::init(const double bounds[6], const int64_t nsub[3]) {
    for (int d = 0; d < 3; ++d) {
        lo[d] = bounds[2 * d];
        len[d] = bounds[2 * d + 1] - bounds[2 * d];
        nel_dir[d] = nsub[d];
        ncp[d] = nsub[d] + 2;  // open knots, p = 2, maximal regularity
        if (nsub[d] < 1 || nsub[d] > (1 << 20) || !(len[d] > 0.0)) return false;
    }
    nel = nel_dir[0] * nel_dir[1] * nel_dir[2];
    nsc = ncp[0] * ncp[1] * ncp[2];
    ndof = 3 * nsc;
    for (int d = 0; d < 3; ++d) {
        Dir1d dd = build_direction(int(nel_dir[d]), len[d]);
        mats1d[d] = dd.distinct;
        type1d[d] = dd.type_of;
        basis1d[d] = dd.basis;
        for (int e = 0; e < int(nel_dir[d]); ++e)
            if (dd.first_cp[size_t(e)] != e) return false;  // uniform grid: element e starts at cp e
    }
    return true;
}

// Element types = distinct (tx, ty, tz) combinations in element order, and the 81x81 matrix of
// each: ke[(ci*27+a)*81 + cj*27+b] = lambda G_ij + mu G_ji (+ mu sum_k G_kk if ci == cj) with
// G_ij = Mz (x) My (x) Mx of the derivative pattern of (i, j) (rust/src/iga/elasticity.rs:87-150).
void Space::element_types(double lambda, double mu, std::vector<double> &ke, std::vector<int32_t> &type_id,
                          std::vector<std::array<int, 3>> &combos) const {
    std::map<std::array<int, 3>, int> seen;
    combos.clear();
    type_id.assign(size_t(nel), 0);
    for (int64_t ez = 0; ez < nel_dir[2]; ++ez)
        for (int64_t ey = 0; ey < nel_dir[1]; ++ey)
            for (int64_t ex = 0; ex < nel_dir[0]; ++ex) {
                std::array<int, 3> key = {type1d[0][ex], type1d[1][ey], type1d[2][ez]};
                auto it = seen.find(key);
                int t;
                if (it == seen.end()) {
                    t = int(combos.size());
                    seen.emplace(key, t);
                    combos.push_back(key);
                } else {
                    t = it->second;
                }
                type_id[size_t(ex + nel_dir[0] * (ey + nel_dir[1] * ez))] = t;
            }
    ke.assign(combos.size() * 81 * 81, 0.0);
    static double g[3][3][27][27];
    double lap[27][27];
    for (size_t t = 0; t < combos.size(); ++t) {
        const Mat1d *m[3] = {&mats1d[0][combos[t][0]], &mats1d[1][combos[t][1]], &mats1d[2][combos[t][2]]};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                int kind[3];
                for (int d = 0; d < 3; ++d) kind[d] = (d == i && d == j) ? 3 : (d == i) ? 1 : (d == j) ? 2 : 0;
                for (int a = 0; a < 27; ++a)
                    for (int b = 0; b < 27; ++b) {
                        int ax = a % 3, ay = (a / 3) % 3, az = a / 9;
                        int bx = b % 3, by = (b / 3) % 3, bz = b / 9;
                        double vx = m[0]->k[kind[0]][ax][bx] * 1.0;
                        double vy = m[1]->k[kind[1]][ay][by] * vx;
                        g[i][j][a][b] = m[2]->k[kind[2]][az][bz] * vy;
                    }
            }
        for (int a = 0; a < 27; ++a)
            for (int b = 0; b < 27; ++b) lap[a][b] = ((0.0 + g[0][0][a][b]) + g[1][1][a][b]) + g[2][2][a][b];
        double *k = ke.data() + t * 81 * 81;
        for (int ci = 0; ci < 3; ++ci)
            for (int cj = 0; cj < 3; ++cj)
                for (int a = 0; a < 27; ++a)
                    for (int b = 0; b < 27; ++b) {
                        double v = lambda * g[ci][cj][a][b] + mu * g[cj][ci][a][b];
                        if (ci == cj) v += mu * lap[a][b];
                        k[(ci * 27 + a) * 81 + cj * 27 + b] = v;
                    }
    }
}

}  // namespace icc

using icc::set_error;

extern "C" {

int icc_space_create(const double bounds[6], const int64_t nsub[3], int32_t degree, icc_space **out) {
    if (!bounds || !nsub || !out) return set_error(ICC_BAD_ARG, "icc_space_create: null argument");
    *out = nullptr;
    if (degree != 2) return set_error(ICC_BAD_ARG, "icc_space_create: only degree 2 is supported");
    auto *sp = new (std::nothrow) icc_space();
    if (!sp) return set_error(ICC_OUT_OF_MEMORY, "icc_space_create: out of host memory");
    if (!sp->s.init(bounds, nsub)) {
        delete sp;
        return set_error(ICC_BAD_ARG, "icc_space_create: invalid bounds or element counts");
    }
    *out = sp;
    return ICC_OK;
}

// A sub-grid of a space: its elements [e0[d], e1[d]) per direction with the parent's B-splines
// (the parent's knots, so the window's element matrices are the parent's, also next to a cut),
// numbered locally: control points [e0, e1 + 2) of the parent, x fastest.
int icc_space_window(const icc_space *sp, const int64_t e0[3], const int64_t e1[3], icc_space **out) {
    if (!sp || !e0 || !e1 || !out) return set_error(ICC_BAD_ARG, "icc_space_window: null argument");
    *out = nullptr;
    const icc::Space &p = sp->s;
    for (int d = 0; d < 3; ++d)
        if (e0[d] < 0 || e1[d] <= e0[d] || e1[d] > p.nel_dir[d])
            return set_error(ICC_BAD_ARG, "icc_space_window: element range outside the space");
    auto *w = new (std::nothrow) icc_space();
    if (!w) return set_error(ICC_OUT_OF_MEMORY, "icc_space_window: out of host memory");
    icc::Space &s = w->s;
    for (int d = 0; d < 3; ++d) {
        const double h = p.len[d] / double(p.nel_dir[d]);
        s.lo[d] = p.lo[d] + double(e0[d]) * h;
        s.len[d] = double(e1[d] - e0[d]) * h;
        s.nel_dir[d] = e1[d] - e0[d];
        s.ncp[d] = s.nel_dir[d] + 2;
        s.mats1d[d] = p.mats1d[d];
        s.basis1d[d] = p.basis1d[d];
        s.type1d[d].assign(p.type1d[d].begin() + e0[d], p.type1d[d].begin() + e1[d]);
    }
    s.nel = s.nel_dir[0] * s.nel_dir[1] * s.nel_dir[2];
    s.nsc = s.ncp[0] * s.ncp[1] * s.ncp[2];
    s.ndof = 3 * s.nsc;
    *out = w;
    return ICC_OK;
}

void icc_space_destroy(icc_space *sp) { delete sp; }

int icc_space_dims(const icc_space *sp, int64_t *ndof, int64_t *nel, int64_t ndof_dir[3], int64_t nel_dir[3]) {
    if (!sp) return set_error(ICC_BAD_ARG, "icc_space_dims: null space");
    if (ndof) *ndof = sp->s.ndof;
    if (nel) *nel = sp->s.nel;
    for (int d = 0; d < 3; ++d) {
        if (ndof_dir) ndof_dir[d] = sp->s.ncp[d];
        if (nel_dir) nel_dir[d] = sp->s.nel_dir[d];
    }
    return ICC_OK;
}

int icc_space_connectivity(const icc_space *sp, int64_t *conn) {
    if (!sp || !conn) return set_error(ICC_BAD_ARG, "icc_space_connectivity: null argument");
    const icc::Space &s = sp->s;
    for (int64_t ez = 0; ez < s.nel_dir[2]; ++ez)
        for (int64_t ey = 0; ey < s.nel_dir[1]; ++ey)
            for (int64_t ex = 0; ex < s.nel_dir[0]; ++ex) {
                int64_t e = ex + s.nel_dir[0] * (ey + s.nel_dir[1] * ez);
                for (int c = 0; c < 3; ++c)
                    for (int a = 0; a < 27; ++a) {
                        int64_t g = (ex + a % 3) + s.ncp[0] * ((ey + (a / 3) % 3) + s.ncp[1] * (ez + a / 9));
                        conn[e * 81 + c * 27 + a] = c * s.nsc + g;
                    }
            }
    return ICC_OK;
}

void icc_lame(double young, double poisson, double *lambda, double *mu) {
    if (lambda) *lambda = young * poisson / ((1.0 + poisson) * (1.0 - 2.0 * poisson));
    if (mu) *mu = young / (2.0 * (1.0 + poisson));
}

int icc_element_matrices(const icc_space *sp, double lambda, double mu, double *ke_types, int32_t max_types,
                         int32_t *type_id, int32_t *ntypes) {
    if (!sp || !ntypes) return set_error(ICC_BAD_ARG, "icc_element_matrices: null argument");
    std::vector<double> ke;
    std::vector<int32_t> tid;
    std::vector<std::array<int, 3>> combos;
    sp->s.element_types(lambda, mu, ke, tid, combos);
    *ntypes = int32_t(combos.size());
    if (ke_types) {
        if (int32_t(combos.size()) > max_types)
            return set_error(ICC_BAD_ARG, "icc_element_matrices: max_types too small");
        std::memcpy(ke_types, ke.data(), ke.size() * sizeof(double));
    }
    if (type_id) std::memcpy(type_id, tid.data(), tid.size() * sizeof(int32_t));
    return ICC_OK;
}

}  // extern "C"
