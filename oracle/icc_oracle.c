/*
 * TEST INFRASTRUCTURE ONLY -- the CPU oracle for the B-spline elasticity hot path.
 *
 * A plain-C restatement of the reference (dshguilherme/immersed_catmull_clark, Rust port in
 * `rust/`) used to check the CUDA product path.  Only `tests/`, `__graft_entry__.smoke()` and
 * the CPU-baseline leg of `bench.py` load it.  The product library (libicc) never links it.
 *
 * Every function names the reference lines it restates.  Arithmetic follows the reference
 * operation for operation (left-to-right sums, no FMA contraction: build with
 * -ffp-contract=off), so small cases agree with the reference to rounding.
 *
 * Pinned by the reference's MATLAB-exported fixtures (rust/tests/fixtures/iga_kernel.json,
 * immersed_tilted_box.json, topopt3d_8x4x2.json), copied into tests/golden/.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef int64_t i64;

#define ORC_MAXD 3

/* ------------------------------------------------------------------------------------------ */
/* quadrature.rs                                                                              */
/* ------------------------------------------------------------------------------------------ */

/* rust/src/iga/quadrature.rs:33-47 legendre_with_derivative */
static void legendre_with_derivative(int n, double z, double *p_out, double *dp_out) {
    double p0 = 1.0, p1 = z;
    if (n == 0) { *p_out = 1.0; *dp_out = 0.0; return; }
    for (int k = 2; k <= n; k++) {
        double kf = (double)k;
        double p2 = ((2.0 * kf - 1.0) * z * p1 - (kf - 1.0) * p0) / kf;
        p0 = p1;
        p1 = p2;
    }
    *dp_out = (double)n * (z * p1 - p0) / (z * z - 1.0);
    *p_out = p1;
}

/* rust/src/iga/quadrature.rs:5-31 gauss_legendre */
void orc_gauss_legendre(int n, double *x, double *w) {
    const double PI = 3.14159265358979323846;
    for (int i = 0; i < n; i++) {
        double z = cos(PI * ((double)i + 0.75) / ((double)n + 0.5));
        double dp = 0.0;
        for (int it = 0; it < 100; it++) {
            double p, d;
            legendre_with_derivative(n, z, &p, &d);
            dp = d;
            double dz = p / d;
            z -= dz;
            if (fabs(dz) < 1e-16) break;
        }
        double p, d;
        legendre_with_derivative(n, z, &p, &d);
        if (d != 0.0) dp = d;
        x[i] = -z;
        w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
}

/* rust/src/iga/quadrature.rs:51-64 open_knots; returns the knot count (buffer >= 2p+2+(nel-1)*mult) */
int orc_open_knots(int nel, int degree, int regularity, double *knots) {
    int mult = degree - regularity;
    int k = 0;
    for (int i = 0; i <= degree; i++) knots[k++] = 0.0;
    for (int i = 1; i < nel; i++) {
        double b = (double)i / (double)nel;
        for (int m = 0; m < mult; m++) knots[k++] = b;
    }
    for (int i = 0; i <= degree; i++) knots[k++] = 1.0;
    return k;
}

/* ------------------------------------------------------------------------------------------ */
/* basis.rs                                                                                   */
/* ------------------------------------------------------------------------------------------ */

/* rust/src/iga/basis.rs:11-15 find_span */
static int find_span(const double *knots, int nk, int p, double x) {
    int ndof = nk - p - 1;
    int count = 0; /* partition_point(|k| k <= x) on a sorted vector */
    while (count < nk && knots[count] <= x) count++;
    int s = count > 0 ? count - 1 : 0;
    if (s < p) s = p;
    if (s > ndof - 1) s = ndof - 1;
    return s;
}

/* rust/src/iga/basis.rs:20-72 basis_funs: values and first derivatives of the p+1 nonzero
 * functions at x; returns the index of the first one. */
int orc_basis_funs(const double *knots, int nk, int p, double x, double *vals, double *ders) {
    int s = find_span(knots, nk, p, x);
    double b[16], bn[16], b_prev[16];
    int blen = 1;
    b[0] = 1.0;
    for (int k = 1; k <= p; k++) {
        if (k == p) for (int r = 0; r < blen; r++) b_prev[r] = b[r];
        for (int r = 0; r <= k; r++) {
            int i = s + r - k;
            double val = 0.0;
            if (r > 0) {
                double d = knots[i + k] - knots[i];
                if (d > 0.0) val += (x - knots[i]) / d * b[r - 1];
            }
            if (r < k) {
                double d = knots[i + k + 1] - knots[i + 1];
                if (d > 0.0) val += (knots[i + k + 1] - x) / d * b[r];
            }
            bn[r] = val;
        }
        for (int r = 0; r <= k; r++) b[r] = bn[r];
        blen = k + 1;
    }
    for (int r = 0; r <= p; r++) { vals[r] = b[r]; ders[r] = 0.0; }
    if (p > 0) {
        for (int r = 0; r <= p; r++) {
            int i = s + r - p;
            double val = 0.0;
            if (r > 0) {
                double d = knots[i + p] - knots[i];
                if (d > 0.0) val += b_prev[r - 1] / d;
            }
            if (r < p) {
                double d = knots[i + p + 1] - knots[i + 1];
                if (d > 0.0) val -= b_prev[r] / d;
            }
            ders[r] = (double)p * val;
        }
    }
    return s - p;
}

/* ------------------------------------------------------------------------------------------ */
/* space.rs                                                                                   */
/* ------------------------------------------------------------------------------------------ */

typedef struct {
    double *knots; int nk;
    int degree, ndof, nel, nquad;
    double *breaks;
    int *connectivity;          /* [nel*(p+1)] */
    double *qn, *qw;            /* [nel*nquad] */
    double *shape, *dshape;     /* [(e*nquad+q)*(p+1)+a] */
} orc_space1d;

typedef struct {
    int dim;
    double lo[ORC_MAXD], lengths[ORC_MAXD];
    int nel_dir[ORC_MAXD];
    i64 nel;
    int degree[ORC_MAXD], nquad[ORC_MAXD], nqn;
    orc_space1d univ[ORC_MAXD];
    int ndof_dir[ORC_MAXD];
    i64 ndof_sc, ndof;
    int nsh_dir[ORC_MAXD], nsh_sc, nsh;
    i64 *conn_sc;               /* [nel*nsh_sc] */
    i64 *connectivity;          /* [nel*nsh] */
} orc_space;

/* rust/src/iga/space.rs:36-72 Space1d::new */
static void space1d_init(orc_space1d *u, int nel_in, int degree, int regularity, int nquad) {
    int p = degree;
    int mult = degree - regularity;
    u->knots = (double *)malloc(sizeof(double) * (size_t)(2 * (p + 1) + (nel_in - 1) * mult));
    u->nk = orc_open_knots(nel_in, degree, regularity, u->knots);
    u->degree = p;
    u->breaks = (double *)malloc(sizeof(double) * (size_t)u->nk);
    int nb = 0;
    for (int i = 0; i < u->nk; i++)
        if (nb == 0 || u->knots[i] != u->breaks[nb - 1]) u->breaks[nb++] = u->knots[i];
    u->nel = nb - 1;
    u->ndof = u->nk - p - 1;
    u->nquad = nquad;
    int nl = p + 1;
    u->connectivity = (int *)malloc(sizeof(int) * (size_t)(u->nel * nl));
    u->qn = (double *)malloc(sizeof(double) * (size_t)(u->nel * nquad));
    u->qw = (double *)malloc(sizeof(double) * (size_t)(u->nel * nquad));
    u->shape = (double *)malloc(sizeof(double) * (size_t)(u->nel * nquad * nl));
    u->dshape = (double *)malloc(sizeof(double) * (size_t)(u->nel * nquad * nl));
    double xg[32], wg[32], v[16], d[16];
    orc_gauss_legendre(nquad, xg, wg);
    for (int e = 0; e < u->nel; e++) {
        double a = u->breaks[e], b = u->breaks[e + 1];
        int first = orc_basis_funs(u->knots, u->nk, p, 0.5 * (a + b), v, d);
        for (int r = 0; r <= p; r++) u->connectivity[e * nl + r] = first + r;
        double h = b - a;
        for (int q = 0; q < nquad; q++) {
            double x = a + 0.5 * (xg[q] + 1.0) * h;
            u->qn[e * nquad + q] = x;
            u->qw[e * nquad + q] = 0.5 * wg[q] * h;
            orc_basis_funs(u->knots, u->nk, p, x, v, d);
            for (int r = 0; r < nl; r++) {
                u->shape[(e * nquad + q) * nl + r] = v[r];
                u->dshape[(e * nquad + q) * nl + r] = d[r];
            }
        }
    }
}

static void space1d_free(orc_space1d *u) {
    free(u->knots); free(u->breaks); free(u->connectivity);
    free(u->qn); free(u->qw); free(u->shape); free(u->dshape);
}

/* lexicographic multi-index, direction 0 fastest (rust/src/iga/space.rs:204-211 unravel) */
static void unravel(i64 idx, const int *dims, int dim, int *out) {
    for (int d = 0; d < dim; d++) { out[d] = (int)(idx % dims[d]); idx /= dims[d]; }
}

/* rust/src/iga/space.rs:107-160 SpaceBox::new / with_params (max regularity, p+1 Gauss points) */
orc_space *orc_space_new(int dim, const double *bounds, const int *nsub, int degree) {
    orc_space *sp = (orc_space *)calloc(1, sizeof(orc_space));
    sp->dim = dim;
    sp->nel = 1; sp->ndof_sc = 1; sp->nsh_sc = 1; sp->nqn = 1;
    for (int d = 0; d < dim; d++) {
        sp->lo[d] = bounds[2 * d];
        sp->lengths[d] = bounds[2 * d + 1] - bounds[2 * d];
        sp->degree[d] = degree;
        sp->nquad[d] = degree + 1;
        space1d_init(&sp->univ[d], nsub[d], degree, degree - 1, degree + 1);
        sp->nel_dir[d] = sp->univ[d].nel;
        sp->nel *= sp->nel_dir[d];
        sp->ndof_dir[d] = sp->univ[d].ndof;
        sp->ndof_sc *= sp->ndof_dir[d];
        sp->nsh_dir[d] = degree + 1;
        sp->nsh_sc *= degree + 1;
        sp->nqn *= degree + 1;
    }
    sp->nsh = dim * sp->nsh_sc;
    sp->ndof = dim * sp->ndof_sc;
    sp->conn_sc = (i64 *)malloc(sizeof(i64) * (size_t)(sp->nel * sp->nsh_sc));
    sp->connectivity = (i64 *)malloc(sizeof(i64) * (size_t)(sp->nel * sp->nsh));
    int esub[ORC_MAXD], asub[ORC_MAXD];
    for (i64 e = 0; e < sp->nel; e++) {
        unravel(e, sp->nel_dir, dim, esub);
        for (int a = 0; a < sp->nsh_sc; a++) {
            unravel(a, sp->nsh_dir, dim, asub);
            i64 g = 0, stride = 1;
            for (int d = 0; d < dim; d++) {
                const orc_space1d *u = &sp->univ[d];
                g += (i64)u->connectivity[esub[d] * (u->degree + 1) + asub[d]] * stride;
                stride *= sp->ndof_dir[d];
            }
            sp->conn_sc[e * sp->nsh_sc + a] = g;
        }
    }
    for (i64 e = 0; e < sp->nel; e++)
        for (int c = 0; c < dim; c++)
            for (int a = 0; a < sp->nsh_sc; a++)
                sp->connectivity[e * sp->nsh + c * sp->nsh_sc + a] =
                    (i64)c * sp->ndof_sc + sp->conn_sc[e * sp->nsh_sc + a];
    return sp;
}

void orc_space_free(orc_space *sp) {
    if (!sp) return;
    for (int d = 0; d < sp->dim; d++) space1d_free(&sp->univ[d]);
    free(sp->conn_sc); free(sp->connectivity); free(sp);
}

/* info[0]=dim info[1]=nel info[2]=ndof info[3]=ndof_sc info[4]=nsh info[5..7]=ndof_dir info[8..10]=nel_dir */
void orc_space_info(const orc_space *sp, i64 *info) {
    info[0] = sp->dim; info[1] = sp->nel; info[2] = sp->ndof; info[3] = sp->ndof_sc; info[4] = sp->nsh;
    for (int d = 0; d < 3; d++) {
        info[5 + d] = d < sp->dim ? sp->ndof_dir[d] : 1;
        info[8 + d] = d < sp->dim ? sp->nel_dir[d] : 1;
    }
}

void orc_space_connectivity(const orc_space *sp, i64 *conn) {
    memcpy(conn, sp->connectivity, sizeof(i64) * (size_t)(sp->nel * sp->nsh));
}

/* rust/src/iga/space.rs:181-200 greville_points: [ndof_sc][dim] */
void orc_space_greville(const orc_space *sp, double *g) {
    int sub[ORC_MAXD];
    for (i64 i = 0; i < sp->ndof_sc; i++) {
        unravel(i, sp->ndof_dir, sp->dim, sub);
        for (int d = 0; d < sp->dim; d++) {
            const orc_space1d *u = &sp->univ[d];
            int p = u->degree, j = sub[d];
            double m;
            if (p == 0) m = 0.5 * (u->knots[j] + u->knots[j + 1]);
            else {
                double s = 0.0;
                for (int k = j + 1; k <= j + p; k++) s += u->knots[k];
                m = s / (double)p;
            }
            g[i * sp->dim + d] = sp->lo[d] + sp->lengths[d] * m;
        }
    }
}

/* ------------------------------------------------------------------------------------------ */
/* elasticity.rs                                                                              */
/* ------------------------------------------------------------------------------------------ */

/* rust/src/iga/elasticity.rs:173-177 lame */
void orc_lame(double young, double poisson, double *lambda, double *mu) {
    *lambda = young * poisson / ((1.0 + poisson) * (1.0 - 2.0 * poisson));
    *mu = young / (2.0 * (1.0 + poisson));
}

/* rust/src/iga/elasticity.rs:153-171 kron (b index fastest, zero entries of a skipped) */
static void kron(const double *a, int na, const double *b, int nb, double *out) {
    int n = na * nb;
    memset(out, 0, sizeof(double) * (size_t)(n * n));
    for (int ia = 0; ia < na; ia++)
        for (int ja = 0; ja < na; ja++) {
            double av = a[ia * na + ja];
            if (av == 0.0) continue;
            for (int ib = 0; ib < nb; ib++)
                for (int jb = 0; jb < nb; jb++)
                    out[(ia * nb + ib) * n + ja * nb + jb] = av * b[ib * nb + jb];
        }
}

/* rust/src/iga/elasticity.rs:30-150 elasticity_element_matrices.
 * Writes up to max_types row-major [nsh x nsh] matrices into `types` and the type of every
 * element into `type_id`; also the 1-D type of every element per direction into tid_dir
 * (tid_dir[d*max_nel_dir + e_d], may be NULL).  Returns ntypes, or -1 if max_types is too small. */
int orc_elasticity_element_matrices(const orc_space *sp, double lambda, double mu, double *types,
                                    i64 *type_id, int max_types, int *tid_dir_out, int max_nel_dir) {
    int dim = sp->dim, nsh_sc = sp->nsh_sc, nsh = sp->nsh;
    /* per direction: distinct 1-D matrix quadruples and the per-element 1-D type */
    double *mats[ORC_MAXD];      /* [ndistinct][4][nl*nl] */
    int *tid_dir[ORC_MAXD];
    for (int d = 0; d < dim; d++) {
        const orc_space1d *u = &sp->univ[d];
        double ld = sp->lengths[d];
        int nl = u->degree + 1, nn = nl * nl;
        double *per = (double *)calloc((size_t)u->nel * 4 * nn, sizeof(double));
        double scale = 0.0;
        for (int e = 0; e < u->nel; e++) {
            double *m = per + (size_t)e * 4 * nn;
            for (int q = 0; q < u->nquad; q++) {
                double w = u->qw[e * u->nquad + q] * ld;
                int base = (e * u->nquad + q) * nl;
                for (int a = 0; a < nl; a++) {
                    double na = u->shape[base + a];
                    double da = u->dshape[base + a] / ld;
                    for (int b = 0; b < nl; b++) {
                        double nb = u->shape[base + b];
                        double db = u->dshape[base + b] / ld;
                        m[0 * nn + a * nl + b] += w * na * nb;
                        m[1 * nn + a * nl + b] += w * da * nb;
                        m[2 * nn + a * nl + b] += w * na * db;
                        m[3 * nn + a * nl + b] += w * da * db;
                    }
                }
            }
            for (int k = 0; k < 4 * nn; k++) scale = fmax(scale, fabs(m[k]));
        }
        i64 *keys = (i64 *)malloc(sizeof(i64) * (size_t)u->nel * 4 * nn);
        int nd = 0;
        tid_dir[d] = (int *)malloc(sizeof(int) * (size_t)u->nel);
        mats[d] = (double *)malloc(sizeof(double) * (size_t)u->nel * 4 * nn);
        for (int e = 0; e < u->nel; e++) {
            const double *m = per + (size_t)e * 4 * nn;
            i64 key[4 * 16 * 16];
            for (int k = 0; k < 4 * nn; k++) key[k] = (i64)round(m[k] / scale * 1e12);
            int t = -1;
            for (int j = 0; j < nd && t < 0; j++)
                if (memcmp(keys + (size_t)j * 4 * nn, key, sizeof(i64) * 4 * nn) == 0) t = j;
            if (t < 0) {
                t = nd++;
                memcpy(keys + (size_t)t * 4 * nn, key, sizeof(i64) * 4 * nn);
                memcpy(mats[d] + (size_t)t * 4 * nn, m, sizeof(double) * 4 * nn);
            }
            tid_dir[d][e] = t;
        }
        free(keys); free(per);
    }
    /* element types = distinct combinations of 1-D types in element order */
    int combos[512][ORC_MAXD];
    int ncombo = 0;
    int esub[ORC_MAXD];
    for (i64 e = 0; e < sp->nel; e++) {
        unravel(e, sp->nel_dir, dim, esub);
        int key[ORC_MAXD];
        for (int d = 0; d < dim; d++) key[d] = tid_dir[d][esub[d]];
        int t = -1;
        for (int j = 0; j < ncombo && t < 0; j++) {
            int same = 1;
            for (int d = 0; d < dim; d++) same &= combos[j][d] == key[d];
            if (same) t = j;
        }
        if (t < 0) {
            t = ncombo++;
            for (int d = 0; d < dim; d++) combos[t][d] = key[d];
        }
        type_id[e] = t;
    }
    if (tid_dir_out)
        for (int d = 0; d < dim; d++)
            for (int e = 0; e < sp->nel_dir[d]; e++) tid_dir_out[d * max_nel_dir + e] = tid_dir[d][e];
    if (ncombo > max_types) {
        for (int d = 0; d < dim; d++) { free(mats[d]); free(tid_dir[d]); }
        return -1;
    }
    size_t nsc2 = (size_t)nsh_sc * nsh_sc;
    double *g = (double *)malloc(sizeof(double) * 9 * nsc2);
    double *tmpa = (double *)malloc(sizeof(double) * nsc2);
    double *tmpb = (double *)malloc(sizeof(double) * nsc2);
    double *lap = (double *)malloc(sizeof(double) * nsc2);
    for (int t = 0; t < ncombo; t++) {
        for (int i = 0; i < dim; i++)
            for (int j = 0; j < dim; j++) {
                double *gij = tmpa;
                gij[0] = 1.0;
                int n = 1;
                for (int d = 0; d < dim; d++) {
                    int k = (d == i && d == j) ? 3 : (d == i) ? 1 : (d == j) ? 2 : 0;
                    int nl = sp->nsh_dir[d];
                    const double *m = mats[d] + ((size_t)combos[t][d] * 4 + k) * nl * nl;
                    kron(m, nl, gij, n, tmpb);
                    n *= nl;
                    memcpy(tmpa, tmpb, sizeof(double) * (size_t)n * n);
                }
                memcpy(g + (size_t)(i * 3 + j) * nsc2, tmpa, sizeof(double) * nsc2);
            }
        for (size_t l = 0; l < nsc2; l++) lap[l] = 0.0;
        for (int k = 0; k < dim; k++)
            for (size_t l = 0; l < nsc2; l++) lap[l] += g[(size_t)(k * 3 + k) * nsc2 + l];
        double *ke = types + (size_t)t * nsh * nsh;
        for (int ci = 0; ci < dim; ci++)
            for (int cj = 0; cj < dim; cj++)
                for (int a = 0; a < nsh_sc; a++)
                    for (int b = 0; b < nsh_sc; b++) {
                        double v = lambda * g[(size_t)(ci * 3 + cj) * nsc2 + a * nsh_sc + b] +
                                   mu * g[(size_t)(cj * 3 + ci) * nsc2 + a * nsh_sc + b];
                        if (ci == cj) v += mu * lap[a * nsh_sc + b];
                        ke[(size_t)(ci * nsh_sc + a) * nsh + cj * nsh_sc + b] = v;
                    }
    }
    free(g); free(tmpa); free(tmpb); free(lap);
    for (int d = 0; d < dim; d++) { free(mats[d]); free(tid_dir[d]); }
    return ncombo;
}

/* ------------------------------------------------------------------------------------------ */
/* fields.rs                                                                                  */
/* ------------------------------------------------------------------------------------------ */

/* rust/src/iga/fields.rs:9-27 element_quad_points */
static void element_quad_points(const orc_space *sp, i64 e, double (*x)[3], double *w) {
    int esub[ORC_MAXD], qsub[ORC_MAXD];
    unravel(e, sp->nel_dir, sp->dim, esub);
    for (int q = 0; q < sp->nqn; q++) {
        unravel(q, sp->nquad, sp->dim, qsub);
        double xq[3] = {0, 0, 0}, wq = 1.0;
        for (int d = 0; d < sp->dim; d++) {
            const orc_space1d *u = &sp->univ[d];
            int k = esub[d] * u->nquad + qsub[d];
            xq[d] = sp->lo[d] + sp->lengths[d] * u->qn[k];
            wq *= sp->lengths[d] * u->qw[k];
        }
        x[q][0] = xq[0]; x[q][1] = xq[1]; x[q][2] = xq[2];
        w[q] = wq;
    }
}

/* rust/src/iga/fields.rs:31-53 element_shape_functions (values only) */
static void element_shape_values(const orc_space *sp, i64 e, double *n) {
    int esub[ORC_MAXD], qsub[ORC_MAXD], asub[ORC_MAXD];
    unravel(e, sp->nel_dir, sp->dim, esub);
    for (int i = 0; i < sp->nqn * sp->nsh_sc; i++) n[i] = 1.0;
    for (int q = 0; q < sp->nqn; q++) {
        unravel(q, sp->nquad, sp->dim, qsub);
        for (int a = 0; a < sp->nsh_sc; a++) {
            unravel(a, sp->nsh_dir, sp->dim, asub);
            for (int d = 0; d < sp->dim; d++) {
                const orc_space1d *u = &sp->univ[d];
                int idx = (esub[d] * u->nquad + qsub[d]) * (u->degree + 1) + asub[d];
                n[q * sp->nsh_sc + a] *= u->shape[idx];
            }
        }
    }
}

/* Load functions used by the reference's tests:
 * kind 0: rust/tests/iga_vs_matlab.rs:62-68 (the fixture load)
 * kind 1: rust/tests/iga_kernel.rs:201-207 (plane-strain MMS load; params = lambda, mu) */
static void load_fn(int kind, const double *prm, int dim, const double *x, double *f) {
    const double PI = 3.14159265358979323846;
    if (kind == 0) {
        if (dim == 2) { f[0] = x[0] * x[1]; f[1] = sin(x[0]) + x[1] * x[1]; f[2] = 0.0; }
        else { f[0] = x[0] * x[1]; f[1] = sin(x[0]) + x[2]; f[2] = x[1] * x[1]; }
    } else {
        double lam = prm[0], mu = prm[1];
        f[0] = PI * PI * (lam + 3.0 * mu) * sin(PI * x[0]) * sin(PI * x[1]);
        f[1] = -PI * PI * (lam + mu) * cos(PI * x[0]) * cos(PI * x[1]);
        f[2] = 0.0;
    }
}

/* rust/src/iga/fields.rs:56-76 load_vector */
void orc_load_vector(const orc_space *sp, int kind, const double *prm, double *out) {
    memset(out, 0, sizeof(double) * (size_t)sp->ndof);
    double (*x)[3] = (double (*)[3])malloc(sizeof(double) * 3 * (size_t)sp->nqn);
    double *w = (double *)malloc(sizeof(double) * (size_t)sp->nqn);
    double *n = (double *)malloc(sizeof(double) * (size_t)(sp->nqn * sp->nsh_sc));
    for (i64 e = 0; e < sp->nel; e++) {
        element_quad_points(sp, e, x, w);
        element_shape_values(sp, e, n);
        for (int q = 0; q < sp->nqn; q++) {
            double fq[3];
            load_fn(kind, prm, sp->dim, x[q], fq);
            for (int a = 0; a < sp->nsh_sc; a++) {
                i64 g = sp->conn_sc[e * sp->nsh_sc + a];
                double wn = w[q] * n[q * sp->nsh_sc + a];
                for (int c = 0; c < sp->dim; c++) out[c * sp->ndof_sc + g] += wn * fq[c];
            }
        }
    }
    free(x); free(w); free(n);
}

/* rust/src/iga/fields.rs:80-94 element_vector_values + rust/tests/iga_kernel.rs:210-219:
 * L2 error of u against the plane-strain MMS field (sin(pi x) sin(pi y), 0). */
double orc_mms_l2_error(const orc_space *sp, const double *u) {
    const double PI = 3.14159265358979323846;
    double (*x)[3] = (double (*)[3])malloc(sizeof(double) * 3 * (size_t)sp->nqn);
    double *w = (double *)malloc(sizeof(double) * (size_t)sp->nqn);
    double *n = (double *)malloc(sizeof(double) * (size_t)(sp->nqn * sp->nsh_sc));
    double e2 = 0.0;
    for (i64 e = 0; e < sp->nel; e++) {
        element_quad_points(sp, e, x, w);
        element_shape_values(sp, e, n);
        for (int q = 0; q < sp->nqn; q++) {
            double v[3] = {0, 0, 0};
            for (int a = 0; a < sp->nsh_sc; a++) {
                i64 g = sp->conn_sc[e * sp->nsh_sc + a];
                for (int c = 0; c < sp->dim; c++) v[c] += n[q * sp->nsh_sc + a] * u[c * sp->ndof_sc + g];
            }
            double ex = sin(PI * x[q][0]) * sin(PI * x[q][1]);
            e2 += w[q] * (pow(v[0] - ex, 2.0) + pow(v[1], 2.0));
        }
    }
    free(x); free(w); free(n);
    return sqrt(e2);
}

/* ------------------------------------------------------------------------------------------ */
/* sparse.rs                                                                                  */
/* ------------------------------------------------------------------------------------------ */

typedef struct {
    i64 nrows, ncols;
    i64 *indptr, *indices;
    double *data;
} orc_csr;

static int cmp_pair(const void *a, const void *b) {
    const i64 *x = (const i64 *)a, *y = (const i64 *)b;
    if (x[0] != y[0]) return x[0] < y[0] ? -1 : 1;
    return x[1] < y[1] ? -1 : (x[1] > y[1]);
}

/* rust/src/sparse.rs:16-57 CsrMatrix::from_triplets (duplicates summed; ties in input order) */
orc_csr *orc_csr_from_triplets(i64 nrows, i64 ncols, i64 nt, const i64 *rows, const i64 *cols,
                               const double *vals) {
    i64 *count = (i64 *)calloc((size_t)nrows + 1, sizeof(i64));
    for (i64 k = 0; k < nt; k++) count[rows[k] + 1]++;
    for (i64 i = 0; i < nrows; i++) count[i + 1] += count[i];
    i64 *next = (i64 *)malloc(sizeof(i64) * (size_t)(nrows + 1));
    memcpy(next, count, sizeof(i64) * (size_t)(nrows + 1));
    i64 *ci = (i64 *)malloc(sizeof(i64) * (size_t)(nt > 0 ? nt : 1));
    double *cv = (double *)malloc(sizeof(double) * (size_t)(nt > 0 ? nt : 1));
    for (i64 k = 0; k < nt; k++) {
        i64 r = rows[k];
        ci[next[r]] = cols[k];
        cv[next[r]] = vals[k];
        next[r]++;
    }
    orc_csr *m = (orc_csr *)calloc(1, sizeof(orc_csr));
    m->nrows = nrows; m->ncols = ncols;
    m->indptr = (i64 *)calloc((size_t)nrows + 1, sizeof(i64));
    m->indices = (i64 *)malloc(sizeof(i64) * (size_t)(nt > 0 ? nt : 1));
    m->data = (double *)malloc(sizeof(double) * (size_t)(nt > 0 ? nt : 1));
    i64 nnz = 0;
    i64 *perm = (i64 *)malloc(sizeof(i64) * 2 * (size_t)(nt > 0 ? nt : 1));
    for (i64 r = 0; r < nrows; r++) {
        i64 s = count[r], e = count[r + 1], len = e - s;
        for (i64 k = 0; k < len; k++) { perm[2 * k] = ci[s + k]; perm[2 * k + 1] = s + k; }
        qsort(perm, (size_t)len, 2 * sizeof(i64), cmp_pair);
        i64 last = -1;
        for (i64 k = 0; k < len; k++) {
            i64 kk = perm[2 * k + 1];
            if (last == ci[kk]) m->data[nnz - 1] += cv[kk];
            else { m->indices[nnz] = ci[kk]; m->data[nnz] = cv[kk]; nnz++; last = ci[kk]; }
        }
        m->indptr[r + 1] = nnz;
    }
    free(perm); free(count); free(next); free(ci); free(cv);
    return m;
}

void orc_csr_free(orc_csr *m) {
    if (!m) return;
    free(m->indptr); free(m->indices); free(m->data); free(m);
}

i64 orc_csr_nnz(const orc_csr *m) { return m->indptr[m->nrows]; }

/* rust/src/sparse.rs:60-68 CsrMatrix::matvec (parallel over rows) */
void orc_csr_matvec(const orc_csr *m, const double *x, double *y) {
#pragma omp parallel for schedule(static)
    for (i64 r = 0; r < m->nrows; r++) {
        double s = 0.0;
        for (i64 k = m->indptr[r]; k < m->indptr[r + 1]; k++) s += m->data[k] * x[m->indices[k]];
        y[r] = s;
    }
}

/* rust/src/sparse.rs:70-78 CsrMatrix::diagonal */
void orc_csr_diagonal(const orc_csr *m, double *d) {
    for (i64 r = 0; r < m->nrows; r++) {
        d[r] = 0.0;
        for (i64 k = m->indptr[r]; k < m->indptr[r + 1]; k++)
            if (m->indices[k] == r) { d[r] = m->data[k]; break; }
    }
}

/* rust/src/sparse.rs:89-91 CsrMatrix::frobenius */
double orc_csr_frobenius(const orc_csr *m) {
    double s = 0.0;
    for (i64 k = 0; k < orc_csr_nnz(m); k++) s += m->data[k] * m->data[k];
    return sqrt(s);
}

/* rust/src/sparse.rs:80-86 CsrMatrix::get */
double orc_csr_get(const orc_csr *m, i64 r, i64 c) {
    i64 lo = m->indptr[r], hi = m->indptr[r + 1];
    while (lo < hi) {
        i64 mid = (lo + hi) / 2;
        if (m->indices[mid] == c) return m->data[mid];
        if (m->indices[mid] < c) lo = mid + 1; else hi = mid;
    }
    return 0.0;
}

/* export the CSR arrays (indptr [nrows+1], indices/data [nnz]) */
void orc_csr_export(const orc_csr *m, i64 *indptr, i64 *indices, double *data) {
    memcpy(indptr, m->indptr, sizeof(i64) * (size_t)(m->nrows + 1));
    memcpy(indices, m->indices, sizeof(i64) * (size_t)orc_csr_nnz(m));
    memcpy(data, m->data, sizeof(double) * (size_t)orc_csr_nnz(m));
}

static int cmp_i64(const void *a, const void *b) {
    i64 x = *(const i64 *)a, y = *(const i64 *)b;
    return x < y ? -1 : (x > y);
}

/* rust/src/sparse.rs:128-157 AssemblyPattern::new followed by :160-175 assemble with
 * elem(e) = types[type_id[e]] and scale[e] (NULL scale = 1, as in sparse.rs:189). */
orc_csr *orc_assemble_pattern(i64 ndof, const i64 *conn, int nsh, i64 nel, const double *types,
                              const i64 *type_id, const double *scale) {
    i64 *rowlen = (i64 *)calloc((size_t)ndof + 1, sizeof(i64));
    for (i64 e = 0; e < nel; e++)
        for (int a = 0; a < nsh; a++) rowlen[conn[e * nsh + a] + 1] += nsh;
    for (i64 i = 0; i < ndof; i++) rowlen[i + 1] += rowlen[i];
    i64 *fill = (i64 *)malloc(sizeof(i64) * (size_t)ndof);
    for (i64 i = 0; i < ndof; i++) fill[i] = rowlen[i];
    i64 *rows = (i64 *)malloc(sizeof(i64) * (size_t)(rowlen[ndof] > 0 ? rowlen[ndof] : 1));
    for (i64 e = 0; e < nel; e++) {
        const i64 *ce = conn + e * nsh;
        for (int a = 0; a < nsh; a++) {
            i64 r = ce[a];
            for (int b = 0; b < nsh; b++) rows[fill[r]++] = ce[b];
        }
    }
    orc_csr *m = (orc_csr *)calloc(1, sizeof(orc_csr));
    m->nrows = ndof; m->ncols = ndof;
    m->indptr = (i64 *)calloc((size_t)ndof + 1, sizeof(i64));
    i64 nnz = 0;
    for (i64 r = 0; r < ndof; r++) {
        i64 s = rowlen[r], len = rowlen[r + 1] - s;
        qsort(rows + s, (size_t)len, sizeof(i64), cmp_i64);
        i64 w = 0;
        for (i64 k = 0; k < len; k++)
            if (w == 0 || rows[s + k] != rows[s + w - 1]) rows[s + w++] = rows[s + k];
        nnz += w;
        m->indptr[r + 1] = nnz;
        fill[r] = w;
    }
    m->indices = (i64 *)malloc(sizeof(i64) * (size_t)(nnz > 0 ? nnz : 1));
    for (i64 r = 0; r < ndof; r++)
        memcpy(m->indices + m->indptr[r], rows + rowlen[r], sizeof(i64) * (size_t)fill[r]);
    free(rows); free(rowlen); free(fill);
    m->data = (double *)calloc((size_t)(nnz > 0 ? nnz : 1), sizeof(double));
    /* assemble: data[pos[k]] += s * ke[k], elements in order (sparse.rs:166-172) */
    for (i64 e = 0; e < nel; e++) {
        const i64 *ce = conn + e * nsh;
        const double *ke = types + (size_t)type_id[e] * nsh * nsh;
        double s = scale ? scale[e] : 1.0;
        for (int a = 0; a < nsh; a++) {
            i64 r = ce[a];
            const i64 *row = m->indices + m->indptr[r];
            i64 len = m->indptr[r + 1] - m->indptr[r];
            for (int b = 0; b < nsh; b++) {
                i64 c = ce[b], lo = 0, hi = len;
                while (lo < hi) {
                    i64 mid = (lo + hi) / 2;
                    if (row[mid] < c) lo = mid + 1; else hi = mid;
                }
                m->data[m->indptr[r] + lo] += s * ke[a * nsh + b];
            }
        }
    }
    return m;
}

/* rust/src/sparse.rs:179-200 assemble (triplet path) */
orc_csr *orc_assemble_triplets(i64 ndof, const i64 *conn, int nsh, i64 nel, const double *types,
                               const i64 *type_id, const double *scale) {
    i64 nt = (i64)nsh * nsh * nel;
    i64 *r = (i64 *)malloc(sizeof(i64) * (size_t)nt);
    i64 *c = (i64 *)malloc(sizeof(i64) * (size_t)nt);
    double *v = (double *)malloc(sizeof(double) * (size_t)nt);
    i64 k = 0;
    for (i64 e = 0; e < nel; e++) {
        const double *ke = types + (size_t)type_id[e] * nsh * nsh;
        double s = scale ? scale[e] : 1.0;
        const i64 *ce = conn + e * nsh;
        for (int a = 0; a < nsh; a++)
            for (int b = 0; b < nsh; b++) { r[k] = ce[a]; c[k] = ce[b]; v[k] = s * ke[a * nsh + b]; k++; }
    }
    orc_csr *m = orc_csr_from_triplets(ndof, ndof, nt, r, c, v);
    free(r); free(c); free(v);
    return m;
}

/* ------------------------------------------------------------------------------------------ */
/* Matrix-free element operator (CPU).  The same y = sum_e s_e K_type(e) u_e as the assembled  */
/* CSR, evaluated element by element as in rust/src/bin/wgpu_matrixfree_benchmark.rs:348-371  */
/* and src/fastformation/topopt_iga_3d.m:252-260.  The scatter runs in 27 colours             */
/* (e_d mod 3), so elements of one colour share no control point and the sum order is fixed.  */
/* 3-D, p = 2 only (nsh = 81).                                                                 */
/* ------------------------------------------------------------------------------------------ */

/* mask_mode: 0 y = K x; 1 y = m.*K(m.*x) (rust/src/topopt_iga.rs:151-159); 2 y = K(m.*x) on free
 * rows and y = x on fixed rows (rust/tests/iga_kernel.rs:101-107). */
void orc_mf_apply(const orc_space *sp, const double *types, const i64 *type_id, const double *scale,
                  const uint8_t *free_mask, int mask_mode, const double *x, double *y) {
    const int nsh = 81;
    i64 nx = sp->nel_dir[0], ny = sp->nel_dir[1], nz = sp->nel_dir[2];
    i64 ncx = sp->ndof_dir[0], ncy = sp->ndof_dir[1], nsc = sp->ndof_sc;
    memset(y, 0, sizeof(double) * (size_t)sp->ndof);
    const double *xm = x;
    double *xbuf = NULL;
    if (mask_mode != 0 && free_mask) {
        xbuf = (double *)malloc(sizeof(double) * (size_t)sp->ndof);
        for (i64 i = 0; i < sp->ndof; i++) xbuf[i] = free_mask[i] ? x[i] : 0.0;
        xm = xbuf;
    }
    for (int color = 0; color < 27; color++) {
        int cx = color % 3, cy = (color / 3) % 3, cz = color / 9;
        i64 mx = (nx - cx + 2) / 3, my = (ny - cy + 2) / 3, mz = (nz - cz + 2) / 3;
        i64 cnt = mx * my * mz;
#pragma omp parallel for schedule(static)
        for (i64 t = 0; t < cnt; t++) {
            i64 ex = cx + 3 * (t % mx), ey = cy + 3 * ((t / mx) % my), ez = cz + 3 * (t / (mx * my));
            i64 e = ex + nx * (ey + ny * ez);
            double ue[81], ye[81];
            i64 idx[81];
            for (int c = 0; c < 3; c++)
                for (int a = 0; a < 27; a++) {
                    int ax = a % 3, ay = (a / 3) % 3, az = a / 9;
                    i64 g = (ex + ax) + ncx * ((ey + ay) + ncy * (ez + az));
                    idx[c * 27 + a] = c * nsc + g;
                    ue[c * 27 + a] = xm[c * nsc + g];
                }
            const double *ke = types + (size_t)type_id[e] * nsh * nsh;
            double s = scale ? scale[e] : 1.0;
            for (int a = 0; a < nsh; a++) {
                double acc = 0.0;
                for (int b = 0; b < nsh; b++) acc += ke[a * nsh + b] * ue[b];
                ye[a] = s * acc;
            }
            for (int a = 0; a < nsh; a++) y[idx[a]] += ye[a];
        }
    }
    if (mask_mode == 1 && free_mask) {
        for (i64 i = 0; i < sp->ndof; i++) if (!free_mask[i]) y[i] = 0.0;
    } else if (mask_mode == 2 && free_mask) {
        for (i64 i = 0; i < sp->ndof; i++) if (!free_mask[i]) y[i] = x[i];
    }
    free(xbuf);
}

/* Jacobi diagonal sum_e s_e K_type(e)[a,a], elements in increasing order (the order in which
 * rust/src/sparse.rs:166-172 accumulates the CSR entries, so it equals CsrMatrix::diagonal). */
void orc_mf_diagonal(const orc_space *sp, const double *types, const i64 *type_id, const double *scale,
                     double *d) {
    const int nsh = sp->nsh;
    memset(d, 0, sizeof(double) * (size_t)sp->ndof);
    for (i64 e = 0; e < sp->nel; e++) {
        const double *ke = types + (size_t)type_id[e] * nsh * nsh;
        double s = scale ? scale[e] : 1.0;
        for (int a = 0; a < nsh; a++) d[sp->connectivity[e * nsh + a]] += s * ke[a * nsh + a];
    }
}

/* ------------------------------------------------------------------------------------------ */
/* solver.rs                                                                                  */
/* ------------------------------------------------------------------------------------------ */

typedef struct {
    const orc_csr *csr;            /* assembled operator, or NULL for the matrix-free one */
    const orc_space *sp;
    const double *types; const i64 *type_id; const double *scale;
    const uint8_t *free_mask;
    int mask_mode;
    double *pm, *tmp;
} orc_closure;

/* the masked closures of rust/src/topopt_iga.rs:151-159 (mode 1) and
 * rust/tests/iga_kernel.rs:101-107 (mode 2) */
static void closure_apply(orc_closure *c, const double *p, double *ap, i64 n) {
    if (c->csr) {
        const double *src = p;
        if (c->mask_mode != 0 && c->free_mask) {
            for (i64 i = 0; i < n; i++) c->pm[i] = c->free_mask[i] ? p[i] : 0.0;
            src = c->pm;
        }
        orc_csr_matvec(c->csr, src, c->tmp);
        for (i64 i = 0; i < n; i++) {
            if (c->mask_mode == 1 && c->free_mask) ap[i] = c->free_mask[i] ? c->tmp[i] : 0.0;
            else if (c->mask_mode == 2 && c->free_mask) ap[i] = c->free_mask[i] ? c->tmp[i] : p[i];
            else ap[i] = c->tmp[i];
        }
    } else {
        orc_mf_apply(c->sp, c->types, c->type_id, c->scale, c->free_mask, c->mask_mode, p, ap);
    }
}

/* rust/src/solver.rs:14-76 PcgSolver::solve */
static void pcg_solve(orc_closure *cl, i64 n, const double *b, const double *diag_a, i64 max_iter,
                      double tol, double *x, i64 *iters_out, double *res_out) {
    double *r = (double *)malloc(sizeof(double) * (size_t)n);
    double *z = (double *)malloc(sizeof(double) * (size_t)n);
    double *p = (double *)malloc(sizeof(double) * (size_t)n);
    double *ap = (double *)malloc(sizeof(double) * (size_t)n);
    double *inv_diag = (double *)malloc(sizeof(double) * (size_t)n);
    for (i64 i = 0; i < n; i++) { x[i] = 0.0; r[i] = b[i]; z[i] = 0.0; p[i] = 0.0; ap[i] = 0.0; }
    for (i64 i = 0; i < n; i++) inv_diag[i] = fabs(diag_a[i]) > 1e-12 ? 1.0 / diag_a[i] : 1.0;
    for (i64 i = 0; i < n; i++) { z[i] = inv_diag[i] * r[i]; p[i] = z[i]; }
    double rz_old = 0.0;
    for (i64 i = 0; i < n; i++) rz_old += r[i] * z[i];
    double nb = 0.0;
    for (i64 i = 0; i < n; i++) nb += b[i] * b[i];
    double norm_b = fmax(sqrt(nb), 1e-16);
    double final_res = 1.0;
    i64 final_iter = 0;
    for (i64 iter = 0; iter < max_iter; iter++) {
        final_iter = iter + 1;
        closure_apply(cl, p, ap, n);
        double p_ap = 0.0;
        for (i64 i = 0; i < n; i++) p_ap += p[i] * ap[i];
        if (!(p_ap > 0.0)) break;
        double alpha = rz_old / p_ap;
        for (i64 i = 0; i < n; i++) { x[i] += alpha * p[i]; r[i] -= alpha * ap[i]; }
        double rr = 0.0;
        for (i64 i = 0; i < n; i++) rr += r[i] * r[i];
        final_res = sqrt(rr) / norm_b;
        if (final_res < tol) break;
        for (i64 i = 0; i < n; i++) z[i] = inv_diag[i] * r[i];
        double rz_new = 0.0;
        for (i64 i = 0; i < n; i++) rz_new += r[i] * z[i];
        double beta = rz_new / rz_old;
        for (i64 i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
        rz_old = rz_new;
    }
    *iters_out = final_iter;
    *res_out = final_res;
    free(r); free(z); free(p); free(ap); free(inv_diag);
}

/* PcgSolver::solve with the masked CSR closure */
void orc_pcg_csr(const orc_csr *m, const uint8_t *free_mask, int mask_mode, const double *b,
                 const double *diag, i64 max_iter, double tol, double *x, i64 *iters, double *res) {
    i64 n = m->nrows;
    orc_closure cl = {m, NULL, NULL, NULL, NULL, free_mask, mask_mode, NULL, NULL};
    cl.pm = (double *)malloc(sizeof(double) * (size_t)n);
    cl.tmp = (double *)malloc(sizeof(double) * (size_t)n);
    pcg_solve(&cl, n, b, diag, max_iter, tol, x, iters, res);
    free(cl.pm); free(cl.tmp);
}

/* PcgSolver::solve with the matrix-free closure (large grids) */
void orc_pcg_mf(const orc_space *sp, const double *types, const i64 *type_id, const double *scale,
                const uint8_t *free_mask, int mask_mode, const double *b, const double *diag,
                i64 max_iter, double tol, double *x, i64 *iters, double *res) {
    orc_closure cl = {NULL, sp, types, type_id, scale, free_mask, mask_mode, NULL, NULL};
    pcg_solve(&cl, sp->ndof, b, diag, max_iter, tol, x, iters, res);
}

/* rust/src/topopt_iga.rs:137-162 CantileverTopOpt::solve_state on an assembled operator:
 * warm-started masked solve; returns the relative residual as the reference does. */
void orc_solve_state(const orc_csr *k, const uint8_t *free_mask, const double *force, const double *u0,
                     double pcg_tol, double *u, i64 *iters, double *res) {
    i64 n = k->nrows;
    double *ku0 = (double *)malloc(sizeof(double) * (size_t)n);
    double *b = (double *)malloc(sizeof(double) * (size_t)n);
    double *diag = (double *)malloc(sizeof(double) * (size_t)n);
    double *du = (double *)malloc(sizeof(double) * (size_t)n);
    orc_csr_matvec(k, u0, ku0);
    for (i64 i = 0; i < n; i++) b[i] = free_mask[i] ? force[i] - ku0[i] : 0.0;
    double nb = 0.0, rb = 0.0;
    for (i64 i = 0; i < n; i++) if (free_mask[i]) nb += force[i] * force[i];
    nb = sqrt(nb);
    for (i64 i = 0; i < n; i++) rb += b[i] * b[i];
    rb = sqrt(rb);
    orc_csr_diagonal(k, diag);
    for (i64 i = 0; i < n; i++) diag[i] = fmax(diag[i], 1e-12);
    double tol = rb > 0.0 ? fmin(pcg_tol * nb / rb, 0.5) : 1.0;
    double r0;
    orc_pcg_csr(k, free_mask, 1, b, diag, 20 * n, tol, du, iters, &r0);
    for (i64 i = 0; i < n; i++) u[i] = free_mask[i] ? u0[i] + du[i] : 0.0;
    *res = r0 * rb / fmax(nb, 1e-300);
    free(ku0); free(b); free(diag); free(du);
}

/* ------------------------------------------------------------------------------------------ */
/* topopt_iga.rs: the structured SIMP cantilever loop (the caller of the hot path)            */
/* ------------------------------------------------------------------------------------------ */

/* rust/src/topopt_iga.rs:73-234 CantileverTopOpt::{new, run}.  cfg = [size0, size1, size2,
 * volfrac, penal, rmin, young, poisson, emin, move_limit, pcg_tol]; nel[3]; max_iter.
 * nload > 0 replaces the reference's single tip load by nload load cases (forces[nload * ndof]):
 * each case keeps its own warm-started state, the compliance is |sum_k F_k'u_k| and the element
 * energies are summed over the cases (the reference loop is the case nload = 1).
 * Outputs: compliance[max_iter] (per iteration), density[nel]; returns iterations run. */
int orc_topopt_run_loads(const int *nel, const double *cfg, int max_iter, int nload_cases, const double *forces,
                         double *compliance_out, double *density_out, i64 *pcg_iters_out) {
    double bounds[6] = {0.0, cfg[0], 0.0, cfg[1], 0.0, cfg[2]};
    double volfrac = cfg[3], penal = cfg[4], rmin = cfg[5], young = cfg[6], poisson = cfg[7];
    double emin = cfg[8], move = cfg[9], pcg_tol = cfg[10];
    orc_space *sp = orc_space_new(3, bounds, nel, 2);
    double lambda, mu;
    orc_lame(young, poisson, &lambda, &mu);
    double *types = (double *)malloc(sizeof(double) * 125 * 81 * 81);
    i64 *type_id = (i64 *)malloc(sizeof(i64) * (size_t)sp->nel);
    orc_elasticity_element_matrices(sp, lambda, mu, types, type_id, 125, NULL, 0);
    i64 n = sp->ndof, ne = sp->nel;
    const int *nd = sp->ndof_dir;
    uint8_t *free_mask = (uint8_t *)malloc((size_t)n);
    memset(free_mask, 1, (size_t)n);
    double *force = (double *)calloc((size_t)n, sizeof(double));
    i64 *load = (i64 *)malloc(sizeof(i64) * (size_t)sp->ndof_sc);
    i64 nload = 0;
    int s[3];
    for (i64 i = 0; i < sp->ndof_sc; i++) {
        unravel(i, nd, 3, s);
        if (s[0] == 0) for (int c = 0; c < 3; c++) free_mask[c * sp->ndof_sc + i] = 0;
        int i1 = s[0] + 1;
        double i2 = (double)s[1] + 1.0, i3 = (double)s[2] + 1.0;
        if (i1 == nd[0] && fabs(i2 - 1.0) <= 1.0 && fabs(i3 - (double)nd[2] / 2.0) <= 1.0) load[nload++] = i;
    }
    for (i64 k = 0; k < nload; k++) force[sp->ndof_sc + load[k]] = -1.0 / (double)nload;
    int ncase = nload_cases > 0 ? nload_cases : 1;
    const double *fcase = nload_cases > 0 ? forces : force;
    /* sensitivity filter (rust/src/topopt_iga.rs:94-120) */
    double h[3];
    for (int d = 0; d < 3; d++) h[d] = sp->lengths[d] / (double)sp->nel_dir[d];
    double r = rmin * (h[0] + h[1] + h[2]) / 3.0;
    double (*cen)[3] = (double (*)[3])malloc(sizeof(double) * 3 * (size_t)ne);
    for (i64 e = 0; e < ne; e++) {
        unravel(e, sp->nel_dir, 3, s);
        for (int d = 0; d < 3; d++) cen[e][d] = ((double)s[d] + 0.5) * h[d];
    }
    i64 *fptr = (i64 *)calloc((size_t)ne + 1, sizeof(i64));
    i64 cap = 64 * ne, nf = 0;
    i64 *fidx = (i64 *)malloc(sizeof(i64) * (size_t)cap);
    double *fw = (double *)malloc(sizeof(double) * (size_t)cap);
    double *fsum = (double *)malloc(sizeof(double) * (size_t)ne);
    for (i64 e = 0; e < ne; e++) {
        for (i64 f = 0; f < ne; f++) {
            double d2 = pow(cen[e][0] - cen[f][0], 2.0) + pow(cen[e][1] - cen[f][1], 2.0) +
                        pow(cen[e][2] - cen[f][2], 2.0);
            if (d2 <= r * r) {
                if (nf == cap) {
                    cap *= 2;
                    fidx = (i64 *)realloc(fidx, sizeof(i64) * (size_t)cap);
                    fw = (double *)realloc(fw, sizeof(double) * (size_t)cap);
                }
                fidx[nf] = f; fw[nf] = fmax(r - sqrt(d2), 0.0); nf++;
            }
        }
        fptr[e + 1] = nf;
        double sm = 0.0;
        for (i64 k = fptr[e]; k < nf; k++) sm += fw[k];
        fsum[e] = sm;
    }
    /* AssemblyPattern::new once (topopt_iga.rs:121) */
    double *x = (double *)malloc(sizeof(double) * (size_t)ne);
    double *x_old = (double *)malloc(sizeof(double) * (size_t)ne);
    double *cand = (double *)malloc(sizeof(double) * (size_t)ne);
    double *scale = (double *)malloc(sizeof(double) * (size_t)ne);
    double *ee = (double *)malloc(sizeof(double) * (size_t)ne);
    double *dc_raw = (double *)malloc(sizeof(double) * (size_t)ne);
    double *dc = (double *)malloc(sizeof(double) * (size_t)ne);
    double *u_all = (double *)calloc((size_t)n * (size_t)ncase, sizeof(double));
    double *un = (double *)malloc(sizeof(double) * (size_t)n);
    for (i64 e = 0; e < ne; e++) x[e] = volfrac;
    int done = 0;
    for (int iter = 1; iter <= max_iter; iter++) {
        memcpy(x_old, x, sizeof(double) * (size_t)ne);
        for (i64 e = 0; e < ne; e++) scale[e] = emin + (1.0 - emin) * pow(x[e], penal);
        orc_csr *k = orc_assemble_pattern(n, sp->connectivity, 81, ne, types, type_id, scale);
        i64 it = 0;
        double c = 0.0;
        for (i64 e = 0; e < ne; e++) ee[e] = 0.0;
        for (int q = 0; q < ncase; q++) {
            const double *fq = fcase + (size_t)q * (size_t)n;
            double *u = u_all + (size_t)q * (size_t)n;
            i64 itq; double res;
            orc_solve_state(k, free_mask, fq, u, pcg_tol, un, &itq, &res);
            it += itq;
            memcpy(u, un, sizeof(double) * (size_t)n);
            double cq = 0.0;
            for (i64 i = 0; i < n; i++) cq += fq[i] * u[i];
            c += cq;
            /* element_energies (topopt_iga.rs:165-184), summed over the cases */
            for (i64 e = 0; e < ne; e++) {
                const double *ke = types + (size_t)type_id[e] * 81 * 81;
                const i64 *ce = sp->connectivity + e * 81;
                double sm = 0.0;
                for (int a = 0; a < 81; a++) {
                    double ua = u[ce[a]], row = 0.0;
                    for (int b = 0; b < 81; b++) row += ke[a * 81 + b] * u[ce[b]];
                    sm += ua * row;
                }
                ee[e] += sm;
            }
        }
        orc_csr_free(k);
        for (i64 e = 0; e < ne; e++) dc_raw[e] = -penal * (1.0 - emin) * pow(x[e], penal - 1.0) * ee[e];
        for (i64 e = 0; e < ne; e++) {
            double sm = 0.0;
            for (i64 q = fptr[e]; q < fptr[e + 1]; q++) sm += fw[q] * x[fidx[q]] * dc_raw[fidx[q]];
            dc[e] = sm / (fsum[e] * fmax(x[e], 1e-3));
        }
        double l1 = 0.0, mx = 0.0;
        for (i64 e = 0; e < ne; e++) mx = fmax(mx, fabs(dc[e]));
        double l2 = 2.0 * mx;
        memcpy(cand, x_old, sizeof(double) * (size_t)ne);
        while ((l2 - l1) / (l1 + l2 + 1e-10) > 1e-4) {
            double lmid = 0.5 * (l1 + l2);
            for (i64 e = 0; e < ne; e++) {
                double be = sqrt(-dc[e] / lmid);
                cand[e] = fmax(fmax(fmin(fmin(x_old[e] * be, x_old[e] + move), 1.0), x_old[e] - move), 0.001);
            }
            double mean = 0.0;
            for (i64 e = 0; e < ne; e++) mean += cand[e];
            mean /= (double)ne;
            if (mean > volfrac) l1 = lmid; else l2 = lmid;
        }
        memcpy(x, cand, sizeof(double) * (size_t)ne);
        double change = 0.0;
        for (i64 e = 0; e < ne; e++) change = fmax(change, fabs(x[e] - x_old[e]));
        compliance_out[iter - 1] = fabs(c);
        if (pcg_iters_out) pcg_iters_out[iter - 1] = it;
        done = iter;
        if (change < 0.01 && iter >= 15) break;
    }
    memcpy(density_out, x, sizeof(double) * (size_t)ne);
    free(x); free(x_old); free(cand); free(scale); free(ee); free(dc_raw); free(dc); free(u_all); free(un);
    free(cen); free(fptr); free(fidx); free(fw); free(fsum);
    free(types); free(type_id); free(free_mask); free(force); free(load);
    orc_space_free(sp);
    return done;
}

int orc_topopt_run(const int *nel, const double *cfg, int max_iter, double *compliance_out,
                   double *density_out, i64 *pcg_iters_out) {
    return orc_topopt_run_loads(nel, cfg, max_iter, 0, NULL, compliance_out, density_out, pcg_iters_out);
}

/* ------------------------------------------------------------------------------------------ */
/* immersed.rs: cell classification, volume fractions, legacy stabilisation, BCs              */
/* ------------------------------------------------------------------------------------------ */

/* rust/src/immersed.rs:41-77 ParityRayCaster::is_inside */
static int ray_is_inside(const double *tris, const double *yz_box, i64 ntri, const double *q) {
    double qx = q[0], qy = q[1], qz = q[2];
    i64 count = 0;
    for (i64 t = 0; t < ntri; t++) {
        const double *bb = yz_box + 4 * t;
        if (!(qy >= bb[0] && qy <= bb[1] && qz >= bb[2] && qz <= bb[3])) continue;
        const double *a = tris + 9 * t, *b = a + 3, *c = a + 6;
        double v0[2] = {c[1] - a[1], c[2] - a[2]};
        double v1[2] = {b[1] - a[1], b[2] - a[2]};
        double v2[2] = {qy - a[1], qz - a[2]};
        double dot00 = v0[0] * v0[0] + v0[1] * v0[1];
        double dot01 = v0[0] * v1[0] + v0[1] * v1[1];
        double dot02 = v0[0] * v2[0] + v0[1] * v2[1];
        double dot11 = v1[0] * v1[0] + v1[1] * v1[1];
        double dot12 = v1[0] * v2[0] + v1[1] * v2[1];
        double inv = 1.0 / (dot00 * dot11 - dot01 * dot01 + 1e-15);
        double u = (dot11 * dot02 - dot01 * dot12) * inv;
        double v = (dot00 * dot12 - dot01 * dot02) * inv;
        if (u >= 0.0 && v >= 0.0 && u + v <= 1.0) {
            double x_hit = a[0] + v * (b[0] - a[0]) + u * (c[0] - a[0]);
            if (x_hit > qx) count++;
        }
    }
    return (int)(count % 2 == 1);
}

/* rust/src/immersed.rs:80-85 MATLAB-compatible linspace */
static void linspace(double a, double b, int n, double *v) {
    double step = (b - a) / (double)(n - 1);
    for (int i = 0; i < n; i++) v[i] = a + (double)i * step;
    v[n - 1] = b;
}

/* rust/src/immersed.rs:89-155 classify_background_cells + element_weights for a triangle mesh
 * (vertices [nv*3], triangles [ntri*3]).  status: 1 inside, 0 outside, -1 cut. */
void orc_element_weights(const double *verts, const i64 *tri, i64 ntri, const double *bounds,
                         const int *res, const int *sub, double *weights, int8_t *status) {
    double *tris = (double *)malloc(sizeof(double) * 9 * (size_t)ntri);
    double *yz = (double *)malloc(sizeof(double) * 4 * (size_t)ntri);
    for (i64 t = 0; t < ntri; t++) {
        for (int k = 0; k < 3; k++)
            for (int d = 0; d < 3; d++) tris[9 * t + 3 * k + d] = verts[3 * tri[3 * t + k] + d];
        const double *a = tris + 9 * t, *b = a + 3, *c = a + 6;
        yz[4 * t + 0] = fmin(fmin(a[1], b[1]), c[1]);
        yz[4 * t + 1] = fmax(fmax(a[1], b[1]), c[1]);
        yz[4 * t + 2] = fmin(fmin(a[2], b[2]), c[2]);
        yz[4 * t + 3] = fmax(fmax(a[2], b[2]), c[2]);
    }
    double *xs[3];
    for (int d = 0; d < 3; d++) {
        xs[d] = (double *)malloc(sizeof(double) * (size_t)(res[d] + 1));
        linspace(bounds[2 * d], bounds[2 * d + 1], res[d] + 1, xs[d]);
    }
    i64 nv0 = res[0] + 1, nv1 = res[1] + 1, nv2 = res[2] + 1;
    uint8_t *inside = (uint8_t *)malloc((size_t)(nv0 * nv1 * nv2));
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < nv0 * nv1 * nv2; i++) {
        i64 a = i % nv0, b = (i / nv0) % nv1, c = i / (nv0 * nv1);
        double q[3] = {xs[0][a], xs[1][b], xs[2][c]};
        inside[i] = (uint8_t)ray_is_inside(tris, yz, ntri, q);
    }
    for (int k = 0; k < res[2]; k++)
        for (int j = 0; j < res[1]; j++)
            for (int i = 0; i < res[0]; i++) {
                int s = 0;
                for (int dk = 0; dk < 2; dk++)
                    for (int dj = 0; dj < 2; dj++)
                        for (int di = 0; di < 2; di++)
                            s += inside[(i + di) + nv0 * ((j + dj) + nv1 * (k + dk))];
                status[i + res[0] * (j + res[1] * k)] = s == 8 ? 1 : (s == 0 ? 0 : -1);
            }
    double h[3];
    for (int d = 0; d < 3; d++) h[d] = (bounds[2 * d + 1] - bounds[2 * d]) / (double)res[d];
    i64 ncell = (i64)res[0] * res[1] * res[2];
#pragma omp parallel for schedule(dynamic, 16)
    for (i64 e = 0; e < ncell; e++) {
        if (status[e] == 1) { weights[e] = 1.0; continue; }
        if (status[e] == 0) { weights[e] = 0.0; continue; }
        i64 idx[3] = {e % res[0], (e / res[0]) % res[1], e / ((i64)res[0] * res[1])};
        double lo[3], hi[3], dx[3];
        for (int d = 0; d < 3; d++) {
            lo[d] = bounds[2 * d] + (double)idx[d] * h[d];
            hi[d] = bounds[2 * d] + (double)(idx[d] + 1) * h[d];
            dx[d] = (hi[d] - lo[d]) / (double)sub[d];
        }
        i64 n_in = 0;
        for (int c = 0; c < sub[2]; c++)
            for (int b = 0; b < sub[1]; b++)
                for (int a = 0; a < sub[0]; a++) {
                    double q[3] = {lo[0] + ((double)a + 0.5) * dx[0], lo[1] + ((double)b + 0.5) * dx[1],
                                   lo[2] + ((double)c + 0.5) * dx[2]};
                    n_in += ray_is_inside(tris, yz, ntri, q);
                }
        weights[e] = (double)n_in / (double)(sub[0] * sub[1] * sub[2]);
    }
    for (int d = 0; d < 3; d++) free(xs[d]);
    free(inside); free(tris); free(yz);
}

/* Analytic counterpart of element_weights for the solid "unit cube minus three axis-aligned
 * through-cylinders of radius r through the centre" (the immersed benchmark geometry): the same
 * corner classification and midpoint sub-sampling rule as rust/src/immersed.rs:89-155, with an
 * exact inside test instead of ray parity.  Cells [0,1]^3 split into res^3. */
static int cyl_inside(const double *q, double r) {
    if (q[0] < 0.0 || q[0] > 1.0 || q[1] < 0.0 || q[1] > 1.0 || q[2] < 0.0 || q[2] > 1.0) return 0;
    double x = q[0] - 0.5, y = q[1] - 0.5, z = q[2] - 0.5, r2 = r * r;
    if (y * y + z * z < r2) return 0;   /* cylinder along x */
    if (x * x + z * z < r2) return 0;   /* along y */
    if (x * x + y * y < r2) return 0;   /* along z */
    return 1;
}

void orc_cylinders_weights(const int *res, const int *sub, double radius, double *weights, int8_t *status) {
    double *xs[3];
    for (int d = 0; d < 3; d++) {
        xs[d] = (double *)malloc(sizeof(double) * (size_t)(res[d] + 1));
        linspace(0.0, 1.0, res[d] + 1, xs[d]);
    }
    i64 nv0 = res[0] + 1, nv1 = res[1] + 1, nv2 = res[2] + 1;
    uint8_t *inside = (uint8_t *)malloc((size_t)(nv0 * nv1 * nv2));
    for (i64 i = 0; i < nv0 * nv1 * nv2; i++) {
        i64 a = i % nv0, b = (i / nv0) % nv1, c = i / (nv0 * nv1);
        double q[3] = {xs[0][a], xs[1][b], xs[2][c]};
        inside[i] = (uint8_t)cyl_inside(q, radius);
    }
    i64 ncell = (i64)res[0] * res[1] * res[2];
    double h[3];
    for (int d = 0; d < 3; d++) h[d] = 1.0 / (double)res[d];
#pragma omp parallel for schedule(static)
    for (i64 e = 0; e < ncell; e++) {
        i64 i = e % res[0], j = (e / res[0]) % res[1], k = e / ((i64)res[0] * res[1]);
        int s = 0;
        for (int dk = 0; dk < 2; dk++)
            for (int dj = 0; dj < 2; dj++)
                for (int di = 0; di < 2; di++) s += inside[(i + di) + nv0 * ((j + dj) + nv1 * (k + dk))];
        status[e] = s == 8 ? 1 : (s == 0 ? 0 : -1);
        if (status[e] != -1) { weights[e] = status[e] == 1 ? 1.0 : 0.0; continue; }
        i64 idx[3] = {i, j, k};
        double lo[3], dx[3];
        for (int d = 0; d < 3; d++) {
            lo[d] = (double)idx[d] * h[d];
            double hi = (double)(idx[d] + 1) * h[d];
            dx[d] = (hi - lo[d]) / (double)sub[d];
        }
        i64 n_in = 0;
        for (int c = 0; c < sub[2]; c++)
            for (int b = 0; b < sub[1]; b++)
                for (int a = 0; a < sub[0]; a++) {
                    double q[3] = {lo[0] + ((double)a + 0.5) * dx[0], lo[1] + ((double)b + 0.5) * dx[1],
                                   lo[2] + ((double)c + 0.5) * dx[2]};
                    n_in += cyl_inside(q, radius);
                }
        weights[e] = (double)n_in / (double)(sub[0] * sub[1] * sub[2]);
    }
    for (int d = 0; d < 3; d++) free(xs[d]);
    free(inside);
}

/* rust/src/iga/basis.rs:72-135 basis_funs_ders (The NURBS Book A2.3): the p+1 nonzero basis
 * functions at x on knot span s and their derivatives up to order n (n <= p <= 4):
 * ders[k * (p + 1) + r] = d^k/dx^k N_{s - p + r}(x). */
static void ders_basis_funs(const double *knots, int p, double x, int n, int s, double *ders) {
    double ndu[5][5], left[5], right[5], a[2][5];
    ndu[0][0] = 1.0;
    for (int j = 1; j <= p; j++) {
        left[j] = x - knots[s + 1 - j];
        right[j] = knots[s + j] - x;
        double saved = 0.0;
        for (int r = 0; r < j; r++) {
            ndu[j][r] = right[r + 1] + left[j - r];
            double temp = ndu[r][j - 1] / ndu[j][r];
            ndu[r][j] = saved + right[r + 1] * temp;
            saved = left[j - r] * temp;
        }
        ndu[j][j] = saved;
    }
    for (int k = 0; k <= n; k++)
        for (int j = 0; j <= p; j++) ders[k * (p + 1) + j] = 0.0;
    for (int j = 0; j <= p; j++) ders[j] = ndu[j][p];
    for (int r = 0; r <= p; r++) {
        int s1 = 0, s2 = 1;
        a[0][0] = 1.0;
        int kmax = n < p ? n : p;
        for (int k = 1; k <= kmax; k++) {
            double d = 0.0;
            int rk = r - k, pk = p - k;
            if (r >= k) {
                a[s2][0] = a[s1][0] / ndu[pk + 1][rk];
                d = a[s2][0] * ndu[rk][pk];
            }
            int j1 = rk >= -1 ? 1 : -rk;
            int j2 = (r - 1) <= pk ? k - 1 : p - r;
            for (int j = j1; j <= j2; j++) {
                a[s2][j] = (a[s1][j] - a[s1][j - 1]) / ndu[pk + 1][rk + j];
                d += a[s2][j] * ndu[rk + j][pk];
            }
            if (r <= pk) {
                a[s2][k] = -a[s1][k - 1] / ndu[pk + 1][r];
                d += a[s2][k] * ndu[r][pk];
            }
            ders[k * (p + 1) + r] = d;
            int t = s1; s1 = s2; s2 = t;
        }
    }
    double fac = (double)p;
    int kmax = n < p ? n : p;
    for (int k = 1; k <= kmax; k++) {
        for (int j = 0; j <= p; j++) ders[k * (p + 1) + j] *= fac;
        fac *= (double)(p - k);
    }
}

/* rust/src/immersed.rs:224-370 ghost_penalty: returns the triplet count and fills rows/cols/vals
 * when they are non-NULL (call once with NULL to size the buffers). */
i64 orc_ghost_penalty(const orc_space *sp, const int8_t *status, double gamma, double young, i64 *ri, i64 *ci,
                      double *vi) {
    int dim = sp->dim;
    double h[ORC_MAXD];
    for (int d = 0; d < dim; d++) h[d] = sp->lengths[d] / (double)sp->nel_dir[d];
    double hsum = 0.0;
    for (int d = 0; d < dim; d++) hsum += h[d];
    double h_char = hsum / (double)dim;
    /* 1-D tangential mass matrices per direction and element (physical) */
    double *mass[ORC_MAXD];
    for (int d = 0; d < dim; d++) {
        const orc_space1d *u = &sp->univ[d];
        int nl = u->degree + 1;
        mass[d] = (double *)calloc((size_t)u->nel * nl * nl, sizeof(double));
        for (int e = 0; e < u->nel; e++) {
            double *m = mass[d] + (size_t)e * nl * nl;
            for (int q = 0; q < u->nquad; q++) {
                double w = u->qw[e * u->nquad + q] * sp->lengths[d];
                const double *sh = u->shape + (size_t)(e * u->nquad + q) * nl;
                for (int a = 0; a < nl; a++)
                    for (int b = 0; b < nl; b++) m[a * nl + b] += w * sh[a] * sh[b];
            }
        }
    }
    /* 1-D jumps of the p-th derivative across interior break k: indices lo..hi and values */
    int *jlo[ORC_MAXD], *jn[ORC_MAXD];
    double *jval[ORC_MAXD];
    for (int d = 0; d < dim; d++) {
        const orc_space1d *u = &sp->univ[d];
        int p = u->degree, nl = p + 1;
        double lp = pow(sp->lengths[d], (double)p);
        jlo[d] = (int *)calloc((size_t)u->nel, sizeof(int));
        jn[d] = (int *)calloc((size_t)u->nel, sizeof(int));
        jval[d] = (double *)calloc((size_t)u->nel * 2 * nl, sizeof(double));
        for (int k = 1; k < u->nel; k++) {
            double x = u->breaks[k];
            int lf = u->connectivity[(k - 1) * nl], rf = u->connectivity[k * nl];
            double dl[25], dr[25];
            ders_basis_funs(u->knots, p, x, p, lf + p, dl);
            ders_basis_funs(u->knots, p, x, p, rf + p, dr);
            int lo = lf < rf ? lf : rf;
            int hi = (lf + p) > (rf + p) ? (lf + p) : (rf + p);
            jlo[d][k] = lo;
            jn[d][k] = hi - lo + 1;
            for (int g = lo; g <= hi; g++) {
                double r_val = (g >= rf && g <= rf + p) ? dr[p * nl + (g - rf)] : 0.0;
                double l_val = (g >= lf && g <= lf + p) ? dl[p * nl + (g - lf)] : 0.0;
                jval[d][(size_t)k * 2 * nl + (g - lo)] = (r_val - l_val) / lp;
            }
        }
    }
    i64 nt = 0;
    for (int d = 0; d < dim; d++) {
        int p = sp->degree[d];
        double coef = gamma * young * pow(h_char, (double)(2 * p - 1));
        for (i64 e2 = 0; e2 < sp->nel; e2++) {
            int s2[ORC_MAXD], s1[ORC_MAXD];
            unravel(e2, sp->nel_dir, dim, s2);
            if (s2[d] == 0) continue;
            for (int dd = 0; dd < dim; dd++) s1[dd] = s2[dd];
            s1[d] -= 1;
            i64 lin1 = 0, stride = 1;
            for (int dd = 0; dd < dim; dd++) { lin1 += (i64)s1[dd] * stride; stride *= sp->nel_dir[dd]; }
            int a1 = status[lin1] == 1 || status[lin1] == -1, a2 = status[e2] == 1 || status[e2] == -1;
            if (!(a1 && a2 && (status[lin1] == -1 || status[e2] == -1))) continue;
            int nl_d = sp->univ[d].degree + 1;
            const double *jv = jval[d] + (size_t)s2[d] * 2 * nl_d;
            int sizes[ORC_MAXD], first[ORC_MAXD];
            for (int dd = 0; dd < dim; dd++) {
                if (dd == d) { sizes[dd] = jn[d][s2[d]]; first[dd] = jlo[d][s2[d]]; }
                else {
                    const orc_space1d *u = &sp->univ[dd];
                    sizes[dd] = u->degree + 1;
                    first[dd] = u->connectivity[s2[dd] * (u->degree + 1)];
                }
            }
            int nloc = 1;
            for (int dd = 0; dd < dim; dd++) nloc *= sizes[dd];
            i64 *gidx = (i64 *)malloc(sizeof(i64) * (size_t)nloc);
            int (*sa)[ORC_MAXD] = malloc(sizeof(int) * ORC_MAXD * (size_t)nloc);
            for (int a = 0; a < nloc; a++) {
                unravel(a, sizes, dim, sa[a]);
                i64 g = 0, st = 1;
                for (int dd = 0; dd < dim; dd++) { g += (i64)(first[dd] + sa[a][dd]) * st; st *= sp->ndof_dir[dd]; }
                gidx[a] = g;
            }
            for (int a = 0; a < nloc; a++)
                for (int b = 0; b < nloc; b++) {
                    double v = coef * jv[sa[a][d]] * jv[sa[b][d]];
                    for (int t = 0; t < dim; t++) {
                        if (t == d) continue;
                        int nl = sp->nsh_dir[t];
                        v *= mass[t][((size_t)s2[t] * nl + sa[a][t]) * nl + sa[b][t]];
                    }
                    if (v == 0.0) continue;
                    for (int c = 0; c < dim; c++) {
                        if (ri) { ri[nt] = c * sp->ndof_sc + gidx[a]; ci[nt] = c * sp->ndof_sc + gidx[b]; vi[nt] = v; }
                        nt++;
                    }
                }
            free(gidx);
            free(sa);
        }
    }
    for (int d = 0; d < dim; d++) { free(mass[d]); free(jlo[d]); free(jn[d]); free(jval[d]); }
    return nt;
}

/* rust/src/immersed.rs:168-222 legacy_stabilization; returns the triplet count and fills
 * rows/cols/vals when they are non-NULL (call once with NULL to size the buffers). */
i64 orc_legacy_stabilization(const orc_space *sp, const int8_t *status, double gamma, i64 *ri, i64 *ci,
                             double *vi) {
    int res[3] = {sp->nel_dir[0], sp->nel_dir[1], sp->nel_dir[2]};
    double h[3];
    for (int d = 0; d < 3; d++) h[d] = sp->lengths[d] / (double)sp->nel_dir[d];
    double alpha = gamma * ((h[0] + h[1] + h[2]) / 3.0);
#define LIN(i, j, k) ((i64)(i) + (i64)res[0] * ((j) + (i64)res[1] * (k)))
#define ACTIVE(e) (status[e] == 1 || status[e] == -1)
#define CUTC(e) (status[e] == -1)
    i64 nt = 0;
    int nsc = sp->nsh_sc;
    int dirs[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int dd = 0; dd < 3; dd++) {
        int di = dirs[dd][0], dj = dirs[dd][1], dk = dirs[dd][2];
        for (int i = 0; i < res[0] - di; i++)
            for (int j = 0; j < res[1] - dj; j++)
                for (int k = 0; k < res[2] - dk; k++) {
                    i64 e1 = LIN(i, j, k), e2 = LIN(i + di, j + dj, k + dk);
                    if (!(ACTIVE(e1) && ACTIVE(e2) && (CUTC(e1) || CUTC(e2)))) continue;
                    for (int c = 0; c < 3; c++) {
                        i64 d1[64], d2[64];
                        for (int a = 0; a < nsc; a++) {
                            d1[a] = sp->connectivity[e1 * sp->nsh + c * nsc + a];
                            d2[a] = sp->connectivity[e2 * sp->nsh + c * nsc + a];
                        }
                        qsort(d1, (size_t)nsc, sizeof(i64), cmp_i64);
                        qsort(d2, (size_t)nsc, sizeof(i64), cmp_i64);
                        int n1 = 0, n2 = 0;
                        for (int a = 0; a < nsc; a++) if (n1 == 0 || d1[a] != d1[n1 - 1]) d1[n1++] = d1[a];
                        for (int a = 0; a < nsc; a++) if (n2 == 0 || d2[a] != d2[n2 - 1]) d2[n2++] = d2[a];
                        i64 common[64], only1[64], only2[64];
                        int nc = 0, no1 = 0, no2 = 0;
                        for (int a = 0; a < n1; a++) {
                            int found = 0;
                            for (int b = 0; b < n2; b++) found |= d2[b] == d1[a];
                            if (found) common[nc++] = d1[a]; else only1[no1++] = d1[a];
                        }
                        for (int b = 0; b < n2; b++) {
                            int found = 0;
                            for (int a = 0; a < n1; a++) found |= d1[a] == d2[b];
                            if (!found) only2[no2++] = d2[b];
                        }
                        if (nc > 0) {
                            double nf = (double)nc;
                            for (int m = 0; m < nc * nc; m++) {
                                int ii = m % nc, jj = m / nc;
                                double s = (alpha / nf) * ((ii == jj ? 1.0 : 0.0) - 1.0 / nf);
                                if (ri) { ri[nt] = common[ii]; ci[nt] = common[ii]; vi[nt] = s; }
                                nt++;
                            }
                        }
                        int np = no1 < no2 ? no1 : no2;
                        for (int k2 = 0; k2 < np; k2++) {
                            i64 p1 = only1[k2], p2 = only2[k2];
                            if (ri) {
                                ri[nt] = p1; ci[nt] = p1; vi[nt] = alpha;
                                ri[nt + 1] = p2; ci[nt + 1] = p2; vi[nt + 1] = alpha;
                                ri[nt + 2] = p1; ci[nt + 2] = p2; vi[nt + 2] = -alpha;
                                ri[nt + 3] = p2; ci[nt + 3] = p1; vi[nt + 3] = -alpha;
                            }
                            nt += 4;
                        }
                    }
                }
    }
#undef LIN
#undef ACTIVE
#undef CUTC
    return nt;
}

/* rust/src/immersed.rs:498-536: bottom clamp (ClampedFace::Bottom) and the default central load
 * on the top face. */
void orc_immersed_bc(const orc_space *sp, uint8_t *free_mask, double *force) {
    const int *nd = sp->ndof_dir;
    memset(free_mask, 1, (size_t)sp->ndof);
    memset(force, 0, sizeof(double) * (size_t)sp->ndof);
    i64 mid_x = (i64)round((double)nd[0] / 2.0), mid_y = (i64)round((double)nd[1] / 2.0);
    i64 nload = 0;
    for (i64 i = 0; i < sp->ndof_sc; i++) {
        i64 i1 = i % nd[0], i2 = (i / nd[0]) % nd[1], i3 = i / ((i64)nd[0] * nd[1]);
        if (i3 == 0) for (int c = 0; c < 3; c++) free_mask[c * sp->ndof_sc + i] = 0;
        if (i3 == nd[2] - 1 && llabs(i1 + 1 - mid_x) <= 2 && llabs(i2 + 1 - mid_y) <= 2) nload++;
    }
    for (i64 i = 0; i < sp->ndof_sc; i++) {
        i64 i1 = i % nd[0], i2 = (i / nd[0]) % nd[1], i3 = i / ((i64)nd[0] * nd[1]);
        if (i3 == nd[2] - 1 && llabs(i1 + 1 - mid_x) <= 2 && llabs(i2 + 1 - mid_y) <= 2)
            force[2 * sp->ndof_sc + i] = -1.0 / (double)nload;
    }
}

/* rust/src/immersed.rs:551-570 solve_immersed_problem on an assembled stiffness */
void orc_solve_immersed(const orc_csr *k, const uint8_t *free_mask, const double *force, double tol,
                        i64 maxit, double *u, i64 *iters, double *res, double *compliance) {
    i64 n = k->nrows;
    double *b = (double *)malloc(sizeof(double) * (size_t)n);
    double *diag = (double *)malloc(sizeof(double) * (size_t)n);
    for (i64 i = 0; i < n; i++) b[i] = free_mask[i] ? force[i] : 0.0;
    orc_csr_diagonal(k, diag);
    for (i64 i = 0; i < n; i++) diag[i] = fmax(diag[i], 1e-6);
    orc_pcg_csr(k, free_mask, 1, b, diag, maxit, tol, u, iters, res);
    for (i64 i = 0; i < n; i++) if (!free_mask[i]) u[i] = 0.0;
    double c = 0.0;
    for (i64 i = 0; i < n; i++) c += force[i] * u[i];
    *compliance = c;
    free(b); free(diag);
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
