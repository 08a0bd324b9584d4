"""TEST INFRASTRUCTURE ONLY: ctypes front end of the C oracle (oracle/icc_oracle.c).

The oracle restates the reference's CPU hot path (rust/src/iga/*, rust/src/sparse.rs,
rust/src/solver.rs, rust/src/topopt_iga.rs, rust/src/immersed.rs) in plain C.  Tests and the
CPU-baseline leg of bench.py use it as the checker; the product package never imports it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
i8p = np.ctypeslib.ndpointer(dtype=np.int8, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        vp = C.c_void_p
        L.orc_gauss_legendre.argtypes = [C.c_int, f64p, f64p]
        L.orc_open_knots.argtypes = [C.c_int, C.c_int, C.c_int, f64p]
        L.orc_open_knots.restype = C.c_int
        L.orc_basis_funs.argtypes = [f64p, C.c_int, C.c_int, C.c_double, f64p, f64p]
        L.orc_basis_funs.restype = C.c_int
        L.orc_space_new.argtypes = [C.c_int, f64p, i32p, C.c_int]
        L.orc_space_new.restype = vp
        L.orc_space_free.argtypes = [vp]
        L.orc_space_info.argtypes = [vp, i64p]
        L.orc_space_connectivity.argtypes = [vp, i64p]
        L.orc_space_greville.argtypes = [vp, f64p]
        L.orc_lame.argtypes = [C.c_double, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_elasticity_element_matrices.argtypes = [vp, C.c_double, C.c_double, f64p, i64p, C.c_int,
                                                      i32p, C.c_int]
        L.orc_elasticity_element_matrices.restype = C.c_int
        L.orc_load_vector.argtypes = [vp, C.c_int, f64p, f64p]
        L.orc_mms_l2_error.argtypes = [vp, f64p]
        L.orc_mms_l2_error.restype = C.c_double
        L.orc_csr_from_triplets.argtypes = [C.c_int64, C.c_int64, C.c_int64, i64p, i64p, f64p]
        L.orc_csr_from_triplets.restype = vp
        L.orc_csr_free.argtypes = [vp]
        L.orc_csr_nnz.argtypes = [vp]
        L.orc_csr_nnz.restype = C.c_int64
        L.orc_csr_matvec.argtypes = [vp, f64p, f64p]
        L.orc_csr_diagonal.argtypes = [vp, f64p]
        L.orc_csr_frobenius.argtypes = [vp]
        L.orc_csr_frobenius.restype = C.c_double
        L.orc_csr_get.argtypes = [vp, C.c_int64, C.c_int64]
        L.orc_csr_get.restype = C.c_double
        L.orc_csr_export.argtypes = [vp, i64p, i64p, f64p]
        L.orc_assemble_pattern.argtypes = [C.c_int64, i64p, C.c_int, C.c_int64, f64p, i64p, vp]
        L.orc_assemble_pattern.restype = vp
        L.orc_assemble_triplets.argtypes = [C.c_int64, i64p, C.c_int, C.c_int64, f64p, i64p, vp]
        L.orc_assemble_triplets.restype = vp
        L.orc_mf_apply.argtypes = [vp, f64p, i64p, vp, vp, C.c_int, f64p, f64p]
        L.orc_mf_diagonal.argtypes = [vp, f64p, i64p, vp, f64p]
        L.orc_pcg_csr.argtypes = [vp, vp, C.c_int, f64p, f64p, C.c_int64, C.c_double, f64p,
                                  C.POINTER(C.c_int64), C.POINTER(C.c_double)]
        L.orc_pcg_mf.argtypes = [vp, f64p, i64p, vp, vp, C.c_int, f64p, f64p, C.c_int64, C.c_double,
                                 f64p, C.POINTER(C.c_int64), C.POINTER(C.c_double)]
        L.orc_solve_state.argtypes = [vp, u8p, f64p, f64p, C.c_double, f64p, C.POINTER(C.c_int64),
                                      C.POINTER(C.c_double)]
        L.orc_topopt_run.argtypes = [i32p, f64p, C.c_int, f64p, f64p, i64p]
        L.orc_topopt_run.restype = C.c_int
        L.orc_topopt_run_loads.argtypes = [i32p, f64p, C.c_int, C.c_int, vp, f64p, f64p, i64p]
        L.orc_topopt_run_loads.restype = C.c_int
        L.orc_element_weights.argtypes = [f64p, i64p, C.c_int64, f64p, i32p, i32p, f64p, i8p]
        L.orc_cylinders_weights.argtypes = [i32p, i32p, C.c_double, f64p, i8p]
        L.orc_legacy_stabilization.argtypes = [vp, i8p, C.c_double, vp, vp, vp]
        L.orc_legacy_stabilization.restype = C.c_int64
        L.orc_ghost_penalty.argtypes = [vp, i8p, C.c_double, C.c_double, vp, vp, vp]
        L.orc_ghost_penalty.restype = C.c_int64
        L.orc_immersed_bc.argtypes = [vp, u8p, f64p]
        L.orc_solve_immersed.argtypes = [vp, u8p, f64p, C.c_double, C.c_int64, f64p,
                                         C.POINTER(C.c_int64), C.POINTER(C.c_double),
                                         C.POINTER(C.c_double)]
        L.orc_num_threads.restype = C.c_int
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def gauss_legendre(n):
    x = np.zeros(n); w = np.zeros(n)
    lib().orc_gauss_legendre(n, x, w)
    return x, w


def open_knots(nel, degree, regularity):
    buf = np.zeros(2 * (degree + 1) + max(nel - 1, 0) * (degree - regularity))
    k = lib().orc_open_knots(nel, degree, regularity, buf)
    return buf[:k]


def basis_funs(knots, degree, x):
    knots = np.ascontiguousarray(knots, dtype=np.float64)
    v = np.zeros(degree + 1); d = np.zeros(degree + 1)
    first = lib().orc_basis_funs(knots, len(knots), degree, float(x), v, d)
    return first, v, d


def lame(young, poisson):
    lam = C.c_double(); mu = C.c_double()
    lib().orc_lame(young, poisson, C.byref(lam), C.byref(mu))
    return lam.value, mu.value


class Space:
    """rust/src/iga/space.rs:107 SpaceBox::new (maximal regularity, p+1 Gauss points)."""

    def __init__(self, bounds, nsub, degree):
        b = np.ascontiguousarray(np.asarray(bounds, dtype=np.float64).reshape(-1))
        self.dim = len(nsub)
        self.degree = degree
        self._h = lib().orc_space_new(self.dim, b, np.asarray(nsub, dtype=np.int32), degree)
        info = np.zeros(11, dtype=np.int64)
        lib().orc_space_info(self._h, info)
        self.nel = int(info[1]); self.ndof = int(info[2]); self.ndof_sc = int(info[3])
        self.nsh = int(info[4])
        self.ndof_dir = [int(v) for v in info[5:5 + self.dim]]
        self.nel_dir = [int(v) for v in info[8:8 + self.dim]]
        self.bounds = np.asarray(bounds, dtype=np.float64).reshape(self.dim, 2)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_space_free(self._h)
            self._h = None

    def connectivity(self):
        c = np.zeros(self.nel * self.nsh, dtype=np.int64)
        lib().orc_space_connectivity(self._h, c)
        return c

    def greville(self):
        g = np.zeros(self.ndof_sc * self.dim)
        lib().orc_space_greville(self._h, g)
        return g.reshape(self.ndof_sc, self.dim)

    def element_matrices(self, lam, mu):
        cap = 512
        types = np.zeros(cap * self.nsh * self.nsh)
        tid = np.zeros(self.nel, dtype=np.int64)
        mx = max(self.nel_dir)
        tdir = np.zeros(self.dim * mx, dtype=np.int32)
        nt = lib().orc_elasticity_element_matrices(self._h, lam, mu, types, tid, cap, tdir, mx)
        assert nt > 0
        return (types[: nt * self.nsh * self.nsh].reshape(nt, self.nsh, self.nsh).copy(), tid,
                [tdir[d * mx: d * mx + self.nel_dir[d]].copy() for d in range(self.dim)])

    def load_vector(self, kind=0, params=(0.0, 0.0)):
        out = np.zeros(self.ndof)
        lib().orc_load_vector(self._h, kind, np.asarray(params, dtype=np.float64), out)
        return out

    def mms_l2_error(self, u):
        return lib().orc_mms_l2_error(self._h, np.ascontiguousarray(u, dtype=np.float64))


class Csr:
    """rust/src/sparse.rs CsrMatrix."""

    def __init__(self, handle, n):
        self._h = handle
        self.n = n

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_csr_free(self._h)
            self._h = None

    @classmethod
    def from_triplets(cls, n, rows, cols, vals):
        rows = np.ascontiguousarray(rows, dtype=np.int64)
        cols = np.ascontiguousarray(cols, dtype=np.int64)
        vals = np.ascontiguousarray(vals, dtype=np.float64)
        return cls(lib().orc_csr_from_triplets(n, n, len(vals), rows, cols, vals), n)

    @classmethod
    def assemble(cls, sp, types, type_id, scale=None, pattern=True):
        t = np.ascontiguousarray(types, dtype=np.float64).reshape(-1)
        tid = np.ascontiguousarray(type_id, dtype=np.int64)
        s = None if scale is None else np.ascontiguousarray(scale, dtype=np.float64)
        f = lib().orc_assemble_pattern if pattern else lib().orc_assemble_triplets
        return cls(f(sp.ndof, sp.connectivity(), sp.nsh, sp.nel, t, tid, _ptr(s)), sp.ndof)

    def nnz(self):
        return lib().orc_csr_nnz(self._h)

    def matvec(self, x):
        y = np.zeros(self.n)
        lib().orc_csr_matvec(self._h, np.ascontiguousarray(x, dtype=np.float64), y)
        return y

    def diagonal(self):
        d = np.zeros(self.n)
        lib().orc_csr_diagonal(self._h, d)
        return d

    def frobenius(self):
        return lib().orc_csr_frobenius(self._h)

    def get(self, r, c):
        return lib().orc_csr_get(self._h, r, c)

    def export(self):
        nnz = self.nnz()
        ip = np.zeros(self.n + 1, dtype=np.int64); ix = np.zeros(nnz, dtype=np.int64)
        d = np.zeros(nnz)
        lib().orc_csr_export(self._h, ip, ix, d)
        return ip, ix, d

    def pcg(self, b, diag, max_iter, tol, free_mask=None, mask_mode=0):
        x = np.zeros(self.n)
        it = C.c_int64(); res = C.c_double()
        fm = None if free_mask is None else np.ascontiguousarray(free_mask, dtype=np.uint8)
        lib().orc_pcg_csr(self._h, _ptr(fm), mask_mode, np.ascontiguousarray(b, dtype=np.float64),
                          np.ascontiguousarray(diag, dtype=np.float64), max_iter, tol, x,
                          C.byref(it), C.byref(res))
        return x, it.value, res.value

    def solve_state(self, free_mask, force, u0, pcg_tol):
        u = np.zeros(self.n)
        it = C.c_int64(); res = C.c_double()
        lib().orc_solve_state(self._h, np.ascontiguousarray(free_mask, dtype=np.uint8),
                              np.ascontiguousarray(force, dtype=np.float64),
                              np.ascontiguousarray(u0, dtype=np.float64), pcg_tol, u,
                              C.byref(it), C.byref(res))
        return u, it.value, res.value


def mf_apply(sp, types, type_id, scale, x, free_mask=None, mask_mode=0):
    t = np.ascontiguousarray(types, dtype=np.float64).reshape(-1)
    y = np.zeros(sp.ndof)
    s = None if scale is None else np.ascontiguousarray(scale, dtype=np.float64)
    fm = None if free_mask is None else np.ascontiguousarray(free_mask, dtype=np.uint8)
    lib().orc_mf_apply(sp._h, t, np.ascontiguousarray(type_id, dtype=np.int64), _ptr(s), _ptr(fm),
                       mask_mode, np.ascontiguousarray(x, dtype=np.float64), y)
    return y


def mf_diagonal(sp, types, type_id, scale):
    t = np.ascontiguousarray(types, dtype=np.float64).reshape(-1)
    d = np.zeros(sp.ndof)
    s = None if scale is None else np.ascontiguousarray(scale, dtype=np.float64)
    lib().orc_mf_diagonal(sp._h, t, np.ascontiguousarray(type_id, dtype=np.int64), _ptr(s), d)
    return d


def pcg_mf(sp, types, type_id, scale, b, diag, max_iter, tol, free_mask=None, mask_mode=0):
    t = np.ascontiguousarray(types, dtype=np.float64).reshape(-1)
    x = np.zeros(sp.ndof)
    it = C.c_int64(); res = C.c_double()
    s = None if scale is None else np.ascontiguousarray(scale, dtype=np.float64)
    fm = None if free_mask is None else np.ascontiguousarray(free_mask, dtype=np.uint8)
    lib().orc_pcg_mf(sp._h, t, np.ascontiguousarray(type_id, dtype=np.int64), _ptr(s), _ptr(fm),
                     mask_mode, np.ascontiguousarray(b, dtype=np.float64),
                     np.ascontiguousarray(diag, dtype=np.float64), max_iter, tol, x,
                     C.byref(it), C.byref(res))
    return x, it.value, res.value


def topopt_run(nel, volfrac, penal, rmin, max_iter, pcg_tol, size=(1.2, 0.6, 0.3), young=1.0,
               poisson=0.3, emin=1e-3, move_limit=0.2, loads=None):
    """rust/src/topopt_iga.rs:187-234 CantileverTopOpt::run with CantileverTopOptConfig.  loads
    (nload x ndof) replaces the single tip load by load cases: compliance |sum_k F_k'u_k| and the
    element energies summed over the cases, each case warm-started from its own previous state."""
    cfg = np.array([size[0], size[1], size[2], volfrac, penal, rmin, young, poisson, emin,
                    move_limit, pcg_tol])
    comp = np.zeros(max_iter)
    ne = int(np.prod(nel))
    dens = np.zeros(ne)
    its = np.zeros(max_iter, dtype=np.int64)
    if loads is None:
        n = lib().orc_topopt_run(np.asarray(nel, dtype=np.int32), cfg, max_iter, comp, dens, its)
    else:
        f = np.ascontiguousarray(np.atleast_2d(loads), dtype=np.float64)
        n = lib().orc_topopt_run_loads(np.asarray(nel, dtype=np.int32), cfg, max_iter, f.shape[0],
                                       f.ctypes.data_as(C.c_void_p), comp, dens, its)
    return comp[:n], dens, its[:n]


def element_weights(verts, tris, bounds, res, sub):
    verts = np.ascontiguousarray(verts, dtype=np.float64).reshape(-1)
    tris = np.ascontiguousarray(tris, dtype=np.int64).reshape(-1)
    ncell = int(np.prod(res))
    w = np.zeros(ncell); st = np.zeros(ncell, dtype=np.int8)
    lib().orc_element_weights(verts, tris, len(tris) // 3,
                              np.ascontiguousarray(bounds, dtype=np.float64).reshape(-1),
                              np.asarray(res, dtype=np.int32), np.asarray(sub, dtype=np.int32), w, st)
    return w, st


def cylinders_weights(res, sub, radius):
    ncell = int(np.prod(res))
    w = np.zeros(ncell); st = np.zeros(ncell, dtype=np.int8)
    lib().orc_cylinders_weights(np.asarray(res, dtype=np.int32), np.asarray(sub, dtype=np.int32),
                                radius, w, st)
    return w, st


def legacy_stabilization(sp, status, gamma):
    st = np.ascontiguousarray(status, dtype=np.int8)
    n = lib().orc_legacy_stabilization(sp._h, st, gamma, None, None, None)
    r = np.zeros(n, dtype=np.int64); c = np.zeros(n, dtype=np.int64); v = np.zeros(n)
    lib().orc_legacy_stabilization(sp._h, st, gamma, _ptr(r), _ptr(c), _ptr(v))
    return r, c, v


def ghost_penalty(sp, status, gamma, young):
    """rust/src/immersed.rs:224-370 ghost_penalty as triplets (rows, cols, vals)."""
    st = np.ascontiguousarray(status, dtype=np.int8)
    n = lib().orc_ghost_penalty(sp._h, st, gamma, young, None, None, None)
    r = np.zeros(n, dtype=np.int64); c = np.zeros(n, dtype=np.int64); v = np.zeros(n)
    lib().orc_ghost_penalty(sp._h, st, gamma, young, _ptr(r), _ptr(c), _ptr(v))
    return r, c, v


def immersed_bc(sp):
    fm = np.zeros(sp.ndof, dtype=np.uint8); f = np.zeros(sp.ndof)
    lib().orc_immersed_bc(sp._h, fm, f)
    return fm, f


def solve_immersed(k, free_mask, force, tol, maxit):
    u = np.zeros(k.n)
    it = C.c_int64(); res = C.c_double(); comp = C.c_double()
    lib().orc_solve_immersed(k._h, np.ascontiguousarray(free_mask, dtype=np.uint8),
                             np.ascontiguousarray(force, dtype=np.float64), tol, maxit, u,
                             C.byref(it), C.byref(res), C.byref(comp))
    return u, it.value, res.value, comp.value


def num_threads():
    return lib().orc_num_threads()
