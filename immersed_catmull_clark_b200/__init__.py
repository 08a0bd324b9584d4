"""B200 matrix-free p = 2 B-spline elasticity operator and Jacobi-PCG, behind a C ABI.

Python front end (ctypes) of libicc.so, shaped like the reference's Rust API so callers and
tests read the same:

* ``SpaceBox(bounds, nsub, 2)``                      rust/src/iga/space.rs:107 SpaceBox::new
* ``lame(young, poisson)``                           rust/src/iga/elasticity.rs:173
* ``elasticity_element_matrices(sp, lam, mu)``       rust/src/iga/elasticity.rs:30
* ``MatrixFreeOperator(sp, em, scale, ...)``         replaces AssemblyPattern::assemble +
  CsrMatrix::{matvec, diagonal} (rust/src/sparse.rs:160, :60, :70) with the device operator
* ``PcgSolver(max_iter, tol).solve(n, b, diag, op)`` rust/src/solver.rs:9-76; the closure
  argument is the operator handle (its mask mode selects the reference's closure)

All compute runs in libicc's CUDA kernels.  There is no CPU fallback: without the built
library or a B200 the calls raise ``IccError``.
"""
import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libicc.so")

ICC_OK = 0
ICC_NOT_CONVERGED = 1
ICC_BREAKDOWN = 2
ICC_BAD_ARG = -1
ICC_CUDA_ERROR = -2
ICC_TIMEOUT = -3
ICC_NO_DEVICE = -4
ICC_OUT_OF_MEMORY = -5
ICC_NAN = -6

MASK_NONE, MASK_ZERO, MASK_IDENTITY = 0, 1, 2
FP64, MIXED = 0, 1

# every symbol include/icc.h declares
EXPORTED = [
    "icc_last_error", "icc_space_create", "icc_space_destroy", "icc_space_dims", "icc_space_connectivity",
    "icc_lame", "icc_element_matrices", "icc_space_window", "icc_op_create", "icc_op_create_lame", "icc_op_destroy",
    "icc_op_update_scale", "icc_op_update_mask", "icc_op_apply", "icc_op_apply_dev", "icc_op_apply_f32",
    "icc_op_apply_f32_dev", "icc_op_diagonal",
    "icc_op_stream", "icc_pcg_solve", "icc_pcg_solve_dev", "icc_op_last_solve_info", "icc_op_profile_apply",
    "icc_op_profile_apply_f32", "icc_solve_state", "icc_op_element_energies", "icc_topopt_create",
    "icc_topopt_destroy", "icc_topopt_run", "icc_cylinder_weights", "icc_pcg_solve_batched",
    "icc_topopt_set_loads",
    "icc_apply_f64_noalloc", "icc_op_set_wait_limit", "icc_op_set_extra_triplets", "icc_ghost_penalty",
    "icc_legacy_stabilization",
]


class IccError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"icc error {code}: {msg}")
        self.code = code


class SolveOpts(C.Structure):
    _fields_ = [("precision", C.c_int32), ("check_every", C.c_int32), ("inner_tol", C.c_double),
                ("max_outer", C.c_int32), ("reserved", C.c_int32)]


class SolveInfo(C.Structure):
    _fields_ = [("iterations", C.c_int64), ("outer_iterations", C.c_int64), ("rel_res", C.c_double),
                ("device_ms", C.c_double), ("fp64_applies", C.c_int64), ("mixed_applies", C.c_int64),
                ("kernel_launches", C.c_int64)]


class TopOptCfg(C.Structure):
    _fields_ = [("size", C.c_double * 3), ("volfrac", C.c_double), ("penal", C.c_double), ("rmin", C.c_double),
                ("young", C.c_double), ("poisson", C.c_double), ("emin", C.c_double), ("move_limit", C.c_double),
                ("pcg_tol", C.c_double), ("precision", C.c_int32), ("reserved", C.c_int32)]


_lib = None
f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")


def lib():
    """Load libicc.so (built in-tree by __graft_entry__.build or immersed_catmull_clark_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise IccError(ICC_NO_DEVICE, f"{LIB_PATH} is not built (run immersed_catmull_clark_b200.build)")
    L = C.CDLL(LIB_PATH)
    vp, i32, i64, dbl = C.c_void_p, C.c_int32, C.c_int64, C.c_double
    L.icc_last_error.restype = C.c_char_p
    L.icc_space_create.argtypes = [f64p, i64p, i32, C.POINTER(vp)]
    L.icc_space_destroy.argtypes = [vp]
    L.icc_space_window.argtypes = [vp, i64p, i64p, C.POINTER(vp)]
    L.icc_space_dims.argtypes = [vp, C.POINTER(i64), C.POINTER(i64), i64p, i64p]
    L.icc_space_connectivity.argtypes = [vp, i64p]
    L.icc_lame.argtypes = [dbl, dbl, C.POINTER(dbl), C.POINTER(dbl)]
    L.icc_lame.restype = None
    L.icc_element_matrices.argtypes = [vp, dbl, dbl, vp, i32, vp, C.POINTER(i32)]
    L.icc_op_create.argtypes = [vp, f64p, i32, i32p, vp, vp, i32, C.POINTER(vp)]
    L.icc_op_create_lame.argtypes = [vp, dbl, dbl, vp, vp, i32, C.POINTER(vp)]
    L.icc_op_destroy.argtypes = [vp]
    L.icc_op_destroy.restype = None
    L.icc_op_update_scale.argtypes = [vp, vp]
    L.icc_op_update_mask.argtypes = [vp, vp, i32]
    L.icc_op_apply.argtypes = [vp, f64p, f64p, i64]
    L.icc_op_apply_dev.argtypes = [vp, vp, vp, i64]
    L.icc_op_apply_f32.argtypes = [vp, f32p, f32p, i64]
    L.icc_op_apply_f32_dev.argtypes = [vp, vp, vp, i64]
    L.icc_op_diagonal.argtypes = [vp, f64p, i64]
    L.icc_op_stream.argtypes = [vp]
    L.icc_op_stream.restype = vp
    L.icc_pcg_solve.argtypes = [vp, f64p, vp, i64, dbl, i64, C.POINTER(SolveOpts), f64p,
                                C.POINTER(i64), C.POINTER(dbl)]
    L.icc_pcg_solve_dev.argtypes = [vp, vp, vp, i64, dbl, i64, C.POINTER(SolveOpts), vp,
                                    C.POINTER(i64), C.POINTER(dbl)]
    L.icc_op_last_solve_info.argtypes = [vp, C.POINTER(SolveInfo)]
    L.icc_op_profile_apply.argtypes = [vp, vp, vp, i32, C.POINTER(dbl), C.POINTER(dbl)]
    L.icc_op_profile_apply_f32.argtypes = [vp, vp, vp, i32, C.POINTER(dbl), C.POINTER(dbl)]
    L.icc_apply_f64_noalloc.argtypes = [i64p, vp, i32, vp, vp, vp, vp, vp]
    L.icc_op_set_wait_limit.argtypes = [vp, i64]
    L.icc_op_set_extra_triplets.argtypes = [vp, i64, vp, vp, vp]
    L.icc_ghost_penalty.argtypes = [vp, vp, dbl, dbl, vp, vp, vp, i64, C.POINTER(i64)]
    L.icc_legacy_stabilization.argtypes = [vp, vp, dbl, vp, vp, vp, i64, C.POINTER(i64)]
    L.icc_solve_state.argtypes = [vp, f64p, f64p, i64, dbl, C.POINTER(SolveOpts), f64p, C.POINTER(i64),
                                  C.POINTER(dbl)]
    L.icc_op_element_energies.argtypes = [vp, f64p, i64, f64p, i64]
    L.icc_topopt_create.argtypes = [i64p, C.POINTER(TopOptCfg), C.POINTER(vp)]
    L.icc_topopt_destroy.argtypes = [vp]
    L.icc_topopt_destroy.restype = None
    L.icc_topopt_run.argtypes = [vp, i32, vp, vp, vp, vp, C.POINTER(i32)]
    L.icc_topopt_set_loads.argtypes = [vp, i32, f64p]
    L.icc_cylinder_weights.argtypes = [i64p, i32p, dbl, f64p, vp]
    L.icc_pcg_solve_batched.argtypes = [i32, vp, vp, vp, dbl, i64, C.POINTER(SolveOpts), vp, vp, vp, vp]
    _lib = L
    return L


def _check(rc, allow=(ICC_OK,)):
    if rc in allow:
        return rc
    raise IccError(rc, lib().icc_last_error().decode())


def _vp(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def lame(young, poisson):
    lam, mu = C.c_double(), C.c_double()
    lib().icc_lame(young, poisson, C.byref(lam), C.byref(mu))
    return lam.value, mu.value


class SpaceBox:
    """p = 2 tensor-product B-spline space on a 3-D box (rust/src/iga/space.rs:107)."""

    def __init__(self, bounds, nsub, degree=2, _handle=None):
        if _handle is None:
            b = np.ascontiguousarray(np.asarray(bounds, dtype=np.float64).reshape(-1))
            ns = np.ascontiguousarray(np.asarray(nsub, dtype=np.int64))
            h = C.c_void_p()
            _check(lib().icc_space_create(b, ns, int(degree), C.byref(h)))
        else:
            h = _handle
        self._h = h
        ndof, nel = C.c_int64(), C.c_int64()
        nd = np.zeros(3, dtype=np.int64); ne = np.zeros(3, dtype=np.int64)
        _check(lib().icc_space_dims(h, C.byref(ndof), C.byref(nel), nd, ne))
        self.ndof, self.nel = ndof.value, nel.value
        self.ndof_dir = [int(v) for v in nd]
        self.nel_dir = [int(v) for v in ne]
        self.ndof_sc = self.ndof // 3
        self.nsh = 81
        self.bounds = np.asarray(bounds, dtype=np.float64).reshape(3, 2)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.icc_space_destroy(h)
            self._h = None

    def window(self, e0, e1):
        """The sub-grid of elements [e0[d], e1[d]) with this space's B-splines, numbered locally
        (icc_space_window): the local space of a slab in the multi-rank solve."""
        a = np.ascontiguousarray(np.asarray(e0, dtype=np.int64))
        b = np.ascontiguousarray(np.asarray(e1, dtype=np.int64))
        h = C.c_void_p()
        _check(lib().icc_space_window(self._h, a, b, C.byref(h)))
        nel = self.nel_dir
        h_el = [(self.bounds[d, 1] - self.bounds[d, 0]) / nel[d] for d in range(3)]
        bounds = np.array([[self.bounds[d, 0] + a[d] * h_el[d], self.bounds[d, 0] + b[d] * h_el[d]] for d in range(3)])
        return SpaceBox(bounds, b - a, 2, _handle=h)

    def connectivity(self):
        c = np.zeros(self.nel * 81, dtype=np.int64)
        _check(lib().icc_space_connectivity(self._h, c))
        return c


@dataclass
class ElementMatrices:
    """rust/src/iga/elasticity.rs:14-26: distinct 81x81 matrices and the type of every element."""
    types: np.ndarray     # [ntypes, 81, 81] float64
    type_id: np.ndarray   # [nel] int32


def elasticity_element_matrices(sp, lam, mu):
    nt = C.c_int32()
    _check(lib().icc_element_matrices(sp._h, lam, mu, None, 0, None, C.byref(nt)))
    types = np.zeros((nt.value, 81, 81))
    tid = np.zeros(sp.nel, dtype=np.int32)
    _check(lib().icc_element_matrices(sp._h, lam, mu, _vp(types), nt.value, _vp(tid), C.byref(nt)))
    return ElementMatrices(types, tid)


class MatrixFreeOperator:
    """Device operator y = A x, A = the masked sum_e s_e K_type(e) (replaces the assembled CSR)."""

    def __init__(self, sp, em, scale=None, free_mask=None, mask_mode=MASK_NONE):
        self.sp = sp
        self.n = sp.ndof
        h = C.c_void_p()
        s = None if scale is None else np.ascontiguousarray(scale, dtype=np.float64)
        fm = None if free_mask is None else np.ascontiguousarray(free_mask, dtype=np.uint8)
        if isinstance(em, ElementMatrices):
            types = np.ascontiguousarray(em.types, dtype=np.float64).reshape(-1)
            tid = np.ascontiguousarray(em.type_id, dtype=np.int32)
            rc = lib().icc_op_create(sp._h, types, len(em.types), tid, _vp(s), _vp(fm), mask_mode, C.byref(h))
        else:
            lam, mu = em
            rc = lib().icc_op_create_lame(sp._h, lam, mu, _vp(s), _vp(fm), mask_mode, C.byref(h))
        _check(rc)
        self._h = h

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.icc_op_destroy(h)
        self._h = None

    def __del__(self):
        self.close()

    @property
    def stream(self):
        return lib().icc_op_stream(self._h)

    def update_scale(self, scale):
        s = None if scale is None else np.ascontiguousarray(scale, dtype=np.float64)
        _check(lib().icc_op_update_scale(self._h, _vp(s)))

    def set_extra_triplets(self, rows, cols, vals):
        """Adds the sparse term S (triplets, duplicates summed) to the operator: y = mask rule of
        (K + S)(m .* x), the stabilised closures of rust/src/topopt_immersed.rs:174-183 and
        rust/src/immersed.rs:558-566.  Empty triplets remove it."""
        r = np.ascontiguousarray(rows, dtype=np.int64)
        c = np.ascontiguousarray(cols, dtype=np.int64)
        v = np.ascontiguousarray(vals, dtype=np.float64)
        if not (len(r) == len(c) == len(v)):
            raise ValueError("rows, cols and vals must have the same length")
        _check(lib().icc_op_set_extra_triplets(self._h, len(v), _vp(r), _vp(c), _vp(v)))

    def update_mask(self, free_mask, mask_mode):
        fm = None if free_mask is None else np.ascontiguousarray(free_mask, dtype=np.uint8)
        _check(lib().icc_op_update_mask(self._h, _vp(fm), mask_mode))

    def matvec(self, x):
        y = np.zeros(self.n)
        _check(lib().icc_op_apply(self._h, np.ascontiguousarray(x, dtype=np.float64), y, self.n))
        return y

    def matvec_f32(self, x):
        """FP32 tensor-core apply (the mixed form's inner operator)."""
        y = np.zeros(self.n, dtype=np.float32)
        _check(lib().icc_op_apply_f32(self._h, np.ascontiguousarray(x, dtype=np.float32), y, self.n))
        return y

    def matvec_f32_dev(self, x_ptr, y_ptr):
        _check(lib().icc_op_apply_f32_dev(self._h, C.c_void_p(x_ptr), C.c_void_p(y_ptr), self.n))

    def matvec_dev(self, x_ptr, y_ptr):
        """Device pointers (e.g. torch tensor .data_ptr()); enqueued on the operator's stream."""
        _check(lib().icc_op_apply_dev(self._h, C.c_void_p(x_ptr), C.c_void_p(y_ptr), self.n))

    def diagonal(self):
        d = np.zeros(self.n)
        _check(lib().icc_op_diagonal(self._h, d, self.n))
        return d

    def profile_apply(self, x_ptr, y_ptr, reps=20):
        """Mean device ms of (brick contraction kernel, node-sum kernel) over reps FP64 applies."""
        a, g = C.c_double(), C.c_double()
        _check(lib().icc_op_profile_apply(self._h, C.c_void_p(x_ptr), C.c_void_p(y_ptr), reps, C.byref(a),
                                          C.byref(g)))
        return a.value, g.value

    def profile_apply_f32(self, x_ptr, y_ptr, reps=20):
        """Mean device ms of (tensor-core brick kernel, node-sum kernel) over reps FP32 applies."""
        a, g = C.c_double(), C.c_double()
        _check(lib().icc_op_profile_apply_f32(self._h, C.c_void_p(x_ptr), C.c_void_p(y_ptr), reps, C.byref(a),
                                              C.byref(g)))
        return a.value, g.value

    def element_energies(self, u):
        """u_e^T K_type(e) u_e per element (rust/src/topopt_iga.rs:165-184)."""
        ee = np.zeros(self.sp.nel)
        _check(lib().icc_op_element_energies(self._h, np.ascontiguousarray(u, dtype=np.float64), self.n, ee,
                                             self.sp.nel))
        return ee

    def set_wait_limit(self, grid_polls):
        """Polls of a grid barrier in the mixed solve's fused vector step before ICC_TIMEOUT."""
        _check(lib().icc_op_set_wait_limit(self._h, int(grid_polls)))

    def last_solve_info(self):
        info = SolveInfo()
        _check(lib().icc_op_last_solve_info(self._h, C.byref(info)))
        return info


class PcgSolver:
    """rust/src/solver.rs:9-76 PcgSolver on the device operator.

    precision FP64 reproduces the reference loop in FP64; MIXED runs FP64 iterative refinement
    around a tensor-core FP32 inner PCG.  ``solve`` returns (x, iters, rel_res) like the
    reference; ``status`` holds the C status (ICC_OK, ICC_NOT_CONVERGED, ICC_BREAKDOWN).
    """

    def __init__(self, max_iter, tol, precision=FP64, check_every=32, inner_tol=0.0, max_outer=0):
        self.max_iter, self.tol = int(max_iter), float(tol)
        self.opts = SolveOpts(precision, check_every, inner_tol, max_outer, 0)
        self.status = None

    def solve(self, n, b, diag_a, op):
        x = np.zeros(n)
        it, res = C.c_int64(), C.c_double()
        d = None if diag_a is None else np.ascontiguousarray(diag_a, dtype=np.float64)
        rc = lib().icc_pcg_solve(op._h, np.ascontiguousarray(b, dtype=np.float64), _vp(d), n, self.tol,
                                 self.max_iter, C.byref(self.opts), x, C.byref(it), C.byref(res))
        self.status = _check(rc, (ICC_OK, ICC_NOT_CONVERGED, ICC_BREAKDOWN))
        return x, it.value, res.value

    def solve_host_ptr(self, n, b, diag_a, x, op):
        """Like solve() but writes into the caller's host array x (e.g. pinned memory)."""
        it, res = C.c_int64(), C.c_double()
        d = None if diag_a is None else np.ascontiguousarray(diag_a, dtype=np.float64)
        rc = lib().icc_pcg_solve(op._h, b, _vp(d), n, self.tol, self.max_iter, C.byref(self.opts), x,
                                 C.byref(it), C.byref(res))
        self.status = _check(rc, (ICC_OK, ICC_NOT_CONVERGED, ICC_BREAKDOWN))
        return it.value, res.value

    def solve_dev(self, n, b_ptr, diag_ptr, x_ptr, op):
        it, res = C.c_int64(), C.c_double()
        rc = lib().icc_pcg_solve_dev(op._h, C.c_void_p(b_ptr), C.c_void_p(diag_ptr) if diag_ptr else None, n,
                                     self.tol, self.max_iter, C.byref(self.opts), C.c_void_p(x_ptr),
                                     C.byref(it), C.byref(res))
        self.status = _check(rc, (ICC_OK, ICC_NOT_CONVERGED, ICC_BREAKDOWN))
        return it.value, res.value


def apply_f64_noalloc(nel_dir, ke_ptr, ntypes, type_id_ptr, scale_ptr, x_ptr, y_ptr, stream=0):
    """icc_apply_f64_noalloc on caller-owned device buffers (raw pointers); allocates nothing."""
    ne = np.ascontiguousarray(np.asarray(nel_dir, dtype=np.int64))
    _check(lib().icc_apply_f64_noalloc(ne, C.c_void_p(ke_ptr), int(ntypes), C.c_void_p(type_id_ptr),
                                       C.c_void_p(scale_ptr) if scale_ptr else None, C.c_void_p(x_ptr),
                                       C.c_void_p(y_ptr), C.c_void_p(stream) if stream else None))


def solve_state(op, force, u0, pcg_tol, precision=FP64):
    """Warm-started masked state solve (rust/src/topopt_iga.rs:137-162) on the device operator.
    Returns (u, iterations, relative residual) as the reference does."""
    u = np.zeros(op.n)
    it, res = C.c_int64(), C.c_double()
    opts = SolveOpts(precision, 32, 0.0, 0, 0)
    rc = lib().icc_solve_state(op._h, np.ascontiguousarray(force, dtype=np.float64),
                               np.ascontiguousarray(u0, dtype=np.float64), op.n, pcg_tol, C.byref(opts), u,
                               C.byref(it), C.byref(res))
    _check(rc, allow=(ICC_OK, ICC_NOT_CONVERGED, ICC_BREAKDOWN))
    return u, it.value, res.value


@dataclass
class TopOptHistory:
    """rust/src/topopt_iga.rs:53-58."""
    compliance: np.ndarray
    change: np.ndarray
    pcg_iterations: np.ndarray
    density: np.ndarray


class CantileverTopOpt:
    """SIMP cantilever loop on the device (rust/src/topopt_iga.rs:60-234, CantileverTopOptConfig
    defaults)."""

    def __init__(self, nel, size=(1.2, 0.6, 0.3), volfrac=0.3, penal=3.0, rmin=1.5, young=1.0, poisson=0.3,
                 emin=1e-3, move_limit=0.2, pcg_tol=1e-10, precision=FP64):
        cfg = TopOptCfg((C.c_double * 3)(*size), volfrac, penal, rmin, young, poisson, emin, move_limit, pcg_tol,
                        precision, 0)
        h = C.c_void_p()
        _check(lib().icc_topopt_create(np.ascontiguousarray(nel, dtype=np.int64), C.byref(cfg), C.byref(h)))
        self._h = h
        self.nel = int(np.prod(nel))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.icc_topopt_destroy(h)
            self._h = None

    def set_loads(self, forces):
        """Load cases (rows of forces, each of ndof).  In the mixed precision their state solves run as
        one batch (one tensor-core apply over all cases per PCG iteration); in FP64 one after another."""
        f = np.ascontiguousarray(np.atleast_2d(forces), dtype=np.float64)
        _check(lib().icc_topopt_set_loads(self._h, f.shape[0], f.reshape(-1)))

    def run(self, max_iter=40):
        comp, chg = np.zeros(max_iter), np.zeros(max_iter)
        its, dens = np.zeros(max_iter, dtype=np.int64), np.zeros(self.nel)
        done = C.c_int32()
        _check(lib().icc_topopt_run(self._h, max_iter, _vp(comp), _vp(chg), _vp(its), _vp(dens), C.byref(done)))
        k = done.value
        return TopOptHistory(comp[:k], chg[:k], its[:k], dens)


def _triplets(fn, *args):
    cnt = C.c_int64()
    _check(fn(*args, None, None, None, 0, C.byref(cnt)))
    n = cnt.value
    r = np.zeros(n, dtype=np.int64)
    c = np.zeros(n, dtype=np.int64)
    v = np.zeros(n)
    _check(fn(*args, _vp(r), _vp(c), _vp(v), n, C.byref(cnt)))
    return r, c, v


def ghost_penalty(sp, status, gamma, young):
    """Face ghost penalty of the immersed solve (rust/src/immersed.rs:224-370) as triplets."""
    st = np.ascontiguousarray(status, dtype=np.int8)
    return _triplets(lib().icc_ghost_penalty, sp._h, _vp(st), float(gamma), float(young))


def legacy_stabilization(sp, status, gamma):
    """The reference's legacy cut-cell springs (rust/src/immersed.rs:156-222) as triplets."""
    st = np.ascontiguousarray(status, dtype=np.int8)
    return _triplets(lib().icc_legacy_stabilization, sp._h, _vp(st), float(gamma))


def cylinder_weights(res, sub, radius):
    """Volume fraction and status (1 inside, 0 outside, -1 cut) of every cell of the unit cube minus
    three orthogonal through-cylinders (rust/src/immersed.rs:88-155 rule), computed on the device."""
    ncell = int(np.prod(res))
    w = np.zeros(ncell)
    st = np.zeros(ncell, dtype=np.int8)
    _check(lib().icc_cylinder_weights(np.ascontiguousarray(res, dtype=np.int64),
                                      np.ascontiguousarray(sub, dtype=np.int32), float(radius), w,
                                      st.ctypes.data_as(C.c_void_p)))
    return w, st


def solve_batched(ops, bs, diags=None, tol=1e-8, max_iter=None, precision=FP64, check_every=32):
    """Independent solves ops[i] x_i = bs[i], all in flight together (icc_pcg_solve_batched).
    Returns (xs, iterations, rel_res, status) per instance."""
    k = len(ops)
    xs = [np.zeros(op.n) for op in ops]
    bs = [np.ascontiguousarray(b, dtype=np.float64) for b in bs]
    ds = None if diags is None else [np.ascontiguousarray(d, dtype=np.float64) for d in diags]
    hv = (C.c_void_p * k)(*[op._h.value for op in ops])
    bv = (C.c_void_p * k)(*[b.ctypes.data for b in bs])
    xv = (C.c_void_p * k)(*[x.ctypes.data for x in xs])
    dv = None if ds is None else (C.c_void_p * k)(*[d.ctypes.data for d in ds])
    its = np.zeros(k, dtype=np.int64)
    res = np.zeros(k)
    st = np.zeros(k, dtype=np.int32)
    mi = max_iter if max_iter is not None else 20 * max(op.n for op in ops)
    opts = SolveOpts(precision, check_every, 0.0, 0, 0)
    _check(lib().icc_pcg_solve_batched(k, hv, bv, dv, tol, mi, C.byref(opts), xv, its.ctypes.data,
                                       res.ctypes.data, st.ctypes.data))
    return xs, its, res, st
