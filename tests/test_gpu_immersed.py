"""Immersed fictitious-domain case on the device: the volume-fraction rule of
rust/src/immersed.rs:88-155 for the cube-minus-cylinders solid (bitwise against the oracle's CPU
evaluation), and the scaled, masked solve (FP64 and mixed) against the oracle's CSR PCG."""
import numpy as np
import pytest

import immersed_catmull_clark_b200 as icc
from immersed_catmull_clark_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("res,sub", [((24, 24, 24), (8, 8, 8)), ((17, 13, 11), (4, 3, 5)), ((1, 2, 3), (2, 2, 2))])
def test_cylinder_weights_match_oracle_bitwise(res, sub):
    w, st = icc.cylinder_weights(res, sub, 0.25)
    wo, sto = O.cylinders_weights(res, sub, 0.25)
    assert np.array_equal(st, sto)
    assert np.array_equal(w, wo)


def test_cylinder_volume():
    # solid volume of the cube minus three r = 0.25 cylinders: 1 - [3 pi r^2 - 16 r^3 + 8 (2 - sqrt 2) r^3]
    w, _ = icc.cylinder_weights((64, 64, 64), (8, 8, 8), 0.25)
    r = 0.25
    exact = 1.0 - (3 * np.pi * r * r - 16 * r ** 3 + 8 * (2 - np.sqrt(2)) * r ** 3)
    assert abs(w.mean() - exact) < 2e-3


def test_immersed_solve_matches_oracle():
    p = W.cylinders(16)
    sp = icc.SpaceBox(p.bounds, p.nel, 2)
    osp = O.Space(p.bounds, p.nel, 2)
    lam, mu = icc.lame(1.0, 0.3)
    em = icc.elasticity_element_matrices(sp, lam, mu)
    k = O.Csr.assemble(osp, em.types, em.type_id.astype(np.int64), p.scale)
    b = W.rhs_masked(p)
    diag = np.maximum(k.diagonal(), 1e-6)       # the immersed clamp (rust/src/immersed.rs:555)
    tol = 1e-8
    xo, ito, reso = k.pcg(b, diag, 20 * sp.ndof, tol, p.free_mask, icc.MASK_ZERO)
    op = icc.MatrixFreeOperator(sp, em, p.scale, p.free_mask, icc.MASK_ZERO)
    x, it, res = icc.PcgSolver(20 * sp.ndof, tol).solve(sp.ndof, b, diag, op)
    assert res < tol and reso < tol
    assert abs(it - ito) <= max(3, 0.02 * ito), (it, ito)
    assert rel(x, xo) < 1e-6
    xm, itm, resm = icc.PcgSolver(20 * sp.ndof, tol, precision=icc.MIXED).solve(sp.ndof, b, diag, op)
    assert resm < tol
    r_true = b - p.free_mask * k.matvec(p.free_mask * xm)
    assert np.linalg.norm(r_true) / np.linalg.norm(b) < 1.5 * tol
    assert rel(xm, xo) < 1e-6
