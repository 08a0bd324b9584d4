"""Many independent solves at once (icc_pcg_solve_batched): uneven cantilever designs, each result
equal to the instance's own sequential solve (the solves are deterministic)."""
import numpy as np
import pytest

import immersed_catmull_clark_b200 as icc
from immersed_catmull_clark_b200 import workloads as W

pytestmark = pytest.mark.gpu


def instances(ks, seed=5):
    out = []
    lam, mu = icc.lame(1.0, 0.3)
    for i, k in enumerate(ks):
        p = W.cantilever((2 * k, k, k), seed=seed + i)
        sp = icc.SpaceBox(p.bounds, p.nel, 2)
        em = icc.elasticity_element_matrices(sp, lam, mu)
        op = icc.MatrixFreeOperator(sp, em, p.scale, p.free_mask, icc.MASK_ZERO)
        out.append((p, sp, op, W.rhs_masked(p)))
    return out


@pytest.mark.parametrize("precision", [icc.FP64, icc.MIXED])
def test_batched_equals_sequential(precision):
    ks = [4, 9, 6, 12, 5, 8]
    inst = instances(ks)
    ops = [o for _, _, o, _ in inst]
    bs = [b for _, _, _, b in inst]
    tol = 1e-8
    xs, its, res, st = icc.solve_batched(ops, bs, tol=tol, precision=precision)
    assert np.all(st == icc.ICC_OK)
    for (p, sp, op, b), x, it, r in zip(inst, xs, its, res):
        s = icc.PcgSolver(20 * sp.ndof, tol, precision=precision)
        xr, itr, rr = s.solve(sp.ndof, b, None, op)
        assert it == itr and r == rr
        assert np.array_equal(x, xr)
        assert r < tol


def test_batched_reports_per_instance_status():
    inst = instances([4, 5])
    ops = [o for _, _, o, _ in inst]
    bs = [b for _, _, _, b in inst]
    xs, its, res, st = icc.solve_batched(ops, bs, tol=1e-14, max_iter=3)
    assert np.all(st == icc.ICC_NOT_CONVERGED) and np.all(its == 3)
