"""Many independent solves at once (icc_pcg_solve_batched): uneven cantilever designs.  FP64
instances equal their own sequential solves bitwise; mixed instances run in one batched solve and
are checked against their tight FP64 solutions."""
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


def test_batched_fp64_equals_sequential():
    # the FP64 instances run as ordinary solves on their own streams: bitwise the sequential result
    ks = [4, 9, 6, 12, 5, 8]
    inst = instances(ks)
    ops = [o for _, _, o, _ in inst]
    bs = [b for _, _, _, b in inst]
    tol = 1e-8
    xs, its, res, st = icc.solve_batched(ops, bs, tol=tol, precision=icc.FP64)
    assert np.all(st == icc.ICC_OK)
    for (p, sp, op, b), x, it, r in zip(inst, xs, its, res):
        s = icc.PcgSolver(20 * sp.ndof, tol)
        xr, itr, rr = s.solve(sp.ndof, b, None, op)
        assert it == itr and r == rr
        assert np.array_equal(x, xr)
        assert r < tol


def test_batched_mixed_one_launch_per_iteration():
    # the mixed instances share every iteration's persistent apply and fused vector step; each
    # reaches the tolerance on its own true residual and is within the mixed form's bar (1e-7) of
    # its tight FP64 solution
    ks = [4, 9, 6, 12, 5, 8, 16]
    inst = instances(ks, seed=11)
    ops = [o for _, _, o, _ in inst]
    bs = [b for _, _, _, b in inst]
    tol = 1e-8
    xs, its, res, st = icc.solve_batched(ops, bs, tol=tol, precision=icc.MIXED)
    assert np.all(st == icc.ICC_OK) and np.all(res < tol)
    for (p, sp, op, b), x, it in zip(inst, xs, its):
        xt, _, _ = icc.PcgSolver(40 * sp.ndof, 1e-12).solve(sp.ndof, b, None, op)
        assert np.linalg.norm(x - xt) / np.linalg.norm(xt) < 1e-7
        r = b - p.free_mask * op.matvec(p.free_mask * x)
        assert np.linalg.norm(r) / np.linalg.norm(b) < 1.5 * tol
    # an instance that starts converged (zero load) stops at once without disturbing the others
    bz = [np.zeros_like(bs[0])] + bs[1:]
    xs2, its2, res2, st2 = icc.solve_batched(ops, bz, tol=tol, precision=icc.MIXED)
    assert np.all(st2 >= 0) and np.all(xs2[0] == 0.0)
    for x, x2 in zip(xs[1:], xs2[1:]):
        assert np.linalg.norm(x - x2) / np.linalg.norm(x) < 1e-7


def test_batched_reports_per_instance_status():
    inst = instances([4, 5])
    ops = [o for _, _, o, _ in inst]
    bs = [b for _, _, _, b in inst]
    xs, its, res, st = icc.solve_batched(ops, bs, tol=1e-14, max_iter=3)
    assert np.all(st == icc.ICC_NOT_CONVERGED) and np.all(its == 3)
