"""Failure paths of the solve, made on the host: a NaN in the load vector must end both precision
forms with ICC_NAN (the reference's PCG would carry the NaN to its last iterate,
rust/src/solver.rs:40-73; here the reductions detect it), and a grid barrier of the mixed solve's
fused vector step whose poll limit runs out must end the solve with ICC_TIMEOUT and leave the
handle usable.  Neither faults, traps nor hangs the GPU: every device wait is bounded."""
import numpy as np
import pytest

import immersed_catmull_clark_b200 as icc
from immersed_catmull_clark_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def cantilever(nel=(16, 8, 8), seed=21):
    p = W.cantilever(nel, seed=seed)
    sp = icc.SpaceBox(p.bounds, p.nel, 2)
    lam, mu = icc.lame(1.0, 0.3)
    em = icc.elasticity_element_matrices(sp, lam, mu)
    op = icc.MatrixFreeOperator(sp, em, p.scale, p.free_mask, icc.MASK_ZERO)
    return p, sp, em, op


@pytest.mark.parametrize("precision", [icc.FP64, icc.MIXED])
def test_nan_in_load_reports_icc_nan(precision):
    p, sp, em, op = cantilever()
    b = W.rhs_masked(p)
    b[np.flatnonzero(p.free_mask)[17]] = np.nan
    with pytest.raises(icc.IccError) as ei:
        icc.PcgSolver(20 * sp.ndof, 1e-8, precision=precision).solve(sp.ndof, b, None, op)
    assert ei.value.code == icc.ICC_NAN
    # the handle still solves a finite system afterwards
    b = W.rhs_masked(p)
    x, it, res = icc.PcgSolver(20 * sp.ndof, 1e-8, precision=precision).solve(sp.ndof, b, None, op)
    assert res < 1e-8


def test_grid_barrier_timeout_then_recovery():
    p, sp, em, op = cantilever()
    b = W.rhs_masked(p)
    solver = icc.PcgSolver(20 * sp.ndof, 1e-8, precision=icc.MIXED)
    op.set_wait_limit(0)   # no poll at all: every CTA that is not the last to arrive gives up
    with pytest.raises(icc.IccError) as ei:
        solver.solve(sp.ndof, b, None, op)
    assert ei.value.code == icc.ICC_TIMEOUT
    op.set_wait_limit(1 << 22)
    x, it, res = solver.solve(sp.ndof, b, None, op)
    assert solver.status == icc.ICC_OK and res < 1e-8
    # the tensor-core apply on the same handle is unaffected
    osp = O.Space(p.bounds, p.nel, 2)
    x32 = np.random.default_rng(2).standard_normal(sp.ndof).astype(np.float32)
    y = op.matvec_f32(x32)
    yo = O.mf_apply(osp, em.types, em.type_id.astype(np.int64), p.scale, x32.astype(np.float64), p.free_mask,
                    icc.MASK_ZERO)
    assert np.linalg.norm(y - yo) / np.linalg.norm(yo) < 5e-6
