"""The device operators of x-slabs (slabs.slab_operator): each slab's local space with the global
grid's element types restricted to it.  Applied to the slabs' parts of a vector and summed on the
shared control-point planes, they give the global operator's y = A x (the communication that does
this sum across ranks is tested with gloo ranks on the CPU)."""
import numpy as np
import pytest

import immersed_catmull_clark_b200 as icc
from immersed_catmull_clark_b200 import slabs as S
from immersed_catmull_clark_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world", [2, 3])
def test_slab_operators_sum_to_global(world):
    p = W.cantilever((24, 8, 6), seed=9)
    sp = icc.SpaceBox(p.bounds, p.nel, 2)
    lam, mu = icc.lame(1.0, 0.3)
    em = icc.elasticity_element_matrices(sp, lam, mu)
    op = icc.MatrixFreeOperator(sp, em, p.scale, p.free_mask, icc.MASK_ZERO)
    x = np.random.default_rng(1).standard_normal(sp.ndof)
    yg = op.matvec(x)
    y = np.zeros(sp.ndof)
    for rank, (e0, e1) in enumerate(S.partition(p.nel[0], world)):
        slab = S.Slab(rank, world, tuple(p.nel), e0, e1)
        lsp, lop = S.slab_operator(icc, slab, p.bounds, em, p.scale, p.free_mask, icc.MASK_ZERO)
        ids = slab.dof_ids()
        np.add.at(y, ids, lop.matvec(x[ids]))
    assert np.linalg.norm(y - yg) / np.linalg.norm(yg) < 1e-13


@pytest.mark.parametrize("world", [2, 3])
def test_slab_tensor_core_operators_sum_to_global(world):
    """The same for the FP32 tensor-core apply the mixed-precision slab solve uses."""
    p = W.cantilever((24, 8, 6), seed=9)
    sp = icc.SpaceBox(p.bounds, p.nel, 2)
    lam, mu = icc.lame(1.0, 0.3)
    em = icc.elasticity_element_matrices(sp, lam, mu)
    op = icc.MatrixFreeOperator(sp, em, p.scale, p.free_mask, icc.MASK_ZERO)
    x = np.random.default_rng(2).standard_normal(sp.ndof).astype(np.float32)
    yg = op.matvec_f32(x).astype(np.float64)
    y = np.zeros(sp.ndof)
    for rank, (e0, e1) in enumerate(S.partition(p.nel[0], world)):
        slab = S.Slab(rank, world, tuple(p.nel), e0, e1)
        lsp, lop = S.slab_operator(icc, slab, p.bounds, em, p.scale, p.free_mask, icc.MASK_ZERO)
        ids = slab.dof_ids()
        np.add.at(y, ids, lop.matvec_f32(np.ascontiguousarray(x[ids])).astype(np.float64))
    assert np.linalg.norm(y - yg) / np.linalg.norm(yg) < 5e-6
