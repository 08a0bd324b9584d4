"""Tensor-core (split-TF32) FP32 apply and the mixed-precision solve against the oracle."""
import numpy as np
import pytest

import immersed_catmull_clark_b200 as icc
from immersed_catmull_clark_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# The 3-term split-TF32 product with FP32 accumulation is FP32-accurate: relative 2-norm error
# of A x against the FP64 oracle.
TC_APPLY_TOL = 5e-6


def rel(a, b):
    return np.linalg.norm(np.asarray(a, dtype=np.float64) - b) / max(np.linalg.norm(b), 1e-300)


def setup(nsub, seed=0, bounds=((0.0, 2.0), (0.0, 1.0), (0.0, 1.0))):
    sp = icc.SpaceBox(bounds, nsub, 2)
    osp = O.Space(bounds, nsub, 2)
    lam, mu = icc.lame(1.0, 0.3)
    em = icc.elasticity_element_matrices(sp, lam, mu)
    rng = np.random.default_rng(seed)
    s = rng.uniform(0.01, 1.0, sp.nel) ** 3
    return sp, osp, em, s, rng


@pytest.mark.parametrize("nsub", [[8, 4, 4], [1, 1, 1], [9, 5, 6], [16, 8, 8], [24, 16, 12]])
def test_tc_apply_matches_oracle(nsub):
    sp, osp, em, s, rng = setup(nsub)
    k = O.Csr.assemble(osp, em.types, em.type_id.astype(np.int64), s)
    op = icc.MatrixFreeOperator(sp, em, s)
    x = rng.standard_normal(sp.ndof).astype(np.float32)
    y = op.matvec_f32(x)
    assert rel(y, k.matvec(x.astype(np.float64))) < TC_APPLY_TOL


@pytest.mark.parametrize("nsub,masked", [([64, 32, 24], False), ([72, 30, 26], True), ([128, 64, 64], True)])
def test_tc_apply_many_bricks_per_cta(nsub, masked):
    # more bricks than SMs: every persistent CTA walks several bricks (A-slot, accumulator and
    # staging reuse across bricks), checked against the oracle's matrix-free element loop
    sp, osp, em, s, rng = setup(nsub, seed=8)
    fm = (rng.uniform(size=sp.ndof) > 0.1).astype(np.uint8) if masked else None
    mode = icc.MASK_ZERO if masked else icc.MASK_NONE
    op = icc.MatrixFreeOperator(sp, em, s, fm, mode)
    x = rng.standard_normal(sp.ndof).astype(np.float32)
    y = op.matvec_f32(x)
    yo = O.mf_apply(osp, em.types, em.type_id.astype(np.int64), s, x.astype(np.float64), fm, mode)
    assert rel(y, yo) < TC_APPLY_TOL
    assert np.array_equal(y, op.matvec_f32(x))


def test_tc_apply_masked_and_deterministic():
    sp, osp, em, s, rng = setup([9, 5, 6], seed=4)
    fm = (rng.uniform(size=sp.ndof) > 0.25).astype(np.uint8)
    k = O.Csr.assemble(osp, em.types, em.type_id.astype(np.int64), s)
    op = icc.MatrixFreeOperator(sp, em, s, fm, icc.MASK_ZERO)
    x = rng.standard_normal(sp.ndof).astype(np.float32)
    y = op.matvec_f32(x)
    assert rel(y, fm * k.matvec(fm * x.astype(np.float64))) < TC_APPLY_TOL
    assert np.array_equal(y, op.matvec_f32(x))


def test_mixed_solve_cantilever():
    # 24x16x12 SIMP cantilever: FP64 refinement around the tensor-core FP32 PCG reaches 1e-8
    p = W.cantilever((24, 16, 12), seed=11)
    sp = icc.SpaceBox(p.bounds, p.nel, 2)
    osp = O.Space(p.bounds, p.nel, 2)
    lam, mu = icc.lame(1.0, 0.3)
    em = icc.elasticity_element_matrices(sp, lam, mu)
    k = O.Csr.assemble(osp, em.types, em.type_id.astype(np.int64), p.scale)
    b = W.rhs_masked(p)
    op = icc.MatrixFreeOperator(sp, em, p.scale, p.free_mask, icc.MASK_ZERO)
    tol = 1e-8
    xm, itm, resm = icc.PcgSolver(20 * sp.ndof, tol, precision=icc.MIXED).solve(sp.ndof, b, None, op)
    info = op.last_solve_info()
    assert resm < tol
    r_true = b - p.free_mask * k.matvec(p.free_mask * xm)
    assert np.linalg.norm(r_true) / np.linalg.norm(b) < 1.5 * tol
    assert info.outer_iterations >= 1 and info.mixed_applies == itm
    xd, itd, resd = icc.PcgSolver(20 * sp.ndof, 1e-12).solve(sp.ndof, b, None, op)
    c_ref, c = p.force @ xd, p.force @ xm
    assert abs(c - c_ref) / abs(c_ref) < 1e-6


def test_tc_apply_identity_rows():
    # ICC_MASK_IDENTITY: K on free rows of the masked input, identity on fixed rows
    sp, osp, em, s, rng = setup([17, 9, 6], seed=12)
    fm = (rng.uniform(size=sp.ndof) > 0.2).astype(np.uint8)
    op = icc.MatrixFreeOperator(sp, em, s, fm, icc.MASK_IDENTITY)
    x = rng.standard_normal(sp.ndof).astype(np.float32)
    y = op.matvec_f32(x)
    yo = O.mf_apply(osp, em.types, em.type_id.astype(np.int64), s, x.astype(np.float64), fm, icc.MASK_IDENTITY)
    assert rel(y, yo) < TC_APPLY_TOL


def test_tc_apply_translation_offset():
    # K annihilates rigid translations: a large constant added to every component must not
    # degrade the FP32 result (the split operands carry only each element's variation)
    sp, osp, em, s, rng = setup([24, 16, 12], seed=13)
    op = icc.MatrixFreeOperator(sp, em, s)
    w = rng.standard_normal(sp.ndof)
    shift = np.repeat([1e3, -2e3, 5e2], sp.ndof_sc)
    v = (w + shift).astype(np.float32)
    y = op.matvec_f32(v)
    yo = O.mf_apply(osp, em.types, em.type_id.astype(np.int64), s, v.astype(np.float64), None, icc.MASK_NONE)
    assert rel(y, yo) < TC_APPLY_TOL


def test_mixed_solve_identity_rows_patch_test():
    # rust/tests/iga_kernel.rs:94-117 with the mixed-precision solve: identity rows on the
    # boundary, a linear field recovered to the solver tolerance
    bounds = ((0.0, 1.0), (0.0, 2.0), (0.5, 1.0))
    nsub = [10, 8, 6]
    sp = icc.SpaceBox(bounds, nsub, 2)
    osp = O.Space(bounds, nsub, 2)
    lam, mu = icc.lame(1.0, 0.3)
    em = icc.elasticity_element_matrices(sp, lam, mu)
    g = osp.greville()
    nsc = sp.ndof_sc
    u = np.zeros(sp.ndof)
    for c in range(3):
        a = [((c * 3 + j) + 1.0) * 1e-2 - 0.03 for j in range(3)]
        u[c * nsc:(c + 1) * nsc] = sum(a[j] * g[:, j] for j in range(3)) + 0.1 * (c + 1.0)
    idx = np.indices(sp.ndof_dir[::-1]).reshape(3, -1)[::-1]
    on = np.zeros(nsc, dtype=bool)
    for d in range(3):
        on |= (idx[d] == 0) | (idx[d] == sp.ndof_dir[d] - 1)
    fixed = np.tile(on, 3)
    fm = (~fixed).astype(np.uint8)
    ub = np.where(fixed, u, 0.0)
    full = icc.MatrixFreeOperator(sp, em)
    b = np.where(fixed, ub, -full.matvec(ub))
    diag = np.where(fixed, 1.0, full.diagonal())
    op = icc.MatrixFreeOperator(sp, em, None, fm, icc.MASK_IDENTITY)
    tol = 1e-10
    x, it, res = icc.PcgSolver(20 * sp.ndof, tol, precision=icc.MIXED).solve(sp.ndof, b, diag, op)
    assert res < tol
    assert rel(x, u) < 1e-8
