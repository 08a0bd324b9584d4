"""FP64 device operator and PCG against the oracle, the golden fixtures and the reference's
invariants (rust/tests/iga_vs_matlab.rs, iga_kernel.rs, immersed_vs_matlab.rs).  All compute goes
through the C ABI (libicc.so)."""
import json
import os

import numpy as np
import pytest

import immersed_catmull_clark_b200 as icc
from immersed_catmull_clark_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# K.u parity bar of the plain FP64 form (relative 2-norm)
APPLY_TOL = 1e-12


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


def setup(nsub, bounds=((0.0, 2.0), (0.0, 1.0), (0.0, 1.0)), seed=0, scale=True):
    sp = icc.SpaceBox(bounds, nsub, 2)
    osp = O.Space(bounds, nsub, 2)
    lam, mu = icc.lame(1.0, 0.3)
    em = icc.elasticity_element_matrices(sp, lam, mu)
    rng = np.random.default_rng(seed)
    s = rng.uniform(0.01, 1.0, sp.nel) ** 3 if scale else None
    return sp, osp, em, s, rng


GRIDS = [[1, 1, 1], [2, 3, 4], [4, 3, 3], [5, 6, 7], [8, 4, 4], [9, 5, 5], [17, 9, 6], [16, 8, 8], [24, 16, 12]]


@pytest.mark.parametrize("nsub", GRIDS)
def test_apply_matches_oracle(nsub):
    sp, osp, em, s, rng = setup(nsub)
    k = O.Csr.assemble(osp, em.types, em.type_id.astype(np.int64), s)
    op = icc.MatrixFreeOperator(sp, em, s)
    for _ in range(2):
        x = rng.standard_normal(sp.ndof)
        assert rel(op.matvec(x), k.matvec(x)) < APPLY_TOL


@pytest.mark.parametrize("mode", [icc.MASK_ZERO, icc.MASK_IDENTITY])
def test_masked_apply_matches_oracle(mode):
    sp, osp, em, s, rng = setup([9, 5, 6], seed=3)
    fm = (rng.uniform(size=sp.ndof) > 0.25).astype(np.uint8)
    k = O.Csr.assemble(osp, em.types, em.type_id.astype(np.int64), s)
    op = icc.MatrixFreeOperator(sp, em, s, fm, mode)
    x = rng.standard_normal(sp.ndof)
    ref = k.matvec(fm * x)
    ref = fm * ref if mode == icc.MASK_ZERO else np.where(fm > 0, ref, x)
    assert rel(op.matvec(x), ref) < APPLY_TOL


def test_fixture_probes(golden_dir):
    # rust/tests/iga_vs_matlab.rs:52-60 on the 3-D p = 2 case, unit scale
    with open(os.path.join(golden_dir, "iga_kernel.json")) as f:
        d = json.load(f)
    case = d["cases"][4]
    sp = icc.SpaceBox(np.array(case["bounds"], dtype=float), case["nsub"], 2)
    em = icc.elasticity_element_matrices(sp, d["lambda"], d["mu"])
    op = icc.MatrixFreeOperator(sp, em)
    probes = np.array(case["probes"]).reshape(sp.ndof, 3)
    for j in range(1, 4):
        v = np.sin(0.37 * np.arange(1, sp.ndof + 1) * j)
        assert rel(op.matvec(v), probes[:, j - 1]) < 1e-13


def test_immersed_volume_operator_fixture(golden_dir):
    # the scaled volume operator (emin + (1-emin) w_e) K_e of rust/src/immersed.rs:483-495 against
    # k_probe - kgp_probe of rust/tests/fixtures/immersed_tilted_box.json
    with open(os.path.join(golden_dir, "immersed_tilted_box.json")) as f:
        d = json.load(f)
    gb = np.array(d["grid_bounds"]).reshape(3, 2)
    sp = icc.SpaceBox(gb, d["grid_res"], 2)
    lam, mu = icc.lame(d["young"], d["poisson"])
    em = icc.elasticity_element_matrices(sp, lam, mu)
    s = d["emin"] + (1 - d["emin"]) * np.array(d["weights"])
    op = icc.MatrixFreeOperator(sp, em, s)
    v = np.sin(0.37 * np.arange(1, sp.ndof + 1))
    assert rel(op.matvec(v), np.array(d["k_probe"]) - np.array(d["kgp_probe"])) < 1e-12


@pytest.mark.parametrize("nsub", [[1, 1, 1], [5, 6, 7], [24, 16, 12]])
def test_diagonal_bit_identical(nsub):
    sp, osp, em, s, _ = setup(nsub, seed=5)
    k = O.Csr.assemble(osp, em.types, em.type_id.astype(np.int64), s)
    op = icc.MatrixFreeOperator(sp, em, s)
    assert np.array_equal(op.diagonal(), k.diagonal())


def test_apply_is_deterministic():
    sp, _, em, s, rng = setup([24, 16, 12], seed=7)
    op = icc.MatrixFreeOperator(sp, em, s)
    x = rng.standard_normal(sp.ndof)
    assert np.array_equal(op.matvec(x), op.matvec(x))


def test_update_scale():
    sp, osp, em, s, rng = setup([9, 5, 5], seed=2)
    op = icc.MatrixFreeOperator(sp, em, s)
    s2 = rng.uniform(0.01, 1.0, sp.nel)
    op.update_scale(s2)
    k = O.Csr.assemble(osp, em.types, em.type_id.astype(np.int64), s2)
    x = rng.standard_normal(sp.ndof)
    assert rel(op.matvec(x), k.matvec(x)) < APPLY_TOL


def test_symmetry_and_rigid_modes():
    # rust/tests/iga_kernel.rs:49-92 on the device operator (unit scale and random scale)
    for scale in (False, True):
        sp, osp, em, s, rng = setup([6, 5, 4], bounds=((0, 1.2), (0, 0.6), (0, 0.3)), scale=scale)
        op = icc.MatrixFreeOperator(sp, em, s)
        fro = O.Csr.assemble(osp, em.types, em.type_id.astype(np.int64), s).frobenius()
        x, y = rng.standard_normal(sp.ndof), rng.standard_normal(sp.ndof)
        ax, ay = op.matvec(x), op.matvec(y)
        assert abs(y @ ax - x @ ay) < 1e-13 * fro * np.linalg.norm(x) * np.linalg.norm(y)
        g = osp.greville()
        nsc = sp.ndof_sc
        modes = []
        for c in range(3):
            m = np.zeros(sp.ndof); m[c * nsc:(c + 1) * nsc] = 1.0
            modes.append(m)
        for a, b in [(0, 1), (1, 2), (0, 2)]:
            m = np.zeros(sp.ndof)
            m[a * nsc:(a + 1) * nsc] = -g[:, b]
            m[b * nsc:(b + 1) * nsc] = g[:, a]
            modes.append(m)
        for m in modes:
            assert np.linalg.norm(op.matvec(m)) / (fro * np.linalg.norm(m)) < 1e-13


def test_pcg_matches_oracle_cantilever():
    # 24x16x12 cantilever (19,656 DOF): FP64 device PCG vs the oracle's PcgSolver on the CSR
    p = W.cantilever((24, 16, 12), seed=11)
    sp = icc.SpaceBox(p.bounds, p.nel, 2)
    osp = O.Space(p.bounds, p.nel, 2)
    lam, mu = icc.lame(1.0, 0.3)
    em = icc.elasticity_element_matrices(sp, lam, mu)
    k = O.Csr.assemble(osp, em.types, em.type_id.astype(np.int64), p.scale)
    b = W.rhs_masked(p)
    diag = np.maximum(k.diagonal(), 1e-12)
    tol = 1e-8
    xo, ito, reso = k.pcg(b, diag, 20 * sp.ndof, tol, p.free_mask, icc.MASK_ZERO)
    op = icc.MatrixFreeOperator(sp, em, p.scale, p.free_mask, icc.MASK_ZERO)
    solver = icc.PcgSolver(20 * sp.ndof, tol)
    x, it, res = solver.solve(sp.ndof, b, diag, op)
    assert solver.status == icc.ICC_OK
    assert res < tol and reso < tol
    assert abs(it - ito) <= max(3, 0.02 * ito), (it, ito)
    # both iterates satisfy the stopping rule; they agree to the solver tolerance scale
    r_true = b - k.matvec(p.free_mask * x) * p.free_mask
    assert np.linalg.norm(r_true) / np.linalg.norm(b) < 2 * tol
    assert rel(x, xo) < 1e-5


def test_pcg_breakdown_and_maxiter():
    sp, osp, em, s, rng = setup([4, 3, 3], seed=9)
    op = icc.MatrixFreeOperator(sp, em, s)
    b = rng.standard_normal(sp.ndof)
    solver = icc.PcgSolver(1, 1e-12)
    x, it, res = solver.solve(sp.ndof, b, None, op)
    assert solver.status == icc.ICC_NOT_CONVERGED and it == 1
    # a negative scale makes the operator indefinite: the reference breaks on p'Ap <= 0
    op.update_scale(-np.ones(sp.nel))
    solver = icc.PcgSolver(100, 1e-12)
    x, it, res = solver.solve(sp.ndof, b, np.ones(sp.ndof), op)
    assert solver.status == icc.ICC_BREAKDOWN and it == 1


def test_patch_test_on_device():
    # rust/tests/iga_kernel.rs:94-117 (p = 2, 3-D): identity rows on the boundary, CG at 1e-12
    bounds = ((0.0, 1.0), (0.0, 2.0), (0.5, 1.0))
    nsub = [5, 4, 3]
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
    b = np.where(fixed, 0.0, -full.matvec(ub))
    diag = np.where(fixed, 1.0, full.diagonal())
    op = icc.MatrixFreeOperator(sp, em, None, fm, icc.MASK_IDENTITY)
    x, it, res = icc.PcgSolver(20 * sp.ndof, 1e-12).solve(sp.ndof, b, diag, op)
    assert res < 1e-11
    uh = np.where(fixed, ub, x)
    assert rel(uh, u) < 1e-10


def test_apply_at_scale_128x64x64():
    # full-size operator (1.7 M DOF) against the oracle's matrix-free CPU loop
    p = W.cantilever((128, 64, 64), smooth=True, seed=1)
    sp = icc.SpaceBox(p.bounds, p.nel, 2)
    osp = O.Space(p.bounds, p.nel, 2)
    lam, mu = icc.lame(1.0, 0.3)
    em = icc.elasticity_element_matrices(sp, lam, mu)
    op = icc.MatrixFreeOperator(sp, em, p.scale, p.free_mask, icc.MASK_ZERO)
    x = np.random.default_rng(4).standard_normal(sp.ndof)
    y = op.matvec(x)
    yo = O.mf_apply(osp, em.types, em.type_id.astype(np.int64), p.scale, x, p.free_mask, icc.MASK_ZERO)
    assert rel(y, yo) < APPLY_TOL
