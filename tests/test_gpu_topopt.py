"""Callers of the path in the SIMP loop on the device: the warm-started state solve, element
energies and the whole cantilever loop (filter + optimality criteria) against the oracle and the
reference's MATLAB fixture (rust/tests/topopt_vs_matlab.rs)."""
import json
import os

import numpy as np
import pytest

import immersed_catmull_clark_b200 as icc
from immersed_catmull_clark_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


def test_topopt_matches_matlab_fixture(golden_dir):
    # rust/tests/topopt_vs_matlab.rs:15-40: 6 iterations of the 8x4x2 cantilever, pcg_tol 1e-12,
    # compliance to 1e-7 and final densities to 1e-6 against the MATLAB export
    with open(os.path.join(golden_dir, "topopt3d_8x4x2.json")) as f:
        t = json.load(f)
    opt = icc.CantileverTopOpt(t["nel"], volfrac=t["volfrac"], penal=t["penal"], rmin=t["rmin"], pcg_tol=1e-12)
    h = opt.run(t["max_iter"])
    cref = np.array(t["compliance"])
    assert len(h.compliance) == len(cref)
    assert np.all(np.abs(h.compliance - cref) / cref < 1e-7)
    assert np.abs(h.density - np.array(t["xPhys"])).max() < 1e-6


def test_topopt_matches_oracle_loop():
    # a 12x6x4 cantilever for 8 iterations against the oracle's CantileverTopOpt::run restatement
    nel = [12, 6, 4]
    comp_o, dens_o, its_o = O.topopt_run(nel, 0.3, 3.0, 1.5, 8, 1e-10)
    h = icc.CantileverTopOpt(nel, pcg_tol=1e-10).run(8)
    assert len(h.compliance) == len(comp_o)
    assert np.all(np.abs(h.compliance - comp_o) / comp_o < 1e-7)
    assert np.abs(h.density - dens_o).max() < 1e-6


def test_topopt_mixed_precision_drift():
    # the same loop with mixed-precision state solves: compliance drift vs FP64 stays small
    nel = [16, 8, 4]
    h64 = icc.CantileverTopOpt(nel, pcg_tol=1e-8).run(6)
    hmx = icc.CantileverTopOpt(nel, pcg_tol=1e-8, precision=icc.MIXED).run(6)
    assert np.all(np.abs(hmx.compliance - h64.compliance) / h64.compliance < 1e-6)
    assert np.abs(hmx.density - h64.density).max() < 1e-4


def setup_cantilever(nel=(24, 16, 12), seed=11):
    p = W.cantilever(nel, seed=seed)
    sp = icc.SpaceBox(p.bounds, p.nel, 2)
    osp = O.Space(p.bounds, p.nel, 2)
    lam, mu = icc.lame(1.0, 0.3)
    em = icc.elasticity_element_matrices(sp, lam, mu)
    return p, sp, osp, em


def test_solve_state_matches_oracle():
    p, sp, osp, em = setup_cantilever()
    k = O.Csr.assemble(osp, em.types, em.type_id.astype(np.int64), p.scale)
    rng = np.random.default_rng(3)
    u0 = rng.standard_normal(sp.ndof) * 1e-2 * p.free_mask   # a warm start, zero on fixed DOFs
    uo, ito, reso = k.solve_state(p.free_mask, p.force, u0, 1e-10)
    op = icc.MatrixFreeOperator(sp, em, p.scale, p.free_mask, icc.MASK_ZERO)
    u, it, res = icc.solve_state(op, p.force, u0, 1e-10)
    assert res < 1e-10 and reso < 1e-10
    assert abs(it - ito) <= max(3, 0.02 * ito), (it, ito)
    assert rel(u, uo) < 1e-7
    assert np.all(u[p.free_mask == 0] == 0.0)
    # mixed precision: the same state to the same tolerance
    um, itm, resm = icc.solve_state(op, p.force, u0, 1e-10, precision=icc.MIXED)
    assert resm < 1e-10
    assert rel(um, uo) < 1e-7


def test_element_energies_match_oracle():
    p, sp, osp, em = setup_cantilever((9, 5, 6), seed=2)
    rng = np.random.default_rng(4)
    u = rng.standard_normal(sp.ndof)
    op = icc.MatrixFreeOperator(sp, em, p.scale)
    ee = op.element_energies(u)
    conn = sp.connectivity().reshape(sp.nel, 81)
    ue = u[conn]
    ref = np.einsum("ea,eab,eb->e", ue, em.types[em.type_id], ue)
    assert np.abs(ee - ref).max() < 1e-12 * np.abs(ref).max()
    # energy identity: sum_e s_e ee_e = u' K u with the scaled operator
    assert abs(p.scale @ ee - u @ op.matvec(u)) < 1e-12 * abs(u @ op.matvec(u))


def test_topopt_duplicate_load_case():
    # the same load twice: compliance doubles, the OC update is unchanged (sensitivities scale by
    # exactly 2), so the densities are bitwise those of the single case
    nel = [12, 6, 4]
    single = icc.CantileverTopOpt(nel, pcg_tol=1e-10)
    h1 = single.run(4)
    f = W.reference_tip_load(nel)
    double = icc.CantileverTopOpt(nel, pcg_tol=1e-10)
    double.set_loads(np.stack([f, f]))
    h2 = double.run(4)
    assert np.allclose(h2.compliance, 2 * h1.compliance, rtol=1e-12, atol=0)
    assert np.array_equal(h2.density, h1.density)


def test_topopt_four_load_cases_mixed_vs_fp64():
    # four tip load cases (shear +-y, axial +x, torsion) as simultaneous right-hand sides
    nel = [16, 8, 8]
    loads = W.tip_load_cases(nel, size=(2.0, 1.0, 1.0))
    runs = []
    for prec in (icc.FP64, icc.MIXED):
        t = icc.CantileverTopOpt(nel, size=(2.0, 1.0, 1.0), pcg_tol=1e-8, precision=prec)
        t.set_loads(loads)
        runs.append(t.run(4))
    h64, hmx = runs
    assert np.all(np.abs(hmx.compliance - h64.compliance) / h64.compliance < 1e-6)
    assert np.abs(hmx.density - h64.density).max() < 1e-4
    assert np.all(h64.compliance[1:] < h64.compliance[0])
