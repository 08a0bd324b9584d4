"""The operator with a stabilisation term (icc_op_set_extra_triplets) on the device: the closures
of the reference's immersed solves, which add the stabilisation matrix to the stiffness inside
PcgSolver::solve (rust/src/immersed.rs:514-548 and :558-566; rust/src/topopt_immersed.rs:174-183).

* The reference fixture rust/tests/fixtures/immersed_tilted_box.json with its legacy springs:
  K*v probe to 1e-12, and the solve against the MATLAB direct solve (u to 1e-6, compliance to
  1e-9), as rust/tests/immersed_vs_matlab.rs:20-73 checks.
* The face ghost penalty: the device operator K + GP against the oracle's CSR assembled from its
  own ghost-penalty triplets (1e-12), in FP64 and on the tensor cores, and its solve against the
  oracle's CSR PCG."""
import json
import os

import numpy as np
import pytest

import immersed_catmull_clark_b200 as icc
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def tilted(golden_dir):
    with open(os.path.join(golden_dir, "immersed_tilted_box.json")) as f:
        d = json.load(f)
    gb = np.array(d["grid_bounds"]).reshape(3, 2)
    sp = icc.SpaceBox(gb, d["grid_res"], 2)
    osp = O.Space(gb, d["grid_res"], 2)
    lam, mu = icc.lame(d["young"], d["poisson"])
    em = icc.elasticity_element_matrices(sp, lam, mu)
    s = d["emin"] + (1 - d["emin"]) * np.array(d["weights"])
    st = np.array(d["status"], dtype=np.int8)
    fm = (np.array(d["free_mask"]) != 0).astype(np.uint8)
    return dict(d=d, sp=sp, osp=osp, em=em, s=s, st=st, fm=fm)


def oracle_k_plus_s(t, r, c, v):
    """The oracle's assembled K (AssemblyPattern) plus the stabilisation CSR from its triplets."""
    k = O.Csr.assemble(t["osp"], t["em"].types, t["em"].type_id.astype(np.int64), t["s"])
    s = O.Csr.from_triplets(t["sp"].ndof, r, c, v)
    ip, ix, dv = k.export()
    rows = np.repeat(np.arange(t["sp"].ndof), np.diff(ip))
    return O.Csr.from_triplets(t["sp"].ndof, np.concatenate([r, rows]), np.concatenate([c, ix]),
                               np.concatenate([v, dv])), s


def test_legacy_fixture_probe_and_solve(tilted):
    t = tilted
    d, sp = t["d"], t["sp"]
    r, c, v = icc.legacy_stabilization(sp, t["st"], d["gamma_gp"])
    op = icc.MatrixFreeOperator(sp, t["em"], t["s"])
    op.set_extra_triplets(r, c, v)
    probe = np.sin(0.37 * np.arange(1, sp.ndof + 1))
    assert rel(op.matvec(probe), np.array(d["k_probe"])) < 1e-12
    # the solve of rust/src/immersed.rs:551-570: masked closure, diagonal clamped at 1e-6
    opm = icc.MatrixFreeOperator(sp, t["em"], t["s"], t["fm"], icc.MASK_ZERO)
    opm.set_extra_triplets(r, c, v)
    force = np.array(d["load"])
    b = np.where(t["fm"] > 0, force, 0.0)
    diag = np.maximum(opm.diagonal(), 1e-6)
    u, it, res = icc.PcgSolver(20 * sp.ndof, 1e-12).solve(sp.ndof, b, diag, opm)
    u = np.where(t["fm"] > 0, u, 0.0)
    assert rel(u, np.array(d["u_direct"])) < 1e-6
    assert abs(force @ u - d["compliance"]) / d["compliance"] < 1e-9
    um, itm, resm = icc.PcgSolver(20 * sp.ndof, 1e-10, precision=icc.MIXED).solve(sp.ndof, b, diag, opm)
    um = np.where(t["fm"] > 0, um, 0.0)
    assert resm < 1e-10
    assert rel(um, np.array(d["u_direct"])) < 1e-6


def test_ghost_penalty_operator_matches_oracle_assembly(tilted):
    t = tilted
    sp = t["sp"]
    r, c, v = icc.ghost_penalty(sp, t["st"], 1e-2, t["d"]["young"])
    ro, co, vo = O.ghost_penalty(t["osp"], t["st"], 1e-2, t["d"]["young"])
    ks, s_only = oracle_k_plus_s(t, ro, co, vo)
    rng = np.random.default_rng(5)
    for mode in (icc.MASK_NONE, icc.MASK_ZERO, icc.MASK_IDENTITY):
        fm = t["fm"] if mode != icc.MASK_NONE else None
        op = icc.MatrixFreeOperator(sp, t["em"], t["s"], fm, mode)
        op.set_extra_triplets(r, c, v)
        x = rng.standard_normal(sp.ndof)
        if mode == icc.MASK_NONE:
            ref = ks.matvec(x)
        else:
            y = ks.matvec(t["fm"] * x)
            ref = t["fm"] * y if mode == icc.MASK_ZERO else np.where(t["fm"] > 0, y, x)
        assert rel(op.matvec(x), ref) < 1e-12, mode
        x32 = x.astype(np.float32)
        x64 = x32.astype(np.float64)
        if mode == icc.MASK_NONE:
            ref32 = ks.matvec(x64)
        else:
            y = ks.matvec(t["fm"] * x64)
            ref32 = t["fm"] * y if mode == icc.MASK_ZERO else np.where(t["fm"] > 0, y, x64)
        assert rel(op.matvec_f32(x32), ref32) < 5e-6, mode
    # the diagonal includes the term's diagonal
    op = icc.MatrixFreeOperator(sp, t["em"], t["s"])
    op.set_extra_triplets(r, c, v)
    dk = O.Csr.assemble(t["osp"], t["em"].types, t["em"].type_id.astype(np.int64), t["s"]).diagonal()
    assert np.abs(op.diagonal() - (dk + s_only.diagonal())).max() <= 1e-15 * np.abs(dk).max()
    # removing the term restores K
    op.set_extra_triplets([], [], [])
    x = rng.standard_normal(sp.ndof)
    kk = O.Csr.assemble(t["osp"], t["em"].types, t["em"].type_id.astype(np.int64), t["s"])
    assert rel(op.matvec(x), kk.matvec(x)) < 1e-12


@pytest.mark.parametrize("precision", [icc.FP64, icc.MIXED])
def test_ghost_penalty_solve_matches_oracle(tilted, precision):
    t = tilted
    sp = t["sp"]
    r, c, v = icc.ghost_penalty(sp, t["st"], 1e-2, t["d"]["young"])
    ks, _ = oracle_k_plus_s(t, r, c, v)
    force = np.array(t["d"]["load"])
    b = np.where(t["fm"] > 0, force, 0.0)
    diag = np.maximum(ks.diagonal(), 1e-6)
    xt, _, _ = ks.pcg(b, diag, 40 * sp.ndof, 1e-14, t["fm"], icc.MASK_ZERO)
    op = icc.MatrixFreeOperator(sp, t["em"], t["s"], t["fm"], icc.MASK_ZERO)
    op.set_extra_triplets(r, c, v)
    x, it, res = icc.PcgSolver(20 * sp.ndof, 1e-10, precision=precision).solve(sp.ndof, b, diag, op)
    assert res < 1e-10
    r_true = b - t["fm"] * ks.matvec(t["fm"] * x)
    assert np.linalg.norm(r_true) / np.linalg.norm(b) < 1.5e-10
    assert rel(x, xt) < 1e-7
