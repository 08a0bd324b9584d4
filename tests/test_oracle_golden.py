"""The CPU oracle against the reference's own golden vectors and invariants.

Mirrors rust/tests/iga_vs_matlab.rs, rust/tests/immersed_vs_matlab.rs,
rust/tests/topopt_vs_matlab.rs and rust/tests/iga_kernel.rs with the same tolerances, so the
oracle that checks the CUDA path is itself pinned to the reference's MATLAB-exported results.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O


def rel_err(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module")
def iga(golden_dir):
    with open(os.path.join(golden_dir, "iga_kernel.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def immersed(golden_dir):
    with open(os.path.join(golden_dir, "immersed_tilted_box.json")) as f:
        return json.load(f)


def test_gauss_rule_is_exact():
    # rust/src/iga/quadrature.rs:72-82
    for n in range(1, 11):
        x, w = O.gauss_legendre(n)
        for k in range(2 * n):
            exact = 2.0 / (k + 1.0) if k % 2 == 0 else 0.0
            assert abs(np.sum(w * x ** k) - exact) < 1e-13
        assert np.all(np.diff(x) > 0)


def test_knot_vector_multiplicities():
    # rust/src/iga/quadrature.rs:84-88
    assert np.array_equal(open_knots := O.open_knots(3, 2, 0),
                          [0, 0, 0, 1 / 3, 1 / 3, 2 / 3, 2 / 3, 1, 1, 1]), open_knots
    assert len(O.open_knots(4, 3, 2)) == 4 + 2 * 3 + 1


def test_partition_of_unity():
    # rust/src/iga/basis.rs:178-211 (values sum to one, derivatives to zero)
    for p in range(1, 5):
        knots = O.open_knots(7, p, p - 1)
        for x in np.linspace(0, 1, 101):
            _, v, d = O.basis_funs(knots, p, x)
            assert abs(v.sum() - 1) < 1e-13 and abs(d.sum()) < 1e-10


def test_space_counts_and_connectivity():
    # rust/src/iga/space.rs:217-228
    sp = O.Space([[0, 1.2], [0, 0.6], [0, 0.3]], [4, 3, 2], 2)
    assert sp.ndof_dir == [6, 5, 4] and sp.ndof == 360 and sp.nsh == 81
    c = sp.connectivity()
    assert c[0] == 0
    assert c.reshape(sp.nel, 81)[-1, 26] == sp.ndof_sc - 1


def test_kernel_matches_matlab_reference(iga):
    # rust/tests/iga_vs_matlab.rs:22-73, tolerance 1e-13
    lam, mu = iga["lambda"], iga["mu"]
    assert len(iga["cases"]) == 6
    for case in iga["cases"]:
        sp = O.Space(np.array(case["bounds"], dtype=float), case["nsub"], case["degree"])
        assert sp.ndof == case["ndof"]
        assert np.array_equal(sp.connectivity(), np.array(case["connectivity"]).reshape(-1))
        types, tid, _ = sp.element_matrices(lam, mu)
        assert len(types) == case["ntypes"]
        k = O.Csr.assemble(sp, types, tid, None, pattern=False)
        assert abs(k.frobenius() - case["frobenius"]) / case["frobenius"] < 1e-13
        probes = np.array(case["probes"]).reshape(sp.ndof, 3)
        for j in range(1, 4):
            v = np.sin(0.37 * np.arange(1, sp.ndof + 1) * j)
            assert rel_err(k.matvec(v), probes[:, j - 1]) < 1e-13
        assert rel_err(sp.load_vector(0), case["load"]) < 1e-13


def test_assembly_pattern_equals_triplet_assembly(iga):
    # AssemblyPattern (rust/src/sparse.rs:128-175) and the triplet path (:179-200) agree
    case = iga["cases"][4]
    sp = O.Space(np.array(case["bounds"], dtype=float), case["nsub"], 2)
    types, tid, _ = sp.element_matrices(iga["lambda"], iga["mu"])
    s = np.random.default_rng(0).uniform(0.01, 1.0, sp.nel)
    a = O.Csr.assemble(sp, types, tid, s, pattern=True)
    b = O.Csr.assemble(sp, types, tid, s, pattern=False)
    v = np.sin(0.37 * np.arange(1, sp.ndof + 1))
    assert rel_err(a.matvec(v), b.matvec(v)) < 1e-14


def test_matrix_free_oracle_equals_csr(iga):
    # the matrix-free CPU element loop reproduces the assembled CSR operator and its diagonal
    sp = O.Space([[0, 2], [0, 1], [0, 1]], [7, 5, 6], 2)
    lam, mu = O.lame(1.0, 0.3)
    types, tid, _ = sp.element_matrices(lam, mu)
    rng = np.random.default_rng(1)
    s = rng.uniform(0.01, 1.0, sp.nel)
    k = O.Csr.assemble(sp, types, tid, s)
    x = rng.standard_normal(sp.ndof)
    assert rel_err(O.mf_apply(sp, types, tid, s, x), k.matvec(x)) < 1e-14
    assert np.array_equal(O.mf_diagonal(sp, types, tid, s), k.diagonal())
    fm = (rng.uniform(size=sp.ndof) > 0.2).astype(np.uint8)
    ym = O.mf_apply(sp, types, tid, s, x, fm, 1)
    yr = fm * k.matvec(fm * x)
    assert rel_err(ym, yr) < 1e-14


def test_immersed_solver_matches_matlab_reference(immersed):
    # rust/tests/immersed_vs_matlab.rs:20-73
    d = immersed
    nodes = np.array(d["nodes"]).reshape(-1, 3)
    tris = np.array(d["elements"]).reshape(-1, 3)
    lo, hi = nodes.min(0), nodes.max(0)
    pad = 0.05 * (hi - lo)
    gb = np.stack([lo - pad, hi + pad], 1)  # padded_bounds, rust/src/immersed.rs:452-464
    assert np.abs(gb.reshape(-1) - np.array(d["grid_bounds"]).reshape(-1)).max() < 1e-14
    w, st = O.element_weights(nodes, tris, gb, d["grid_res"], [4, 4, 4])
    assert np.array_equal(st, np.array(d["status"], dtype=np.int8))
    assert np.abs(w - np.array(d["weights"])).max() < 1e-7
    sp = O.Space(gb, d["grid_res"], d["degree"])
    lam, mu = O.lame(d["young"], d["poisson"])
    types, tid, _ = sp.element_matrices(lam, mu)
    r, c, v = O.legacy_stabilization(sp, st, d["gamma_gp"])
    stab = O.Csr.from_triplets(sp.ndof, r, c, v)
    kgp = d["kgp_frobenius"]
    assert abs(stab.frobenius() - kgp) <= 1e-12 * max(kgp, 1.0)
    scale = d["emin"] + (1 - d["emin"]) * w
    conn = sp.connectivity().reshape(sp.nel, 81)
    rows = [r, np.repeat(conn, 81, axis=1).reshape(-1)]
    cols = [c, np.tile(conn, (1, 81)).reshape(-1)]
    vals = [v, (scale[:, None, None] * types[tid]).reshape(-1)]
    k = O.Csr.from_triplets(sp.ndof, np.concatenate(rows), np.concatenate(cols), np.concatenate(vals))
    x = np.sin(0.37 * np.arange(1, sp.ndof + 1))
    assert rel_err(k.matvec(x), d["k_probe"]) < 1e-12
    # the scaled volume operator alone (the hot path) against k_probe - kgp_probe
    kv = O.Csr.assemble(sp, types, tid, scale)
    assert rel_err(kv.matvec(x), np.array(d["k_probe"]) - np.array(d["kgp_probe"])) < 1e-12
    fm, f = O.immersed_bc(sp)
    assert rel_err(f, d["load"]) < 1e-15
    assert np.array_equal(fm, np.array(d["free_mask"], dtype=np.uint8))
    u, it, res, comp = O.solve_immersed(k, fm, f, 1e-12, 20 * sp.ndof)
    assert rel_err(u, d["u_direct"]) < 1e-6
    assert abs(comp - d["compliance"]) / d["compliance"] < 1e-9


def test_topopt_matches_matlab_reference(golden_dir):
    # rust/tests/topopt_vs_matlab.rs:15-40
    with open(os.path.join(golden_dir, "topopt3d_8x4x2.json")) as f:
        t = json.load(f)
    comp, dens, _ = O.topopt_run(t["nel"], t["volfrac"], t["penal"], t["rmin"], t["max_iter"], 1e-12)
    cref = np.array(t["compliance"])
    assert len(comp) == len(cref)
    assert np.all(np.abs(comp - cref) / cref < 1e-7)
    assert np.abs(dens - np.array(t["xPhys"])).max() < 1e-6


def _rigid_modes(sp):
    g = sp.greville()
    modes = []
    for c in range(sp.dim):
        m = np.zeros(sp.ndof); m[c * sp.ndof_sc:(c + 1) * sp.ndof_sc] = 1.0
        modes.append(m)
    planes = [(0, 1)] if sp.dim == 2 else [(0, 1), (1, 2), (0, 2)]
    for a, b in planes:
        m = np.zeros(sp.ndof)
        m[a * sp.ndof_sc:(a + 1) * sp.ndof_sc] = -g[:, b]
        m[b * sp.ndof_sc:(b + 1) * sp.ndof_sc] = g[:, a]
        modes.append(m)
    return modes


def test_stiffness_symmetric_and_annihilates_rigid_modes():
    # rust/tests/iga_kernel.rs:49-92
    for bounds, nsub, p in [([[0, 1], [0, 0.5]], [4, 3], 3), ([[0, 1.2], [0, 0.6], [0, 0.3]], [3, 2, 2], 2)]:
        sp = O.Space(bounds, nsub, p)
        lam, mu = O.lame(1.0, 0.3)
        types, tid, _ = sp.element_matrices(lam, mu)
        k = O.Csr.assemble(sp, types, tid, None, pattern=False)
        fro = k.frobenius()
        ip, ix, d = k.export()
        for r in range(sp.ndof):
            for idx in range(ip[r], ip[r + 1]):
                assert abs(d[idx] - k.get(ix[idx], r)) < 1e-13 * fro
        for m in _rigid_modes(sp):
            assert np.linalg.norm(k.matvec(m)) / (fro * np.linalg.norm(m)) < 1e-13


def _all_boundary(sp):
    fixed = np.zeros(sp.ndof, dtype=bool)
    idx = np.indices(sp.ndof_dir[::-1]).reshape(sp.dim, -1)[::-1]  # x fastest
    on = np.zeros(sp.ndof_sc, dtype=bool)
    for d in range(sp.dim):
        on |= (idx[d] == 0) | (idx[d] == sp.ndof_dir[d] - 1)
    for c in range(sp.dim):
        fixed[c * sp.ndof_sc:(c + 1) * sp.ndof_sc] = on
    return fixed


def _solve_dirichlet(k, sp, rhs, fixed, u_fixed):
    # rust/tests/iga_kernel.rs:29-52 (identity rows on fixed DOFs, CG at 1e-12)
    ub = np.where(fixed, u_fixed, 0.0)
    b = np.where(fixed, 0.0, rhs - k.matvec(ub))
    diag = np.where(fixed, 1.0, k.diagonal())
    x, _, res = k.pcg(b, diag, 20 * sp.ndof, 1e-12, (~fixed).astype(np.uint8), 2)
    assert res < 1e-11
    return np.where(fixed, ub, x)


def test_patch_test_reproduces_linear_field():
    # rust/tests/iga_kernel.rs:94-117
    for bounds, nsub, p in [([[0, 2], [-1, 0.5]], [5, 4], 2), ([[0, 1], [0, 2], [0.5, 1]], [3, 4, 3], 3)]:
        sp = O.Space(bounds, nsub, p)
        g = sp.greville()
        dim = sp.dim
        u = np.zeros(sp.ndof)
        for c in range(dim):
            a = [((c * dim + j) + 1.0) * 1e-2 - 0.03 for j in range(dim)]
            u[c * sp.ndof_sc:(c + 1) * sp.ndof_sc] = sum(a[j] * g[:, j] for j in range(dim)) + 0.1 * (c + 1.0)
        lam, mu = O.lame(1.0, 0.3)
        types, tid, _ = sp.element_matrices(lam, mu)
        k = O.Csr.assemble(sp, types, tid, None, pattern=False)
        fixed = _all_boundary(sp)
        uh = _solve_dirichlet(k, sp, np.zeros(sp.ndof), fixed, u)
        assert rel_err(uh, u) < 1e-10


def test_manufactured_solution_rate():
    # rust/tests/iga_kernel.rs:119-151 (p = 2 only, to keep the CPU suite fast)
    lam, mu = O.lame(1.0, 0.3)
    p = 2
    errs = []
    for nel in (4, 8, 16):
        sp = O.Space([[0, 1], [0, 1]], [nel, nel], p)
        types, tid, _ = sp.element_matrices(lam, mu)
        k = O.Csr.assemble(sp, types, tid, None, pattern=False)
        f = sp.load_vector(1, (lam, mu))
        fixed = _all_boundary(sp)
        u = _solve_dirichlet(k, sp, f, fixed, np.zeros(sp.ndof))
        errs.append(sp.mms_l2_error(u))
    rate = np.log2(errs[1] / errs[2])
    assert rate > p + 1 - 0.25, (errs, rate)
