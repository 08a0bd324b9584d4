"""Cut-cell stabilisation terms built by the library on the host (icc_ghost_penalty,
icc_legacy_stabilization) against the oracle's restatements of rust/src/immersed.rs:156-370, the
reference fixture's stabilisation norm (rust/tests/immersed_vs_matlab.rs:53-54), and the ghost
penalty's consistency on polynomials up to degree p (rust/tests/immersed_cad_bc.rs:63-97).  No GPU:
both builders are host code."""
import json
import os

import numpy as np
import pytest

import immersed_catmull_clark_b200 as icc
from oracle import oracle as O


def csr_dense(n, r, c, v):
    a = np.zeros((n, n))
    np.add.at(a, (r, c), v)
    return a


def tilted_box(golden_dir):
    with open(os.path.join(golden_dir, "immersed_tilted_box.json")) as f:
        d = json.load(f)
    gb = np.array(d["grid_bounds"]).reshape(3, 2)
    return d, gb


def test_legacy_matches_fixture_and_oracle(golden_dir):
    d, gb = tilted_box(golden_dir)
    st = np.array(d["status"], dtype=np.int8)
    sp = icc.SpaceBox(gb, d["grid_res"], 2)
    osp = O.Space(gb, d["grid_res"], 2)
    r, c, v = icc.legacy_stabilization(sp, st, d["gamma_gp"])
    ro, co, vo = O.legacy_stabilization(osp, st, d["gamma_gp"])
    assert np.array_equal(r, ro) and np.array_equal(c, co) and np.array_equal(v, vo)
    a = csr_dense(sp.ndof, r, c, v)
    fro = np.linalg.norm(a)
    assert abs(fro - d["kgp_frobenius"]) <= 1e-12 * max(d["kgp_frobenius"], 1.0)


@pytest.mark.parametrize("nsub,bounds,seed", [([7, 5, 6], ((0.0, 1.3), (-0.2, 0.7), (0.1, 0.6)), 1),
                                              ([12, 14, 10], ((0.0, 1.0), (0.0, 1.0), (0.0, 1.0)), 2),
                                              ([3, 2, 9], ((-1.0, 1.0), (0.0, 0.5), (0.0, 3.0)), 3)])
def test_ghost_penalty_matches_oracle(nsub, bounds, seed):
    sp = icc.SpaceBox(bounds, nsub, 2)
    osp = O.Space(bounds, nsub, 2)
    rng = np.random.default_rng(seed)
    st = rng.choice(np.array([1, 0, -1], dtype=np.int8), size=sp.nel, p=[0.4, 0.2, 0.4])
    r, c, v = icc.ghost_penalty(sp, st, 1e-2, 2.5)
    ro, co, vo = O.ghost_penalty(osp, st, 1e-2, 2.5)
    assert len(v) == len(vo)
    assert np.array_equal(r, ro) and np.array_equal(c, co)
    assert np.abs(v - vo).max() <= 1e-13 * np.abs(vo).max()


def poly_coeffs_1d(nel, lo, length, deg):
    """Control values of the 1-D spline that equals x^deg (deg <= 2, so it lies in the space):
    collocation at the Greville points, exact for any field of the space."""
    kn = O.open_knots(nel, 2, 1)
    n = nel + 2
    grev = np.array([(kn[i + 1] + kn[i + 2]) / 2.0 for i in range(n)])
    b = np.zeros((n, n))
    for i, xi in enumerate(grev):
        first, v, _ = O.basis_funs(kn, 2, xi)
        b[i, first:first + 3] = v
    return np.linalg.solve(b, (lo + length * grev) ** deg)


def test_ghost_penalty_consistency():
    # rust/tests/immersed_cad_bc.rs:63-97: j(u, v) vanishes on every component field that is a
    # polynomial of degree <= p = 2 in one direction, and penalises a rough field
    bounds = ((0.0, 1.3), (-0.2, 0.7), (0.1, 0.6))
    nsub = [6, 5, 4]
    sp = icc.SpaceBox(bounds, nsub, 2)
    st = -np.ones(sp.nel, dtype=np.int8)
    r, c, v = icc.ghost_penalty(sp, st, 1.0, 1.0)
    a = csr_dense(sp.ndof, r, c, v)
    norm = np.linalg.norm(a)
    assert norm > 0.0
    nsc = sp.ndof_sc
    idx = np.indices(sp.ndof_dir[::-1]).reshape(3, -1)[::-1]
    for d, deg in [(0, 1), (1, 2), (2, 2)]:
        cd = poly_coeffs_1d(nsub[d], bounds[d][0], bounds[d][1] - bounds[d][0], deg)
        u = np.zeros(sp.ndof)
        comp = (d + 1) % 3
        u[comp * nsc:(comp + 1) * nsc] = cd[idx[d]]
        assert np.linalg.norm(a @ u) < 1e-10 * norm * np.linalg.norm(u), (d, deg)
    # a cubic along x is penalised (its second derivative jumps are nonzero only if it is not in
    # the space; the control values of the quadratic interpolant plus a rough part are)
    rnd = ((np.arange(sp.ndof) * 7919) % 101) / 101.0
    assert np.linalg.norm(a @ rnd) > 0.0
