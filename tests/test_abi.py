"""C-ABI checks that need no GPU: the library loads, exports every symbol include/icc.h declares,
its host-side set-up (numbering, element matrices) matches the oracle and the reference's golden
fixture, and device entry points fail loudly instead of falling back to the CPU."""
import ctypes as C
import json
import os
import re

import numpy as np
import pytest

import immersed_catmull_clark_b200 as icc
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_header_symbols_are_exported():
    header = open(os.path.join(ROOT, "include", "icc.h")).read()
    declared = set(re.findall(r"\b(icc_[a-z_0-9]+)\s*\(", header))
    assert declared == set(icc.EXPORTED)
    L = C.CDLL(icc.LIB_PATH)
    for name in declared:
        assert hasattr(L, name), name


def test_lame_matches_reference_formula():
    lam, mu = icc.lame(1.0, 0.3)
    assert (lam, mu) == O.lame(1.0, 0.3)


def test_space_numbering_matches_fixture(golden_dir):
    with open(os.path.join(golden_dir, "iga_kernel.json")) as f:
        d = json.load(f)
    case = d["cases"][4]  # 3-D, p = 2 (rust/tests/iga_vs_matlab.rs:38-43)
    sp = icc.SpaceBox(np.array(case["bounds"], dtype=float), case["nsub"], 2)
    assert sp.ndof == case["ndof"]
    assert np.array_equal(sp.connectivity(), np.array(case["connectivity"]))
    em = icc.elasticity_element_matrices(sp, d["lambda"], d["mu"])
    assert len(em.types) == case["ntypes"]


@pytest.mark.parametrize("nsub", [[4, 3, 3], [1, 1, 1], [2, 3, 4], [5, 6, 7], [24, 16, 12], [9, 2, 5]])
def test_element_matrices_bit_identical_to_oracle(nsub):
    bounds = [[0.0, 2.0], [0.0, 1.0], [0.0, 1.0]]
    sp = icc.SpaceBox(bounds, nsub, 2)
    osp = O.Space(bounds, nsub, 2)
    lam, mu = icc.lame(1.0, 0.3)
    em = icc.elasticity_element_matrices(sp, lam, mu)
    otypes, otid, _ = osp.element_matrices(lam, mu)
    assert np.array_equal(sp.connectivity(), osp.connectivity())
    assert np.array_equal(em.type_id, otid)
    assert np.array_equal(em.types, otypes)  # same arithmetic order: bitwise equal


def test_bad_arguments_rejected():
    with pytest.raises(icc.IccError):
        icc.SpaceBox([[0, 1], [0, 1], [0, 1]], [2, 2, 2], 3)
    with pytest.raises(icc.IccError):
        icc.SpaceBox([[0, 1], [0, 1], [0, 1]], [0, 2, 2], 2)


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device error path")
def test_operator_fails_loudly_without_device():
    sp = icc.SpaceBox([[0, 1], [0, 1], [0, 1]], [2, 2, 2], 2)
    lam, mu = icc.lame(1.0, 0.3)
    with pytest.raises(icc.IccError) as ei:
        icc.MatrixFreeOperator(sp, (lam, mu))
    assert ei.value.code in (icc.ICC_NO_DEVICE, icc.ICC_CUDA_ERROR)


@pytest.mark.parametrize("e0,e1", [((0, 0, 0), (3, 4, 2)), ((2, 1, 0), (7, 4, 3)), ((4, 0, 1), (9, 4, 3))])
def test_space_window_keeps_parent_matrices(e0, e1):
    # a window of the space (the local space of a slab) has the parent's element matrices, also next
    # to a cut inside the grid, and its local numbering covers the parent's control points [e0, e1 + 2)
    sp = icc.SpaceBox(np.array([[0.0, 1.8], [0.0, 0.8], [0.0, 0.6]]), (9, 4, 3), 2)
    lam, mu = icc.lame(1.0, 0.3)
    em = icc.elasticity_element_matrices(sp, lam, mu)
    w = sp.window(e0, e1)
    assert w.nel_dir == [b - a for a, b in zip(e0, e1)]
    assert w.ndof_dir == [b - a + 2 for a, b in zip(e0, e1)]
    ew = icc.elasticity_element_matrices(w, lam, mu)
    nx, ny, _ = sp.nel_dir
    for ez in range(e0[2], e1[2]):
        for ey in range(e0[1], e1[1]):
            for ex in range(e0[0], e1[0]):
                g = ex + nx * (ey + ny * ez)
                l = (ex - e0[0]) + w.nel_dir[0] * ((ey - e0[1]) + w.nel_dir[1] * (ez - e0[2]))
                assert np.array_equal(ew.types[ew.type_id[l]], em.types[em.type_id[g]])
    with pytest.raises(icc.IccError):
        sp.window((0, 0, 0), (10, 4, 3))
