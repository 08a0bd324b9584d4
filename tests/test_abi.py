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
