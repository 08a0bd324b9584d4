"""Host-side checks of the synthetic inputs (no GPU): the tip load cases of the multi-RHS topology
configuration and the reference cantilever load."""
import numpy as np

from immersed_catmull_clark_b200 import workloads as W


def _greville(n, length):
    kn = np.concatenate([[0.0, 0.0, 0.0], np.arange(1, n) / n, [1.0, 1.0, 1.0]])
    return length * (kn[1:-2] + kn[2:-1]) / 2.0


def test_tip_load_cases_resultants():
    nel = (8, 6, 5)
    size = (2.0, 1.0, 1.0)
    L = W.tip_load_cases(nel, size)
    cx, cy, cz = (n + 2 for n in nel)
    nsc = cx * cy * cz
    gy, gz = _greville(nel[1], size[1]), _greville(nel[2], size[2])
    Y = np.broadcast_to(gy[None, :, None], (cz, cy, cx)).reshape(-1)
    Z = np.broadcast_to(gz[:, None, None], (cz, cy, cx)).reshape(-1)
    totals = [[L[k, c * nsc:(c + 1) * nsc].sum() for c in range(3)] for k in range(4)]
    assert np.allclose(totals[0], [0, 1, 0]) and np.allclose(totals[1], [0, -1, 0])
    assert np.allclose(totals[2], [1, 0, 0]) and np.allclose(totals[3], [0, 0, 0], atol=1e-14)
    # quadratic B-splines reproduce linear functions at the Greville abscissae, so the consistent
    # loads carry the traction's moment exactly: the couple is 1 about the face's centre line
    fy, fz = L[3, nsc:2 * nsc], L[3, 2 * nsc:]
    moment = np.sum(fz * (Y - 0.5 * size[1]) - fy * (Z - 0.5 * size[2]))
    assert abs(moment - 1.0) < 1e-12
    # every load sits on the tip face x = size0 (ix = last)
    ix = np.arange(nsc) % cx
    for k in range(4):
        for c in range(3):
            assert np.all(L[k, c * nsc:(c + 1) * nsc][ix != cx - 1] == 0.0)


def test_reference_tip_load():
    # rust/src/topopt_iga.rs:78-97 for 8x4x2 elements: the points with i1 = last, i2 <= 2, |i3 - 2| <= 1
    f = W.reference_tip_load([8, 4, 2])
    nd = (10, 6, 4)
    nsc = nd[0] * nd[1] * nd[2]
    sel = np.nonzero(f)[0]
    assert np.all((sel >= nsc) & (sel < 2 * nsc))
    assert abs(f.sum() + 1.0) < 1e-15
    idx = sel - nsc
    assert np.all(idx % nd[0] == nd[0] - 1)
    assert np.all((idx // nd[0]) % nd[1] <= 1)
