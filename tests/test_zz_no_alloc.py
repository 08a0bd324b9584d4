"""The allocation-free apply, icc_apply_f64_noalloc.

It serves callers that may not allocate device memory themselves: applications that hand the
library buffers from their own device pool and forbid cudaMalloc/cudaFree, and loops that must
not allocate after start-up.  Its only scratch is a fixed array inside the library.  This test
gives it caller-owned buffers (allocated here by torch, standing in for the application's pool)
and checks it against the handle-based apply, twice in a row, because every call reuses the
shared array.  The file name keeps it last in collection order.
"""
import numpy as np
import pytest

import immersed_catmull_clark_b200 as icc

pytestmark = pytest.mark.gpu

APPLY_TOL = 1e-12  # the FP64 apply parity bar used by the other GPU tests


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("nsub", [[24, 16, 12], [9, 5, 6]])
def test_noalloc_apply_matches_handle_apply(nsub):
    import torch
    dev = torch.device("cuda", 0)
    bounds = [[0.0, 2.0], [0.0, 1.0], [0.0, 1.0]]
    sp = icc.SpaceBox(bounds, nsub, 2)
    lam, mu = icc.lame(1.0, 0.3)
    em = icc.elasticity_element_matrices(sp, lam, mu)
    rng = np.random.default_rng(17)
    scale = rng.uniform(0.01, 1.0, sp.nel) ** 3
    op = icc.MatrixFreeOperator(sp, em, scale)
    ke = torch.from_numpy(np.ascontiguousarray(em.types).reshape(-1)).to(dev)
    tid = torch.from_numpy(em.type_id).to(dev)
    s = torch.from_numpy(scale).to(dev)
    y_ref = torch.empty(sp.ndof, dtype=torch.float64, device=dev)
    y = torch.empty_like(y_ref)
    for call in range(2):
        x = torch.from_numpy(rng.standard_normal(sp.ndof)).to(dev)
        op.matvec_dev(x.data_ptr(), y_ref.data_ptr())
        torch.cuda.synchronize()
        icc.apply_f64_noalloc(sp.nel_dir, ke.data_ptr(), len(em.types), tid.data_ptr(), s.data_ptr(),
                              x.data_ptr(), y.data_ptr())
        torch.cuda.synchronize()
        err = _rel(y.cpu().numpy(), y_ref.cpu().numpy())
        assert err < APPLY_TOL, (call, err)


def test_noalloc_unit_scale_and_untyped_elements():
    # scale = NULL means s_e = 1 (a handle built without a scale); type ids outside [0, ntypes)
    # contribute nothing (a handle whose scale is 0 on those elements); and once the array's
    # address is resolved, a call leaves the device's free memory unchanged
    import torch
    dev = torch.device("cuda", 0)
    nsub = [17, 9, 6]
    sp = icc.SpaceBox([[0.0, 2.0], [0.0, 1.0], [0.0, 1.0]], nsub, 2)
    lam, mu = icc.lame(1.0, 0.3)
    em = icc.elasticity_element_matrices(sp, lam, mu)
    rng = np.random.default_rng(23)
    ke = torch.from_numpy(np.ascontiguousarray(em.types).reshape(-1)).to(dev)
    tid = torch.from_numpy(em.type_id).to(dev)
    x = torch.from_numpy(rng.standard_normal(sp.ndof)).to(dev)
    y = torch.empty_like(x)
    y_ref = torch.empty_like(x)
    unit = icc.MatrixFreeOperator(sp, em)
    unit.matvec_dev(x.data_ptr(), y_ref.data_ptr())
    torch.cuda.synchronize()
    icc.apply_f64_noalloc(sp.nel_dir, ke.data_ptr(), len(em.types), tid.data_ptr(), 0, x.data_ptr(), y.data_ptr())
    torch.cuda.synchronize()
    assert _rel(y.cpu().numpy(), y_ref.cpu().numpy()) < APPLY_TOL
    free0 = torch.cuda.mem_get_info(dev)[0]
    icc.apply_f64_noalloc(sp.nel_dir, ke.data_ptr(), len(em.types), tid.data_ptr(), 0, x.data_ptr(), y.data_ptr())
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(dev)[0] == free0
    # untyped elements
    ids = em.type_id.copy()
    off = rng.choice(sp.nel, size=sp.nel // 5, replace=False)
    ids[off[: len(off) // 2]] = -1
    ids[off[len(off) // 2:]] = len(em.types)
    scale = rng.uniform(0.01, 1.0, sp.nel)
    s0 = scale.copy()
    s0[off] = 0.0
    ref_op = icc.MatrixFreeOperator(sp, em, s0)
    ref_op.matvec_dev(x.data_ptr(), y_ref.data_ptr())
    s = torch.from_numpy(scale).to(dev)
    tid_bad = torch.from_numpy(ids).to(dev)
    torch.cuda.synchronize()
    icc.apply_f64_noalloc(sp.nel_dir, ke.data_ptr(), len(em.types), tid_bad.data_ptr(), s.data_ptr(), x.data_ptr(),
                          y.data_ptr())
    torch.cuda.synchronize()
    assert _rel(y.cpu().numpy(), y_ref.cpu().numpy()) < APPLY_TOL


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch
    dev = torch.device("cuda", 0)
    buf = torch.zeros(16, dtype=torch.float64, device=dev)
    ids = torch.zeros(16, dtype=torch.int32, device=dev)
    with pytest.raises(icc.IccError) as ei:
        icc.apply_f64_noalloc([128, 64, 64], buf.data_ptr(), 1, ids.data_ptr(), 0, buf.data_ptr(), buf.data_ptr())
    assert ei.value.code == icc.ICC_BAD_ARG
