"""The x-slab forms of the PCG on two and three ranks (gloo, CPU): partitioning, the halo sum of the
two shared control-point planes and the distributed reductions, with the oracle's element loop as
each rank's local operator, against the single-domain oracle (rust/src/solver.rs:14-76 on the whole
grid).  The mixed-precision form runs its FP32 recurrence on the oracle's apply rounded to FP32
(input and output), with FP64 residual replacement across the slabs."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from immersed_catmull_clark_b200 import slabs as S
from immersed_catmull_clark_b200 import workloads as W


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, nel, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    os.environ["OMP_NUM_THREADS"] = "1"   # the ranks share the host's cores
    torch.set_num_threads(1)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle as O
        p = W.cantilever(nel, seed=5)
        gsp = O.Space(p.bounds, p.nel, 2)
        lam, mu = O.lame(1.0, 0.3)
        types, tid, _ = gsp.element_matrices(lam, mu)
        slab = S.Slab(rank, world, tuple(nel), *S.partition(nel[0], world)[rank])
        lsp = O.Space(slab.bounds(p.bounds), (slab.e1 - slab.e0, nel[1], nel[2]), 2)
        eids, dids = slab.element_ids(), slab.dof_ids()
        ltid, lscale, lmask = tid[eids], p.scale[eids], p.free_mask[dids]

        def apply(x):
            y = O.mf_apply(lsp, types, ltid, lscale, x.numpy(), lmask, 1)
            return torch.from_numpy(y)

        pcg = S.SlabPcg(slab, apply, torch.device("cpu"))
        # the distributed apply equals the global one on every local DOF
        xg = np.random.default_rng(3).standard_normal(gsp.ndof)
        yg = O.mf_apply(gsp, types, tid, p.scale, xg, p.free_mask, 1)
        yl = pcg.full_apply(torch.from_numpy(xg[dids].copy())).numpy()
        apply_err = float(np.abs(yl - yg[dids]).max() / np.abs(yg).max())
        # the solve
        b = W.rhs_masked(p)
        dg = np.maximum(O.mf_diagonal(gsp, types, tid, p.scale), 1e-12)
        dl = torch.from_numpy(O.mf_diagonal(lsp, types, ltid, lscale))
        pcg.halo.sum(dl)
        dl = torch.clamp(dl, min=1e-12)
        diag_err = float(np.abs(dl.numpy() - dg[dids]).max() / dg.max())
        x, it, res, status = pcg.solve(torch.from_numpy(b[dids].copy()), dl, 20 * gsp.ndof, 1e-10)
        xo, ito, reso = O.pcg_mf(gsp, types, tid, p.scale, b, dg, 20 * gsp.ndof, 1e-10, p.free_mask, 1)
        sol_err = float(np.linalg.norm(x.numpy() - xo[dids]) / np.linalg.norm(xo[dids]))
        q.put((rank, apply_err, diag_err, sol_err, it, ito, res, status))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,nel", [(2, (8, 3, 3)), (3, (7, 2, 2))])
def test_slab_pcg_matches_single_domain(world, nel):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, nel, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    out = [q.get(timeout=300) for _ in range(world)]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    for rank, apply_err, diag_err, sol_err, it, ito, res, status in out:
        assert apply_err < 1e-13, (rank, apply_err)
        assert diag_err < 1e-14, (rank, diag_err)
        assert status == "ok" and res < 1e-10
        assert abs(it - ito) <= 2, (it, ito)
        assert sol_err < 1e-8, (rank, sol_err)


def _rank_main_mixed(rank, world, port, nel, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    os.environ["OMP_NUM_THREADS"] = "1"
    torch.set_num_threads(1)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle as O
        p = W.cantilever(nel, seed=11)
        gsp = O.Space(p.bounds, p.nel, 2)
        lam, mu = O.lame(1.0, 0.3)
        types, tid, _ = gsp.element_matrices(lam, mu)
        slab = S.Slab(rank, world, tuple(nel), *S.partition(nel[0], world)[rank])
        lsp = O.Space(slab.bounds(p.bounds), (slab.e1 - slab.e0, nel[1], nel[2]), 2)
        eids, dids = slab.element_ids(), slab.dof_ids()
        ltid, lscale, lmask = tid[eids], p.scale[eids], p.free_mask[dids]

        def apply64(x):
            return torch.from_numpy(O.mf_apply(lsp, types, ltid, lscale, x.numpy(), lmask, 1))

        def apply32(x):
            y = O.mf_apply(lsp, types, ltid, lscale, x.numpy().astype(np.float64), lmask, 1)
            return torch.from_numpy(y.astype(np.float32))

        pcg = S.SlabMixedPcg(slab, apply64, apply32, torch.device("cpu"))
        b = W.rhs_masked(p)
        dg = np.maximum(O.mf_diagonal(gsp, types, tid, p.scale), 1e-12)
        dl = torch.from_numpy(O.mf_diagonal(lsp, types, ltid, lscale))
        pcg.halo.sum(dl)
        dl = torch.clamp(dl, min=1e-12)
        x, it, res, status = pcg.solve(torch.from_numpy(b[dids].copy()), dl, 20 * gsp.ndof, 1e-10)
        # the single-domain FP64 solution, tight
        xo, ito, _ = O.pcg_mf(gsp, types, tid, p.scale, b, dg, 40 * gsp.ndof, 1e-13, p.free_mask, 1)
        _, ito10, _ = O.pcg_mf(gsp, types, tid, p.scale, b, dg, 20 * gsp.ndof, 1e-10, p.free_mask, 1)
        sol_err = float(np.linalg.norm(x.numpy() - xo[dids]) / np.linalg.norm(xo[dids]))
        q.put((rank, sol_err, it, ito10, res, status, pcg.replacements))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,nel", [(2, (8, 3, 3)), (3, (9, 3, 2))])
def test_slab_mixed_pcg_matches_single_domain(world, nel):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main_mixed, args=(r, world, port, nel, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    out = [q.get(timeout=300) for _ in range(world)]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    for rank, sol_err, it, ito, res, status, repl in out:
        assert status == "ok" and res < 1e-10, (rank, status, res)
        assert sol_err < 1e-8, (rank, sol_err)
        assert repl >= 1
        # FP32 inner iterations with replacement stay near the FP64 count
        assert it <= 1.5 * ito + 10, (it, ito)
    # every rank stopped at the same iteration (the stopping test is global)
    assert len({o[2] for o in out}) == 1


def test_partition():
    assert S.partition(10, 3) == [(0, 4), (4, 7), (7, 10)]
    with pytest.raises(ValueError):
        S.partition(2, 3)
    s = S.Slab(1, 3, (10, 2, 2), 4, 7)
    assert s.ncp == (5, 4, 4) and s.owner_weight().sum() == 3 * 4 * 4 * 3
    assert s.dof_ids()[0] == 4
