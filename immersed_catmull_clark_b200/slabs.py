"""Multi-GPU forms of the Jacobi-PCG: the element grid cut into slabs along x, one per rank.

The reference has no distribution (rayon threads only).  The grid splits naturally along x: rank r
owns the elements [e0_r, e1_r) and the control points [e0_r, e1_r + 2) of them, so neighbouring
slabs share two control-point planes.  Every rank applies its slab's operator (the device operator
on the slab's window of the global space, icc_space_window: local numbering, the global B-splines
and element types), then the
partial sums on the two shared planes are exchanged with the neighbours and added: both ranks then
hold the full y = A x on those planes.  Dot products count each control point once (a shared plane
belongs to the lower rank) and are summed over ranks with one all-reduce for p'Ap and one for
(r'r, r'z) per iteration; the recurrence, its stopping rule and its breakdown rule are those of
rust/src/solver.rs:14-76.

The mixed-precision form (SlabMixedPcg) runs the same recurrence in FP32 on the tensor-core apply
of every slab, with the halo sum in FP32, every dot product in FP64, and FP64 residual
replacement across the slabs, as the single-GPU mixed solve does.

The local operator is any callable y = apply(x) on the slab's vectors (torch tensors on the
rank's device), so the same code runs the device operator over NCCL and, on CPU ranks over gloo,
any stand-in.
"""
from dataclasses import dataclass

import numpy as np
import torch
import torch.distributed as dist


def partition(nx, world):
    """Balanced contiguous element ranges along x: [(e0, e1)] per rank (every rank >= 1 element)."""
    if nx < world:
        raise ValueError(f"{nx} elements along x cannot be cut into {world} slabs")
    base, extra = divmod(nx, world)
    out, e = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((e, e + n))
        e += n
    return out


@dataclass
class Slab:
    """Rank `rank`'s part of a grid of nel = (nx, ny, nz) elements: elements [e0, e1) along x and
    the local control-point numbering (component-blocked, x fastest) of its e1 - e0 + 2 planes."""
    rank: int
    world: int
    nel: tuple
    e0: int
    e1: int

    @property
    def ncp(self):
        return (self.e1 - self.e0 + 2, self.nel[1] + 2, self.nel[2] + 2)

    @property
    def nsc(self):
        c = self.ncp
        return c[0] * c[1] * c[2]

    @property
    def ndof(self):
        return 3 * self.nsc

    def bounds(self, global_bounds):
        """Physical extent of the slab (the global box cut at element faces)."""
        gb = np.asarray(global_bounds, dtype=np.float64).reshape(3, 2)
        h = (gb[0, 1] - gb[0, 0]) / self.nel[0]
        b = gb.copy()
        b[0] = [gb[0, 0] + self.e0 * h, gb[0, 0] + self.e1 * h]
        return b

    def element_ids(self):
        """Global element indices of the slab's elements in local order (x fastest)."""
        nx, ny, nz = self.nel
        ex = np.arange(self.e0, self.e1)
        ey, ez = np.arange(ny), np.arange(nz)
        return (ex[None, None, :] + nx * (ey[None, :, None] + ny * ez[:, None, None])).reshape(-1)

    def dof_ids(self):
        """Global DOF index of every local DOF (component-blocked on both sides)."""
        gcx, gcy, gcz = self.nel[0] + 2, self.nel[1] + 2, self.nel[2] + 2
        gnsc = gcx * gcy * gcz
        cx, cy, cz = self.ncp
        ix = np.arange(self.e0, self.e0 + cx)
        iy, iz = np.arange(cy), np.arange(cz)
        sc = (ix[None, None, :] + gcx * (iy[None, :, None] + gcy * iz[:, None, None])).reshape(-1)
        return np.concatenate([c * gnsc + sc for c in range(3)])

    def owner_weight(self):
        """1 on the control points this rank counts in dot products, 0 on the two planes it shares
        with the next rank (which counts them)."""
        cx, cy, cz = self.ncp
        w = np.ones((3, cz, cy, cx))
        if self.rank < self.world - 1:
            w[:, :, :, cx - 2:] = 0.0
        return w.reshape(-1)


class HaloComm:
    """Sum of the shared control-point planes with the neighbouring ranks (point-to-point over
    the default process group)."""

    def __init__(self, slab, device):
        self.slab = slab
        cx, cy, cz = slab.ncp
        self.shape = (3, cz, cy, cx)
        self.device = device

    def sum(self, y):
        """y (local, flat) += the neighbours' partial sums on the shared planes, in place."""
        s = self.slab
        v = y.view(self.shape)
        ops, bufs = [], []
        if s.rank > 0:
            send_lo = v[:, :, :, 0:2].contiguous()
            recv_lo = torch.empty_like(send_lo)
            ops += [dist.P2POp(dist.isend, send_lo, s.rank - 1), dist.P2POp(dist.irecv, recv_lo, s.rank - 1)]
            bufs.append((0, recv_lo))
        if s.rank < s.world - 1:
            send_hi = v[:, :, :, -2:].contiguous()
            recv_hi = torch.empty_like(send_hi)
            ops += [dist.P2POp(dist.isend, send_hi, s.rank + 1), dist.P2POp(dist.irecv, recv_hi, s.rank + 1)]
            bufs.append((1, recv_hi))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for side, buf in bufs:
            if side == 0:
                v[:, :, :, 0:2] += buf
            else:
                v[:, :, :, -2:] += buf
        return y


class SlabPcg:
    """rust/src/solver.rs:9-76 PcgSolver over x-slabs: x starts at 0, Jacobi inv_diag = |d| > 1e-12
    ? 1/d : 1, stop when ||r|| / max(||b||, 1e-16) < tol, break when p'Ap <= 0.  `apply(x)` returns
    the slab's partial y = A_local x (mask rule included); the halo sum completes it."""

    def __init__(self, slab, apply, device):
        self.slab = slab
        self.apply = apply
        self.halo = HaloComm(slab, device)
        self.w = torch.from_numpy(slab.owner_weight()).to(device)

    def full_apply(self, x):
        return self.halo.sum(self.apply(x))

    def _allreduce(self, vals):
        t = torch.stack(vals)
        dist.all_reduce(t)
        return t

    def solve(self, b, diag, max_iter, tol):
        """b, diag: the slab's local vectors (diag complete on the shared planes).  Returns
        (x_local, iterations, rel_res, status) with status 'ok', 'max_iter' or 'breakdown'."""
        w = self.w
        inv = torch.where(diag.abs() > 1e-12, 1.0 / diag, torch.ones_like(diag))
        x = torch.zeros_like(b)
        r = b.clone()
        z = inv * r
        p = z.clone()
        rz, bb = self._allreduce([(w * r * z).sum(), (w * b * b).sum()])
        nb = max(float(bb.sqrt()), 1e-16)
        res = 1.0
        for it in range(1, max_iter + 1):
            ap = self.full_apply(p)
            pap = float(self._allreduce([(w * p * ap).sum()])[0])
            if not pap > 0.0:
                return x, it, res, "breakdown"
            alpha = float(rz) / pap
            x += alpha * p
            r -= alpha * ap
            z = inv * r
            rr, rz_new = self._allreduce([(w * r * r).sum(), (w * r * z).sum()])
            res = float(rr.sqrt()) / nb
            if res < tol:
                return x, it, res, "ok"
            beta = float(rz_new) / float(rz)
            rz = rz_new
            p = z + beta * p
        return x, max_iter, res, "max_iter"


class SlabMixedPcg(SlabPcg):
    """The mixed-precision form over x-slabs (reliable updates).  The FP32 recurrence x32, r32, p
    uses `apply32` (FP32 tensors in and out: the slab's tensor-core apply) and the halo sum in FP32;
    every dot product is accumulated in FP64 and summed over the ranks.  Whenever the FP32 residual
    has fallen by `delta` since the last replacement, or after `seg` iterations, or when it meets
    the tolerance, the FP32 solution is added to the FP64 solution, the FP64 true residual
    b - A x (`apply64` and the halo sum in FP64) replaces the FP32 residual, and the direction goes
    on with beta = r'z(true) / r'z(previous).  The solve stops on the FP64 true residual, with the
    reference's stopping rule ||r|| / max(||b||, 1e-16) < tol and its breakdown rule p'Ap <= 0
    (rust/src/solver.rs:38-71)."""

    def __init__(self, slab, apply64, apply32, device, delta=0.6, seg=512):
        super().__init__(slab, apply64, device)
        self.apply32 = apply32
        self.delta = delta
        self.seg = seg
        self.replacements = 0

    def _dot(self, pairs):
        """FP64 sums over the ranks of w * a * b for each (a, b) pair (FP32 or FP64 tensors)."""
        w = self.w
        return self._allreduce([(w * a.double() * b.double()).sum() for a, b in pairs])

    def solve(self, b, diag, max_iter, tol):
        """b, diag: the slab's local FP64 vectors (diag complete on the shared planes).  Returns
        (x_local, iterations, true rel_res, status) with status 'ok', 'max_iter' or 'breakdown';
        self.replacements counts the FP64 residual replacements."""
        inv64 = torch.where(diag.abs() > 1e-12, 1.0 / diag, torch.ones_like(diag))
        inv32 = inv64.float()
        x64 = torch.zeros_like(b)
        nb = max(float(self._dot([(b, b)])[0].sqrt()), 1e-16)
        r64 = b.clone()
        res_true = float(self._dot([(r64, r64)])[0].sqrt()) / nb
        self.replacements = 0
        if res_true < tol:
            return x64, 0, res_true, "ok"
        x32 = torch.zeros_like(b, dtype=torch.float32)
        r32 = r64.float()
        z = inv32 * r32
        p = z.clone()
        rz = float(self._dot([(r32, z)])[0])
        res_repl, it_repl = res_true, 0
        for it in range(1, max_iter + 1):
            ap = self.halo.sum(self.apply32(p))
            pap = float(self._dot([(p, ap)])[0])
            if not pap > 0.0:
                return x64 + x32.double(), it, res_true, "breakdown"
            alpha = rz / pap
            x32 += float(alpha) * p
            r32 -= float(alpha) * ap
            z = inv32 * r32
            rr, rz_new = self._dot([(r32, r32), (r32, z)])
            res32 = float(rr.sqrt()) / nb
            if res32 < self.delta * res_repl or it - it_repl >= self.seg or res32 < tol:
                # FP64 residual replacement
                x64 += x32.double()
                x32.zero_()
                r64 = b - self.full_apply(x64)
                res_true = float(self._dot([(r64, r64)])[0].sqrt()) / nb
                self.replacements += 1
                if res_true < tol:
                    return x64, it, res_true, "ok"
                r32 = r64.float()
                z = inv32 * r32
                rz_true = float(self._dot([(r32, z)])[0])
                beta = rz_true / rz
                rz = rz_true
                res_repl, it_repl = res_true, it
            else:
                beta = float(rz_new) / rz
                rz = float(rz_new)
            p = z + float(beta) * p
        return x64 + x32.double(), max_iter, res_true, "max_iter"


def device_apply(op):
    """The local apply of a slab's device operator (MatrixFreeOperator) on torch tensors."""
    def apply(x):
        y = torch.empty_like(x)
        torch.cuda.current_stream().synchronize()   # x is complete before the operator's stream reads it
        op.matvec_dev(x.data_ptr(), y.data_ptr())
        torch.cuda.ExternalStream(op.stream).synchronize()
        return y
    return apply


def device_apply_f32(op):
    """The local FP32 apply of a slab's device operator on the tensor cores (FP32 torch tensors)."""
    def apply(x):
        y = torch.empty_like(x)
        torch.cuda.current_stream().synchronize()
        op.matvec_f32_dev(x.data_ptr(), y.data_ptr())
        torch.cuda.ExternalStream(op.stream).synchronize()
        return y
    return apply


def slab_operator(icc, slab, global_bounds, em_global, scale_global, free_mask_global, mask_mode, space=None):
    """The device operator of a slab: the slab's window of the global space (local numbering, the
    global B-splines, so the operator also runs on the tensor cores next to a cut), the global
    element types restricted to the slab, the slab's element scales and mask.  `space` is the global
    SpaceBox (built from global_bounds and the slab's grid when not given)."""
    if space is None:
        space = icc.SpaceBox(global_bounds, slab.nel, 2)
    sp = space.window((slab.e0, 0, 0), (slab.e1, slab.nel[1], slab.nel[2]))
    eids = slab.element_ids()
    em = icc.ElementMatrices(em_global.types, np.ascontiguousarray(em_global.type_id[eids]))
    scale = None if scale_global is None else np.ascontiguousarray(scale_global[eids])
    fm = None if free_mask_global is None else np.ascontiguousarray(free_mask_global[slab.dof_ids()])
    return sp, icc.MatrixFreeOperator(sp, em, scale, fm, mask_mode)
