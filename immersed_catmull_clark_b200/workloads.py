"""Synthetic inputs of the benchmark configurations (numpy, seeded PCG64; the immersed volume
fractions come from the library's device kernel).

* cantilever(nel, smooth):  the SIMP cantilever on the box [0,2] x [0,1] x [0,1]: E0 = 1,
  E_min = 1e-9, nu = 0.3, SIMP penalty 3, densities i.i.d. U[0.01, 1] (optionally smoothed by a
  3x3x3 box filter with clamped indices), control points with ix = 0 clamped in all components,
  and the consistent load of a unit total downward traction spread uniformly over the face
  x = 2.  24x16x12 elements is the CPU-runnable case, 128x64x64 the at-scale case.
* cylinders(n):  the immersed case: unit cube minus three orthogonal through-cylinders of
  radius 0.25, per-cell volume fraction by 8^3 midpoint sub-sampling after corner
  classification (the rule of rust/src/immersed.rs:89-155 with an exact inside test), alpha <
  1e-3 inactive, alpha floored at 1e-6, clamped at z = 0, pressure 1 on the z = 1 face.

The element scale follows the reference: s_e = E_min + rho^p (E0 - E_min) (rust/src/topopt_iga.rs:132
with E0 folded into the Lame parameters); immersed cells use E_min + rho^p (E0 - E_min) alpha_e
(rust/src/immersed.rs:484, rust/src/topopt_immersed.rs:166) and inactive cells none.
"""
from dataclasses import dataclass

import numpy as np

E0, EMIN, NU, PENAL = 1.0, 1e-9, 0.3, 3.0


@dataclass
class Problem:
    name: str
    bounds: np.ndarray      # [3, 2]
    nel: tuple              # (nx, ny, nz)
    scale: np.ndarray       # [nel] float64, s_e
    free_mask: np.ndarray   # [ndof] uint8
    force: np.ndarray       # [ndof] float64
    density: np.ndarray     # [nel]
    alpha: np.ndarray = None  # [nel] volume fraction (immersed)

    @property
    def ncp(self):
        return tuple(n + 2 for n in self.nel)

    @property
    def ndof(self):
        cx, cy, cz = self.ncp
        return 3 * cx * cy * cz


def open_knot_integrals(nel, length):
    """int_0^L N_i for the p = 2 open uniform knot vector: L (k[i+3] - k[i]) / 3."""
    kn = np.concatenate([[0.0, 0.0, 0.0], np.arange(1, nel) / nel, [1.0, 1.0, 1.0]])
    return length * (kn[3:] - kn[:-3]) / 3.0


def box_filter_clamped(r):
    """3x3x3 mean with clamped (edge-replicated) indices; r has shape (nz, ny, nx)."""
    p = np.pad(r, 1, mode="edge")
    nz, ny, nx = r.shape
    acc = np.zeros_like(r)
    for dz in range(3):
        for dy in range(3):
            for dx in range(3):
                acc += p[dz:dz + nz, dy:dy + ny, dx:dx + nx]
    return acc / 27.0


def cantilever(nel=(24, 16, 12), smooth=False, seed=0, name=None):
    nx, ny, nz = nel
    bounds = np.array([[0.0, 2.0], [0.0, 1.0], [0.0, 1.0]])
    rng = np.random.default_rng(seed)
    rho = rng.uniform(0.01, 1.0, size=(nz, ny, nx))
    if smooth:
        rho = box_filter_clamped(rho)
    rho = rho.reshape(-1)
    scale = EMIN + rho ** PENAL * (E0 - EMIN)
    cx, cy, cz = nx + 2, ny + 2, nz + 2
    nsc = cx * cy * cz
    ix = np.arange(nsc) % cx
    free = np.ones(3 * nsc, dtype=np.uint8)
    for c in range(3):
        free[c * nsc:(c + 1) * nsc][ix == 0] = 0
    wy = open_knot_integrals(ny, bounds[1, 1] - bounds[1, 0])
    wz = open_knot_integrals(nz, bounds[2, 1] - bounds[2, 0])
    area = (bounds[1, 1] - bounds[1, 0]) * (bounds[2, 1] - bounds[2, 0])
    force = np.zeros(3 * nsc)
    face = np.zeros((cz, cy))
    face[:, :] = -(wz[:, None] * wy[None, :]) / area
    fz = force[2 * nsc:3 * nsc].reshape(cz, cy, cx)
    fz[:, :, cx - 1] = face
    return Problem(name or f"cantilever_{nx}x{ny}x{nz}", bounds, (nx, ny, nz), scale, free, force, rho)


def _cyl_inside(x, y, z, r):
    inside = (x >= 0) & (x <= 1) & (y >= 0) & (y <= 1) & (z >= 0) & (z <= 1)
    x, y, z = x - 0.5, y - 0.5, z - 0.5
    r2 = r * r
    hole = (y * y + z * z < r2) | (x * x + z * z < r2) | (x * x + y * y < r2)
    return inside & ~hole


def cylinder_fractions(n, sub=8, radius=0.25):
    """Per-cell volume fraction and status (1 inside, 0 outside, -1 cut) on an n^3 grid of [0,1]^3
    (rust/src/immersed.rs:88-155 rule), computed by the library's device kernel."""
    from . import cylinder_weights
    return cylinder_weights((n, n, n), (sub, sub, sub), radius)


def cylinders(n=96, sub=8, radius=0.25, name=None):
    bounds = np.array([[0.0, 1.0], [0.0, 1.0], [0.0, 1.0]])
    alpha, _ = cylinder_fractions(n, sub, radius)
    alpha = alpha.astype(np.float32).astype(np.float64)   # stored in FP32
    active = alpha >= 1e-3
    a = np.where(active, np.maximum(alpha, 1e-6), 0.0)
    # s_e = E_min + rho^p (E0 - E_min) alpha_e on active cells (density 1), no stiffness elsewhere
    scale = np.where(active, EMIN + (E0 - EMIN) * a, 0.0)
    cx = cy = cz = n + 2
    nsc = cx * cy * cz
    # control points touched by no active cell carry no stiffness: mask them out
    act = active.reshape(n, n, n)
    touched = np.zeros((cz, cy, cx), dtype=bool)
    for dz in range(3):
        for dy in range(3):
            for dx in range(3):
                touched[dz:dz + n, dy:dy + n, dx:dx + n] |= act
    iz = np.arange(nsc) // (cx * cy)
    free_sc = touched.reshape(-1) & (iz != 0)
    free = np.tile(free_sc.astype(np.uint8), 3)
    # consistent pressure load on the solid part of z = 1: -int_{top face, solid} N_i dA
    w1 = open_knot_integrals(n, 1.0)
    top = alpha.reshape(n, n, n)[n - 1] > 0  # cells of the top layer with material
    # per-cell exact integral of N_ix N_iy over a cell: use 3-point Gauss per cell
    force = np.zeros(3 * nsc)
    fz = force[2 * nsc:].reshape(cz, cy, cx)
    gx, gw = np.polynomial.legendre.leggauss(3)
    kn = np.concatenate([[0.0, 0.0, 0.0], np.arange(1, n) / n, [1.0, 1.0, 1.0]])
    def basis(e, t):
        # the three nonzero quadratic B-splines on element e at local t in [0,1]
        x = (e + t) / n
        vals = np.zeros(3)
        for r in range(3):
            i = e + r
            vals[r] = _bspline2(kn, i, x)
        return vals
    sub_pts = 8
    soff = (np.arange(sub_pts) + 0.5) / sub_pts
    for j in range(n):
        for i in range(n):
            if not top[j, i]:
                continue
            # fraction of the top face of the cell covered by solid, by sub-sampling at z = 1
            xs_ = (i + soff) / n
            ys_ = (j + soff) / n
            YY, XX = np.meshgrid(ys_, xs_, indexing="ij")
            solid = _cyl_inside(XX, YY, np.full_like(XX, 1.0 - 1e-12), radius)
            if not solid.any():
                continue
            bx = np.stack([basis(i, t) for t in soff])  # [sub, 3]
            by = np.stack([basis(j, t) for t in soff])
            wgt = solid.astype(float) * (1.0 / n / sub_pts) ** 2
            contrib = np.einsum("yx,ya,xb->ab", wgt, by, bx)  # [3 (y), 3 (x)]
            fz[cz - 1, j:j + 3, i:i + 3] -= contrib
    del w1, gx, gw
    rho = np.ones(n ** 3)
    return Problem(name or f"cylinders_{n}", bounds, (n, n, n), scale, free, force * free, rho, alpha)


def _bspline2(kn, i, x):
    """Quadratic B-spline N_i(x) on knots kn (Cox-de Boor), right end included in the last span."""
    def n0(j, x):
        if kn[j] <= x < kn[j + 1]:
            return 1.0
        if x == kn[-1] and kn[j] < kn[j + 1] == kn[-1]:
            return 1.0
        return 0.0

    def nk(j, k, x):
        if k == 0:
            return n0(j, x)
        a = 0.0
        d1 = kn[j + k] - kn[j]
        if d1 > 0:
            a += (x - kn[j]) / d1 * nk(j, k - 1, x)
        d2 = kn[j + k + 1] - kn[j + 1]
        if d2 > 0:
            a += (kn[j + k + 1] - x) / d2 * nk(j + 1, k - 1, x)
        return a

    return nk(i, 2, x)


def rhs_masked(p: Problem):
    return np.where(p.free_mask > 0, p.force, 0.0)


def _first_moments(nel, length, x0):
    """int_0^L N_i(x) (x - x0) dx for the p = 2 open uniform basis (3-point Gauss per element)."""
    kn = np.concatenate([[0.0, 0.0, 0.0], np.arange(1, nel) / nel, [1.0, 1.0, 1.0]])
    gx, gw = np.polynomial.legendre.leggauss(3)
    m = np.zeros(nel + 2)
    h = 1.0 / nel
    for e in range(nel):
        for t, w in zip(gx, gw):
            u = (e + 0.5 * (t + 1.0)) * h            # parameter in [0, 1]
            for r in range(3):
                m[e + r] += w * 0.5 * h * length * _bspline2(kn, e + r, u) * (u * length - x0)
    return m


def tip_load_cases(nel, size=(2.0, 1.0, 1.0)):
    """Four consistent load cases on the tip face x = size0 of the clamped cantilever box: shear +y,
    shear -y and axial +x (unit total force each, uniform traction) and a torsion couple about the
    face's centre line (traction tau (0, -(z - zc), y - yc) with unit moment).  [4, ndof]."""
    nx, ny, nz = nel
    cx, cy, cz = nx + 2, ny + 2, nz + 2
    nsc = cx * cy * cz
    iy, iz = open_knot_integrals(ny, size[1]), open_knot_integrals(nz, size[2])
    my, mz = _first_moments(ny, size[1], 0.5 * size[1]), _first_moments(nz, size[2], 0.5 * size[2])
    area = size[1] * size[2]
    polar = area * (size[1] ** 2 + size[2] ** 2) / 12.0     # int (y - yc)^2 + (z - zc)^2 dA
    tau = 1.0 / polar
    loads = np.zeros((4, 3 * nsc))
    for k, (comp, val) in enumerate([(1, 1.0), (1, -1.0), (0, 1.0)]):
        f = loads[k, comp * nsc:(comp + 1) * nsc].reshape(cz, cy, cx)
        f[:, :, cx - 1] = val / area * np.outer(iz, iy)
    fy = loads[3, nsc:2 * nsc].reshape(cz, cy, cx)
    fz = loads[3, 2 * nsc:].reshape(cz, cy, cx)
    fy[:, :, cx - 1] = -tau * np.outer(mz, iy)
    fz[:, :, cx - 1] = tau * np.outer(iz, my)
    return loads


def reference_tip_load(nel):
    """The reference cantilever's load (rust/src/topopt_iga.rs:78-97): -1/count in y on the control
    points with i1 = last, |i2 - 1| <= 1, |i3 - ncp3/2| <= 1 (1-based)."""
    nd = [n + 2 for n in nel]
    nsc = nd[0] * nd[1] * nd[2]
    idx = np.arange(nsc)
    s0, s1, s2 = idx % nd[0], (idx // nd[0]) % nd[1], idx // (nd[0] * nd[1])
    sel = (s0 + 1 == nd[0]) & (np.abs(s1 + 1.0 - 1.0) <= 1.0) & (np.abs(s2 + 1.0 - nd[2] / 2.0) <= 1.0)
    f = np.zeros(3 * nsc)
    f[nsc + idx[sel]] = -1.0 / sel.sum()
    return f


def batched_designs(count=64, kmin=8, kmax=48, seed=2026):
    """The batched-designs configuration: `count` cantilever designs of 2k x k x k elements with
    k ~ U{kmin..kmax} drawn from the seed, design i with its own densities (seed + 1 + i).
    Returns (ks, problems)."""
    rng = np.random.default_rng(seed)
    ks = rng.integers(kmin, kmax + 1, size=count)
    return ks, [cantilever((2 * int(k), int(k), int(k)), seed=seed + 1 + i) for i, k in enumerate(ks)]
