"""Seeded synthetic cases: grids, block layouts, connectivity and initial states.

A ``Case`` is target-independent: ``apply(target)`` replays it on anything
with the Solver call surface (add_block / set_boundary / connect /
set_state), so the GPU product and the CPU oracle see bit-identical inputs.

Families (the configurations the reference is measured on; the reference
itself only hard-codes the 2D Riemann problem, class_flow_field.f90:207-243):
  * riemann2d          four-quadrant 2D Riemann problem, nodal-centred grid
                       of method_gridgen.f90:84-136 (dx = L/(n-1)), quadrant
                       states drawn from a seed, transmissive boundaries
  * riemann2d_reference the exact hard-coded reference IC (x_mid=y_mid=0.8)
  * isentropic_vortex  3D Euler vortex in a periodic box [-5,5]^3, one block
                       or the 8 uneven blocks of VORTEX_BLOCKS_128
  * taylor_green       3D Navier-Stokes TGV on [0,2pi)^3, periodic
  * blast / shock_tube seeded 3D Euler cases of the batched configuration
All states are conservative (rho, rho*u, rho*v, rho*w, rho*E) in the
(5, nk, nj, ni) layout (Fortran (ni,nj,nk,5)).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import abi

GAMMA = 1.4


def prim_to_cons(rho, u, v, w, p, gamma=GAMMA):
    """convert_p_to_q_blk_sub (class_flow_field.f90:353-377), same rounding order."""
    q = np.empty((5,) + np.shape(rho), dtype=np.float64)
    q[0] = rho
    q[1] = rho * u
    q[2] = rho * v
    q[3] = rho * w
    q[4] = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
    return q


def cons_to_prim(q, gamma=GAMMA):
    rho = q[0]
    u = q[1] / rho
    v = q[2] / rho
    w = q[3] / rho
    p = (gamma - 1.0) * (q[4] - 0.5 * rho * (u * u + v * v + w * w))
    return np.stack([rho, u, v, w, p])


@dataclass
class Case:
    name: str
    cfg: dict
    blocks: list = field(default_factory=list)      # [(nvert(3), dr(3))]
    bcs: list = field(default_factory=list)         # [(blk, region, kind)]
    conns: list = field(default_factory=list)       # [(blk, range, donor, drange, dtype)]
    states: list = field(default_factory=list)      # [(5,nk,nj,ni)]
    origins: list = field(default_factory=list)     # global index of each block's cell (0,0,0)
    meta: dict = field(default_factory=dict)

    @property
    def ncells(self) -> int:
        return int(sum(n[0] * n[1] * n[2] for n, _ in self.blocks))

    def config(self, **over) -> abi.FvmConfig:
        d = dict(self.cfg)
        d.update(over)
        return abi.make_config(**d)

    def apply(self, target, states: bool = True, case_id: int | None = None):
        """Replay the case on `target`. With case_id, the blocks go to that
        case of a multi-case Solver and the engine's block ids are kept in
        self.block_ids (local block b -> engine block id)."""
        ids = []
        for n, dr in self.blocks:
            ids.append(target.add_block(n, dr) if case_id is None else target.add_case_block(case_id, n, dr))
        self.block_ids = ids
        for blk, region, kind in self.bcs:
            target.set_boundary(ids[blk], region, kind)
        for blk, rng, donor, drng, dtype in self.conns:
            target.connect(ids[blk], rng, ids[donor], drng, dtype)
        if states:
            self.apply_states(target)
        return target

    def apply_states(self, target):
        """Upload the initial states to the blocks apply() created."""
        for b, q in enumerate(self.states):
            target.set_state(self.block_ids[b], q)
        return target


# ---------------------------------------------------------------- 2D Riemann
def _quadrant_fill(x, y, xm, ym, states):
    """init_value_sub (defs_block_data.f90:166-201): regions 1..4 in order,
    inclusive bounds, later regions overwrite earlier ones."""
    shape = np.broadcast(x, y).shape
    out = [np.zeros(shape) for _ in range(5)]
    regions = [((xm, 1.0), (ym, 1.0)), ((0.0, xm), (ym, 1.0)), ((0.0, xm), (0.0, ym)), ((xm, 1.0), (0.0, ym))]
    for (x0, x1), (y0, y1), st in zip([r[0] for r in regions], [r[1] for r in regions], states):
        m = (x >= x0) & (x <= x1) & (y >= y0) & (y <= y1)
        for k in range(5):
            out[k] = np.where(m, st[k], out[k])
    return out


def riemann2d(n: int = 256, seed: int = 0, nk: int = 1, split: float = 0.5, **cfg) -> Case:
    """Four-quadrant Riemann problem on n x n nodes of [0,1]^2 (dx = 1/(n-1)).
    Quadrant (rho,u,v,p): rho~U[0.5,1.5], p~U[0.3,1.5], u,v~U[-0.5,0.5]."""
    rng = np.random.default_rng(seed)
    states = []
    for _ in range(4):
        rho = rng.uniform(0.5, 1.5)
        u = rng.uniform(-0.5, 0.5)
        v = rng.uniform(-0.5, 0.5)
        p = rng.uniform(0.3, 1.5)
        states.append((rho, u, v, 0.0, p))
    dx = 1.0 / (n - 1)
    x = dx * np.arange(n, dtype=np.float64)
    X, Y = np.meshgrid(x, x, indexing="xy")  # (nj, ni)
    rho, u, v, w, p = _quadrant_fill(X, Y, split, split, states)
    q = prim_to_cons(rho, u, v, w, p)
    q = np.broadcast_to(q[:, None, :, :], (5, nk, n, n)).copy()
    base = dict(idimension=2, reconstruct=abi.RECON_MUSCL, limiter=abi.LIMITER_MINMOD, kappa=1.0 / 3.0,
                flux_split=abi.FLUX_ROE, entropy_fix=0.2, rk_stages=3)
    base.update(cfg)
    c = Case(name=f"riemann2d_{n}", cfg=base, meta={"quadrants": states, "dx": dx})
    c.blocks.append(((n, n, nk), (dx, dx, 1.0)))
    c.states.append(q)
    c.origins.append((0, 0, 0))
    return c


def riemann2d_reference(n: int = 21, nk: int = 2, **cfg) -> Case:
    """The IC hard-coded in class_flow_field.f90:207-243 on the grid of
    case/Riemann-2D.nml (gridSize 21,21; square 1.0; 2D => nk = 2)."""
    states = [(1.5, 0.0, 0.0, 0.0, 1.5), (0.5323, 1.206, 0.0, 0.0, 0.3), (0.138, 1.206, 1.206, 0.0, 0.029),
              (0.5323, 0.0, 1.206, 0.0, 0.3)]
    dx = 1.0 / (n - 1)
    x = dx * np.arange(n, dtype=np.float64)
    X, Y = np.meshgrid(x, x, indexing="xy")
    rho, u, v, w, p = _quadrant_fill(X, Y, 0.8, 0.8, states)
    q = prim_to_cons(rho, u, v, w, p)
    q = np.broadcast_to(q[:, None, :, :], (5, nk, n, n)).copy()
    base = dict(idimension=2, reconstruct=abi.RECON_MUSCL, limiter=abi.LIMITER_MINMOD, kappa=0.33333,
                flux_split=abi.FLUX_ROE, entropy_fix=0.2, rk_stages=3, timestep_set=abi.DT_FIXED, dt=2.0e-4)
    base.update(cfg)
    c = Case(name="riemann2d_reference", cfg=base)
    c.blocks.append(((n, n, nk), (dx, dx, 1.0)))
    c.states.append(q)
    c.origins.append((0, 0, 0))
    return c


# ---------------------------------------------------------------- periodic boxes
def periodic_box_connections(N, boxes, periodic=(True, True, True)):
    """Connections for blocks tiling a box of N[0] x N[1] x N[2] cells.

    boxes: [(lo(3), hi(3))] global cell ranges (hi exclusive). Every face ghost
    cell (3 layers, tangential real range) is mapped to the block holding the
    global cell it stands for, wrapped across periodic axes. Returns the
    connection tuples and the (blk, region, TRANSMISSIVE) list for
    non-periodic outer faces."""
    conns, bcs = [], []
    for b, (lo, hi) in enumerate(boxes):
        n = [hi[a] - lo[a] for a in range(3)]
        for a in range(3):
            t = [d for d in range(3) if d != a]
            for side in (0, 1):
                region = 2 * a + side + 1
                layers = []  # (local normal index, wrapped global normal index)
                for g in (1, 2, 3):
                    gl = lo[a] - g if side == 0 else hi[a] - 1 + g
                    loc = -g if side == 0 else n[a] - 1 + g
                    if gl < 0 or gl >= N[a]:
                        if not periodic[a]:
                            layers = None
                            break
                        gl %= N[a]
                    layers.append((loc, gl))
                if layers is None:
                    bcs.append((b, region, abi.BC_TRANSMISSIVE))
                    continue
                layers.sort()
                for d, (dlo, dhi) in enumerate(boxes):
                    o1 = (max(lo[t[0]], dlo[t[0]]), min(hi[t[0]], dhi[t[0]]))
                    o2 = (max(lo[t[1]], dlo[t[1]]), min(hi[t[1]], dhi[t[1]]))
                    if o1[0] >= o1[1] or o2[0] >= o2[1]:
                        continue
                    inside = [(loc, gl) for loc, gl in layers if dlo[a] <= gl < dhi[a]]
                    # group consecutive layers with contiguous donor coordinates
                    groups = []
                    for loc, gl in inside:
                        if groups and groups[-1][-1][0] == loc - 1 and groups[-1][-1][1] == gl - 1:
                            groups[-1].append((loc, gl))
                        else:
                            groups.append([(loc, gl)])
                    for grp in groups:
                        rng = [None, None, None]
                        drng = [None, None, None]
                        rng[a] = (grp[0][0], grp[-1][0])
                        drng[a] = (grp[0][1] - dlo[a], grp[-1][1] - dlo[a])
                        for tt, ov in zip(t, (o1, o2)):
                            rng[tt] = (ov[0] - lo[tt], ov[1] - 1 - lo[tt])
                            drng[tt] = (ov[0] - dlo[tt], ov[1] - 1 - dlo[tt])
                        conns.append((b, tuple(rng), d, tuple(drng), (1, 2, 3)))
    return conns, bcs


# 8 uneven blocks tiling 128^3 with non-conforming interfaces: the x = 64
# plane splits the left half at y = 64 then z = 64 / z = 48 and the right
# half at z = 64 then y = 80 / y = 48.
def vortex_blocks(N: int = 128):
    h = N // 2
    f = lambda v: v * N // 128  # noqa: E731
    return [
        ((0, 0, 0), (h, h, h)),
        ((0, 0, h), (h, h, N)),
        ((0, h, 0), (h, N, f(48))),
        ((0, h, f(48)), (h, N, N)),
        ((h, 0, 0), (N, f(80), h)),
        ((h, f(80), 0), (N, N, h)),
        ((h, 0, h), (N, f(48), N)),
        ((h, f(48), h), (N, N, N)),
    ]


def vortex_fields(x, y, z, t=0.0, beta=5.0, gamma=GAMMA, L=10.0, uinf=(1.0, 1.0, 1.0)):
    """Isentropic vortex (axis along z) advected by uinf for time t in a
    periodic box of side L centred on 0 (nearest periodic image)."""
    xb = x - uinf[0] * t
    yb = y - uinf[1] * t
    xb = (xb + L / 2) % L - L / 2
    yb = (yb + L / 2) % L - L / 2
    r2 = xb * xb + yb * yb
    e = np.exp(0.5 * (1.0 - r2))
    du = -beta / (2 * math.pi) * e * yb
    dv = beta / (2 * math.pi) * e * xb
    dT = -(gamma - 1.0) * beta * beta / (8.0 * gamma * math.pi * math.pi) * e * e
    T = 1.0 + dT
    rho = T ** (1.0 / (gamma - 1.0))
    p = rho * T
    u = uinf[0] + du
    v = uinf[1] + dv
    w = uinf[2] + 0.0 * x
    return rho, u, v, w, p


def isentropic_vortex(N: int = 128, layout: str = "blocks8", beta: float = 5.0, **cfg) -> Case:
    """3D Euler isentropic vortex on the periodic box [-5,5]^3 with N^3 cells
    (cell centres), as one block or the 8 uneven blocks of vortex_blocks()."""
    L = 10.0
    dx = L / N
    boxes = vortex_blocks(N) if layout == "blocks8" else [((0, 0, 0), (N, N, N))]
    base = dict(idimension=3, reconstruct=abi.RECON_WENO, flux_split=abi.FLUX_AUSM, rk_stages=4,
                timestep_set=abi.DT_CFL, cfl=0.5)
    base.update(cfg)
    c = Case(name=f"vortex_{layout}_{N}", cfg=base, meta={"beta": beta, "L": L, "N": N, "dx": dx, "boxes": boxes})
    conns, bcs = periodic_box_connections((N, N, N), boxes)
    for lo, hi in boxes:
        n = tuple(hi[a] - lo[a] for a in range(3))
        c.blocks.append((n, (dx, dx, dx)))
        c.origins.append(lo)
        xs = [-L / 2 + (np.arange(lo[a], hi[a], dtype=np.float64) + 0.5) * dx for a in range(3)]
        Z, Y, X = np.meshgrid(xs[2], xs[1], xs[0], indexing="ij")
        c.states.append(prim_to_cons(*vortex_fields(X, Y, Z, 0.0, beta)))
    c.conns = conns
    c.bcs = []
    return c


def vortex_exact(case: Case, t: float):
    """Exact conservative state of each block of an isentropic_vortex case at time t."""
    L, dx, beta = case.meta["L"], case.meta["dx"], case.meta["beta"]
    out = []
    for (lo, hi) in case.meta["boxes"]:
        xs = [-L / 2 + (np.arange(lo[a], hi[a], dtype=np.float64) + 0.5) * dx for a in range(3)]
        Z, Y, X = np.meshgrid(xs[2], xs[1], xs[0], indexing="ij")
        out.append(prim_to_cons(*vortex_fields(X, Y, Z, t, beta)))
    return out


# ---------------------------------------------------------------- Taylor-Green
def taylor_green(N: int = 128, Ma: float = 0.1, Re: float = 1600.0, Pr: float = 0.71, **cfg) -> Case:
    """Compressible Taylor-Green vortex on [0,2pi)^3, rho0 = V0 = L = 1,
    p0 = 1/(gamma Ma^2), mu = 1/Re, periodic on all faces."""
    dx = 2 * math.pi / N
    xs = (np.arange(N, dtype=np.float64) + 0.5) * dx
    Z, Y, X = np.meshgrid(xs, xs, xs, indexing="ij")
    p0 = 1.0 / (GAMMA * Ma * Ma)
    u = np.sin(X) * np.cos(Y) * np.cos(Z)
    v = -np.cos(X) * np.sin(Y) * np.cos(Z)
    w = np.zeros_like(X)
    p = p0 + (1.0 / 16.0) * (np.cos(2 * X) + np.cos(2 * Y)) * (np.cos(2 * Z) + 2.0)
    rho = np.ones_like(X)
    base = dict(idimension=3, equation=abi.EQ_NAVIER_STOKES, mu=1.0 / Re, prandtl=Pr,
                reconstruct=abi.RECON_MUSCL, limiter=abi.LIMITER_VANALBADA, kappa=1.0 / 3.0,
                flux_split=abi.FLUX_ROE, entropy_fix=0.05, rk_stages=3, timestep_set=abi.DT_CFL, cfl=0.5)
    base.update(cfg)
    c = Case(name=f"tgv_{N}", cfg=base, meta={"N": N, "dx": dx})
    c.blocks.append(((N, N, N), (dx, dx, dx)))
    c.origins.append((0, 0, 0))
    c.bcs = [(0, r, abi.BC_PERIODIC) for r in range(1, 7)]
    c.states.append(prim_to_cons(rho, u, v, w, p))
    return c


def kinetic_energy(q, dV=1.0):
    """Volume-integrated kinetic energy sum 0.5*rho|u|^2 dV."""
    return float(0.5 * np.sum((q[1] ** 2 + q[2] ** 2 + q[3] ** 2) / q[0]) * dV)


def enstrophy(q, dx, dV=None):
    """Volume-integrated enstrophy sum 0.5*rho|curl u|^2 dV of a periodic
    single-block state (5, nk, nj, ni) with uniform spacing dx: the vorticity
    from second-order central differences, wrapped across every face (the
    Taylor-Green box). Fixed operation order, so equal states give equal
    values bit for bit."""
    dV = dx ** 3 if dV is None else dV
    rho = q[0]
    u, v, w = q[1] / rho, q[2] / rho, q[3] / rho

    def d(f, axis):  # axis 2 = x (i), 1 = y (j), 0 = z (k)
        return (np.roll(f, -1, axis=axis) - np.roll(f, 1, axis=axis)) / (2.0 * dx)

    wx = d(w, 1) - d(v, 0)
    wy = d(u, 0) - d(w, 2)
    wz = d(v, 2) - d(u, 1)
    return float(0.5 * np.sum(rho * (wx * wx + wy * wy + wz * wz)) * dV)


# ---------------------------------------------------------------- batched families
def blast(n=(64, 64, 64), seed=0, **cfg) -> Case:
    """Spherical blast in a unit box: (rho,p) inside / outside a sphere of
    seeded radius, rho~U[0.2,2], p~U[0.1,5], at rest, transmissive faces."""
    rng = np.random.default_rng(seed)
    r0 = rng.uniform(0.1, 0.3)
    rin, rout = rng.uniform(0.2, 2.0, size=2)
    pin, pout = rng.uniform(0.1, 5.0, size=2)
    h = [1.0 / m for m in n]
    xs = [(np.arange(n[a], dtype=np.float64) + 0.5) * h[a] for a in range(3)]
    Z, Y, X = np.meshgrid(xs[2], xs[1], xs[0], indexing="ij")
    inside = (X - 0.5) ** 2 + (Y - 0.5) ** 2 + (Z - 0.5) ** 2 <= r0 * r0
    rho = np.where(inside, rin, rout)
    p = np.where(inside, pin, pout)
    z = np.zeros_like(rho)
    base = dict(idimension=3, rk_stages=3, timestep_set=abi.DT_CFL, cfl=0.4)
    base.update(cfg)
    c = Case(name=f"blast_{seed}", cfg=base)
    c.blocks.append((tuple(n), tuple(h)))
    c.origins.append((0, 0, 0))
    c.states.append(prim_to_cons(rho, z, z, z, p))
    return c


def shock_tube(n=(64, 64, 64), seed=0, **cfg) -> Case:
    """Oblique shock tube: two seeded states split by a plane through the box
    centre with a random unit normal."""
    rng = np.random.default_rng(seed)
    nv = rng.normal(size=3)
    nv /= np.linalg.norm(nv)
    rl, rr = rng.uniform(0.2, 2.0, size=2)
    pl, pr = rng.uniform(0.1, 5.0, size=2)
    h = [1.0 / m for m in n]
    xs = [(np.arange(n[a], dtype=np.float64) + 0.5) * h[a] for a in range(3)]
    Z, Y, X = np.meshgrid(xs[2], xs[1], xs[0], indexing="ij")
    side = (X - 0.5) * nv[0] + (Y - 0.5) * nv[1] + (Z - 0.5) * nv[2] < 0.0
    rho = np.where(side, rl, rr)
    p = np.where(side, pl, pr)
    z = np.zeros_like(rho)
    base = dict(idimension=3, rk_stages=3, timestep_set=abi.DT_CFL, cfl=0.4)
    base.update(cfg)
    c = Case(name=f"shocktube_{seed}", cfg=base)
    c.blocks.append((tuple(n), tuple(h)))
    c.origins.append((0, 0, 0))
    c.states.append(prim_to_cons(rho, z, z, z, p))
    return c


def assemble(case: Case, per_block):
    """Place per-block arrays (., nk, nj, ni) into one global array using origins."""
    N = [0, 0, 0]
    for (n, _), o in zip(case.blocks, case.origins):
        for a in range(3):
            N[a] = max(N[a], o[a] + n[a])
    lead = per_block[0].shape[:-3]
    out = np.zeros(lead + (N[2], N[1], N[0]))
    for a, (n, _), o in zip(per_block, case.blocks, case.origins):
        out[..., o[2]:o[2] + n[2], o[1]:o[1] + n[1], o[0]:o[0] + n[0]] = a
    return out
