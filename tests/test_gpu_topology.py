"""Block connections with permuted and reversed axes (the signed donor_type
of ClassGeomFace, defs_face_geom.f90:378-402): a periodic box in two blocks
whose second block stores the box with its x and y axes swapped (or y also
reversed). The reference maps indices only (no vector rotation), and so does
this library; the GPU path must match the oracle bit for bit."""
import numpy as np
import pytest

import oracle as orc
from fvm3d import abi, cases
from fvm3d.solver import Solver

pytestmark = pytest.mark.gpu

N = 16
H = N // 2


def two_block_box(reverse: bool, **cfg):
    dx = 1.0 / N
    xs = (np.arange(N) + 0.5) * dx
    Z, Y, X = np.meshgrid(xs, xs, xs, indexing="ij")
    rho = 1.0 + 0.2 * np.exp(-60 * ((X - 0.3) ** 2 + (Y - 0.6) ** 2 + (Z - 0.5) ** 2))
    p = 1.0 + 0.5 * np.exp(-60 * ((X - 0.3) ** 2 + (Y - 0.6) ** 2 + (Z - 0.5) ** 2))
    zero = np.zeros_like(rho)
    q = cases.prim_to_cons(rho, zero, zero, zero, p)          # (5, z, y, x)
    base = dict(idimension=3, reconstruct=abi.RECON_WENO, flux_split=abi.FLUX_ROE, rk_stages=3,
                timestep_set=abi.DT_FIXED, dt=2e-3)
    base.update(cfg)
    c = cases.Case(name="swapped_box", cfg=base)
    # block A: x in [0, H), its own axes; block B: x in [H, N) with local
    # i = global y (reversed: N-1-y), local j = global x - H
    qa = q[:, :, :, :H]
    qb = q[:, :, :, H:].transpose(0, 1, 3, 2)                 # (5, z, x-H, y) = (5, k, j, i)
    if reverse:
        qb = qb[:, :, :, ::-1]
    c.blocks = [((H, N, N), (dx, dx, dx)), ((N, H, N), (dx, dx, dx))]
    c.states = [np.ascontiguousarray(qa), np.ascontiguousarray(qb)]
    A, B = 0, 1
    ilo, ihi = ((N - 1, 0) if reverse else (0, N - 1))       # B's i for A's j = 0 .. N-1
    sg = -1 if reverse else 1
    c.bcs = [(A, r, abi.BC_PERIODIC) for r in (3, 4, 5, 6)] + [(B, r, abi.BC_PERIODIC) for r in (1, 2, 5, 6)]
    c.bcs += [(A, 1, abi.BC_CONNECTED), (A, 2, abi.BC_CONNECTED), (B, 3, abi.BC_CONNECTED), (B, 4, abi.BC_CONNECTED)]
    c.conns = [
        # A i-max ghosts (global x = H..H+2) <- B j = 0..2
        (A, ((H, H + 2), (0, N - 1), (0, N - 1)), B, ((0, 2), (ilo, ihi), (0, N - 1)), (2, sg * 1, 3)),
        # A i-min ghosts (global x = N-3..N-1, periodic) <- B j = H-3..H-1
        (A, ((-3, -1), (0, N - 1), (0, N - 1)), B, ((H - 3, H - 1), (ilo, ihi), (0, N - 1)), (2, sg * 1, 3)),
        # B j-min ghosts (global x = H-3..H-1) <- A i = H-3..H-1
        (B, ((0, N - 1), (-3, -1), (0, N - 1)), A, ((ilo, ihi), (H - 3, H - 1), (0, N - 1)), (sg * 2, 1, 3)),
        # B j-max ghosts (global x = N..N+2, periodic) <- A i = 0..2
        (B, ((0, N - 1), (H, H + 2), (0, N - 1)), A, ((ilo, ihi), (0, 2), (0, N - 1)), (sg * 2, 1, 3)),
    ]
    return c


@pytest.mark.parametrize("reverse", [False, True])
@pytest.mark.parametrize("recon,flux", [(abi.RECON_WENO, abi.FLUX_ROE), (abi.RECON_MUSCL, abi.FLUX_AUSM)])
def test_permuted_connections_exact(reverse, recon, flux):
    c = two_block_box(reverse, reconstruct=recon, flux_split=flux, limiter=abi.LIMITER_MINMOD)
    g = c.apply(Solver(c.config()))
    o = c.apply(orc.Oracle(c.config()))
    g.step(4)
    o.step(4)
    for b in range(2):
        assert np.array_equal(g.get_state(b), o.get_state(b)), f"block {b}"


@pytest.mark.parametrize("p,periodic,builder", [
    (6, (True, True, True), "vortex"),
    (4, (False, False, False), "blast"),
])
def test_partitioned_case_gpu_equals_single_block_and_oracle(p, periodic, builder):
    # partition.partition_case (the IF split of method_partition.f90:576-666)
    # run on the GPU: the p connected pieces reassemble to the unsplit GPU
    # run and to the oracle's unsplit run bit for bit
    from fvm3d import partition

    if builder == "vortex":
        c1 = cases.isentropic_vortex(N=24, layout="single", rk_stages=3, reconstruct=abi.RECON_MUSCL,
                                     limiter=abi.LIMITER_MINMOD, flux_split=abi.FLUX_ROE)
    else:
        c1 = cases.blast((24, 20, 16), seed=2, reconstruct=abi.RECON_WENO, flux_split=abi.FLUX_AUSM,
                         compat=abi.COMPAT_TEXTBOOK)
    cp = partition.partition_case(c1, p, periodic=periodic)
    assert len(cp.blocks) == p
    g1 = c1.apply(Solver(c1.config()))
    gp = cp.apply(Solver(cp.config()))
    o1 = c1.apply(orc.Oracle(c1.config()))
    t1, _, _ = g1.step(3)
    tp, _, _ = gp.step(3)
    o1.step(3)
    qp = cases.assemble(cp, [gp.get_state(b) for b in range(p)])
    assert np.array_equal(qp, g1.get_state(0))
    assert np.array_equal(qp, o1.get_state(0))
    assert t1 == tp
