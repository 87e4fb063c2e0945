"""Parity on the three solver configurations at their stated sizes.

* 2D four-quadrant Riemann problem, 256 x 256, MUSCL / minmod (kappa 1/3) +
  Roe (entropy fix 0.2), SSP-RK3, 500 steps of a fixed dt = 0.5 min(dx / (|u_d|
  + c)) of the initial state (the reference has only a fixed time step,
  class_time_discret.f90:111-122).
* 3D Euler isentropic vortex, 128^3 in 8 uneven periodic blocks, WENO5 +
  AUSM, classic RK4, CFL 0.5.
* 3D Navier-Stokes Taylor-Green vortex, 128^3, MUSCL / Van Albada + Roe,
  central viscous fluxes, SSP-RK3, CFL 0.5: kinetic-energy and enstrophy
  histories, step by step.

Each compares the CUDA path (through the C ABI) with the CPU oracle on the
same seeded inputs. Bounds: the exact FP64 form is bit-identical (state,
last-stage rhs, time); residual norms agree to 1e-12 relative (their
summation order differs); the FP64 form holds 1e-12 relative max-norm on the
smooth vortex, 1e-10 mean |d rho| across the Riemann problem's shocks and
1e-10 relative on the Taylor-Green histories; the FP32-flux form holds 1e-6
mean |d rho| on the vortex, 1e-5 on the Riemann problem and 1e-6 / 1e-5
relative on the kinetic energy / enstrophy."""
import numpy as np
import pytest

import oracle as orc
from fvm3d import abi, cases
from fvm3d.solver import Solver

pytestmark = pytest.mark.gpu


def riemann_fixed_dt(case):
    """0.5 min over cells and axes of dx / (|u_d| + c) of the initial state."""
    q = case.states[0]
    rho, u, v, _, p = cases.cons_to_prim(q)
    c = np.sqrt(cases.GAMMA * p / rho)
    dx = case.meta["dx"]
    return 0.5 * min(float((dx / (np.abs(u) + c)).min()), float((dx / (np.abs(v) + c)).min()))


@pytest.fixture(scope="module")
def riemann256():
    c = cases.riemann2d(n=256, seed=0)
    dt = riemann_fixed_dt(c)
    o = c.apply(orc.Oracle(c.config(dt=dt)))
    to, rao, rro, _ = o.step(500)
    ref = dict(q=o.get_state(0), rhs=o.get_rhs(0), t=to, ra=rao, rr=rro)
    o.close()
    return c, dt, ref


def test_riemann256_500_steps_exact(riemann256):
    c, dt, ref = riemann256
    g = c.apply(Solver(c.config(dt=dt, store_rhs=1)))
    tg, rag, rrg = g.step(500)
    assert np.array_equal(g.get_state(0), ref["q"])
    assert np.array_equal(g.get_rhs(0), ref["rhs"])
    assert tg == ref["t"]
    np.testing.assert_allclose(rag, ref["ra"], rtol=1e-12, atol=0)
    np.testing.assert_allclose(rrg, ref["rr"], rtol=1e-12, atol=0)
    g.close()


@pytest.mark.parametrize("prec,bound", [(abi.PREC_FP64, 1e-10), (abi.PREC_FP32_FLUX, 1e-5)])
def test_riemann256_500_steps_fast_forms(riemann256, prec, bound):
    c, dt, ref = riemann256
    g = c.apply(Solver(c.config(dt=dt, precision=prec)))
    g.step(500)
    err = float(np.abs(g.get_state(0)[0] - ref["q"][0]).mean())
    assert err <= bound, err
    g.close()


@pytest.fixture(scope="module")
def vortex128():
    c = cases.isentropic_vortex(N=128, layout="blocks8")
    o = c.apply(orc.Oracle(c.config()))
    to, rao, _, _ = o.step(3)
    ref = dict(q=[o.get_state(b) for b in range(8)], rhs=[o.get_rhs(b) for b in range(8)], t=to, ra=rao)
    o.close()
    return c, ref


def test_vortex128_blocks8_exact(vortex128):
    c, ref = vortex128
    g = c.apply(Solver(c.config(store_rhs=1)))
    tg, rag, _ = g.step(3)
    for b in range(8):
        assert np.array_equal(g.get_state(b), ref["q"][b]), f"block {b}"
        assert np.array_equal(g.get_rhs(b), ref["rhs"][b]), f"rhs block {b}"
    assert tg == ref["t"]
    np.testing.assert_allclose(rag, ref["ra"], rtol=1e-12, atol=0)
    g.close()


def test_vortex128_blocks8_fast_forms(vortex128):
    c, ref = vortex128
    g = c.apply(Solver(c.config(precision=abi.PREC_FP64)))
    g.step(3)
    for b in range(8):
        a, r = g.get_state(b), ref["q"][b]
        assert np.abs(a - r).max() <= 1e-12 * np.abs(r).max(), f"fp64 block {b}"
    g.close()
    f = c.apply(Solver(c.config(precision=abi.PREC_FP32_FLUX)))
    f.step(3)
    cells = sum(q[0].size for q in ref["q"])
    err = sum(float(np.abs(f.get_state(b)[0] - ref["q"][b][0]).sum()) for b in range(8)) / cells
    assert err <= 1e-6, err
    f.close()


TGV_STEPS = 20


def _histories(target, case, steps):
    dx = case.meta["dx"]
    ke, en = [], []
    for _ in range(steps):
        target.step(1)
        q = target.get_state(0)
        ke.append(cases.kinetic_energy(q, dx ** 3))
        en.append(cases.enstrophy(q, dx))
    return np.array(ke), np.array(en)


@pytest.fixture(scope="module")
def tgv128():
    c = cases.taylor_green(N=128)
    o = c.apply(orc.Oracle(c.config()))
    ke, en = _histories(o, c, TGV_STEPS)
    o.close()
    return c, ke, en


def test_tgv128_histories_exact(tgv128):
    c, ke, en = tgv128
    g = c.apply(Solver(c.config()))
    kg, eg = _histories(g, c, TGV_STEPS)
    assert np.array_equal(kg, ke)
    assert np.array_equal(eg, en)
    # the flow decays: kinetic energy falls every step
    assert (np.diff(ke) < 0).all()
    g.close()


@pytest.mark.parametrize("prec,bke,ben", [(abi.PREC_FP64, 1e-10, 1e-10), (abi.PREC_FP32_FLUX, 1e-6, 1e-5)])
def test_tgv128_histories_fast_forms(tgv128, prec, bke, ben):
    c, ke, en = tgv128
    g = c.apply(Solver(c.config(precision=prec)))
    kg, eg = _histories(g, c, TGV_STEPS)
    assert (np.abs(kg - ke) <= bke * np.abs(ke)).all(), np.abs(kg / ke - 1).max()
    assert (np.abs(eg - en) <= ben * np.abs(en)).all(), np.abs(eg / en - 1).max()
    g.close()
