"""Known-answer tests that pin the CPU oracle (the reference's own tests hold
no numbers, and no Fortran compiler exists here to run the reference)."""
import math

import numpy as np
import pytest

import oracle as orc
from fvm3d import abi, cases

G = 1.4


def phys_flux(s, d, gamma=G):
    rho, u, v, w, p = s
    vel = (u, v, w)
    Vn = vel[d]
    H = gamma / (gamma - 1.0) * p / rho + 0.5 * (u * u + v * v + w * w)
    F = np.array([rho * Vn, rho * u * Vn, rho * v * Vn, rho * w * Vn, rho * H * Vn])
    F[1 + d] += p
    return F


def rand_state(rng, mach=None):
    rho = rng.uniform(0.2, 2.0)
    p = rng.uniform(0.1, 5.0)
    c = math.sqrt(G * p / rho)
    vel = rng.uniform(-1, 1, 3) * c * (0.8 if mach is None else mach)
    return np.array([rho, vel[0], vel[1], vel[2], p])


@pytest.mark.parametrize("flux", [abi.FLUX_ROE, abi.FLUX_AUSM, abi.FLUX_VANLEER])
@pytest.mark.parametrize("d", [0, 1, 2])
def test_flux_consistency_subsonic(flux, d):
    rng = np.random.default_rng(10 + d)
    for _ in range(50):
        s = rand_state(rng, mach=0.5)
        F = orc.flux_point(flux, d, G, 0.2, s, s)
        np.testing.assert_allclose(F, phys_flux(s, d), rtol=1e-13, atol=1e-13)


def test_roe_consistency_exact():
    # L = R: every wave jump is zero and F = 0.5*(F_L + F_R) = F_L bit for bit
    rng = np.random.default_rng(1)
    for _ in range(50):
        s = rand_state(rng, mach=2.0)
        for d in range(3):
            F = orc.flux_point(abi.FLUX_ROE, d, G, 0.05, s, s)
            np.testing.assert_allclose(F, phys_flux(s, d), rtol=1e-15, atol=1e-15)


def test_vanleer_supersonic_quirk_and_textbook():
    # scheme_FVS_VanLeer.f90:84-95 keeps the subsonic factors for |M|>=1, so the
    # reference momentum flux of a supersonic state is not the Euler flux;
    # the textbook form gives the full flux.
    s = np.array([1.0, 2.5, 0.1, -0.2, 1.0])  # M = 2.5/sqrt(1.4) > 1
    F_ref = orc.flux_point(abi.FLUX_VANLEER, 0, G, 0.0, s, s, compat=0)
    F_tb = orc.flux_point(abi.FLUX_VANLEER, 0, G, 0.0, s, s, compat=1)
    np.testing.assert_allclose(F_tb, phys_flux(s, 0), rtol=1e-14)
    assert F_ref[0] == pytest.approx(phys_flux(s, 0)[0], rel=1e-14)  # mass flux rho*c*M
    assert abs(F_ref[1] - phys_flux(s, 0)[1]) > 1e-3


def test_flux_upwind_supersonic_roe():
    s = np.array([1.0, 3.0, 0.0, 0.0, 1.0])
    t = np.array([0.5, 3.0, 0.0, 0.0, 0.4])
    F = orc.flux_point(abi.FLUX_ROE, 0, G, 0.0, s, t)
    np.testing.assert_allclose(F, phys_flux(s, 0), rtol=1e-12)


def test_weno_polynomials():
    # candidate stencils are exact for quadratics; weights sum to one
    for compat in (0, 1):
        for a, b, c in [(1.0, 0.0, 0.0), (0.3, 1.7, 0.0), (2.0, -0.5, 0.25)]:
            x = np.arange(-2, 3, dtype=float)  # cell averages of u(x)=a+bx+cx^2
            u = a + b * x + c * (x * x + 1.0 / 12.0)
            face = a + b * 0.5 + c * 0.25  # point value at x = 1/2
            assert orc.weno_point(u, compat) == pytest.approx(face, rel=1e-12, abs=1e-12)


def test_weno_is1_quirk():
    # IS_1 as written uses (u2+u4)^2: for a large constant offset the central
    # stencil weight collapses in the reference form but not in the textbook one
    h = 0.05
    x = h * np.arange(-2, 3, dtype=float)
    u = 10.0 + np.sin(x) * 2.0 * math.sin(0.5 * h) / h  # cell averages of 10 + sin
    r_ref = orc.weno_point(u, 0)
    r_tb = orc.weno_point(u, 1)
    exact = 10.0 + math.sin(0.5 * h)
    assert r_ref != r_tb
    assert abs(r_tb - exact) < 1e-7
    assert abs(r_ref - exact) > abs(r_tb - exact)


def py_minmod(x, y):
    return 0.5 * (math.copysign(1, x) + math.copysign(1, y)) * min(abs(x), abs(y))


def py_vanleer(x, y):
    return (math.copysign(1, x) + math.copysign(1, y)) * x * y / (abs(x) + abs(y) + 1e-6)


def py_vanalbada(x, y):
    return (x * (y * y + 1e-6) + y * (x * x + 1e-6)) / (x * x + y * y + 1e-6)


@pytest.mark.parametrize("lim", [abi.LIMITER_NONE, abi.LIMITER_MINMOD, abi.LIMITER_VANLEER,
                                 abi.LIMITER_VANALBADA, abi.SCHEME_NULL])
def test_muscl_matches_formula(lim):
    rng = np.random.default_rng(lim + 7)
    k = 1.0 / 3.0
    for _ in range(200):
        p1, p2, p3 = rng.normal(size=3)
        dm, dp = p2 - p1, p3 - p2
        if lim == abi.LIMITER_MINMOD:
            bm, bp = py_minmod(dm, dp), py_minmod(dp, dm)
        elif lim == abi.LIMITER_VANLEER:
            bm = bp = py_vanleer(dm, dp)
        elif lim == abi.LIMITER_VANALBADA:
            bm = bp = py_vanalbada(dm, dp)
        else:
            bm, bp = dm, dp
        L = p2 + 0.25 * ((1 - k) * bm + (1 + k) * bp)
        R = p2 - 0.25 * ((1 - k) * bp + (1 + k) * bm)
        assert orc.muscl_point(p1, p2, p3, -1, lim, k) == L
        assert orc.muscl_point(p1, p2, p3, 1, lim, k) == R


def test_muscl_linear_and_extremum():
    k = 1.0 / 3.0
    for lim in (abi.LIMITER_NONE, abi.LIMITER_MINMOD):
        assert orc.muscl_point(1.0, 2.0, 3.0, -1, lim, k) == pytest.approx(2.5)
        assert orc.muscl_point(1.0, 2.0, 3.0, 1, lim, k) == pytest.approx(1.5)
    # local maximum: minmod gives first order
    assert orc.muscl_point(1.0, 2.0, 1.0, -1, abi.LIMITER_MINMOD, k) == 2.0


def _run(case, steps, **cfg):
    o = case.apply(orc.Oracle(case.config(**cfg)))
    out = o.step(steps)
    return o, out


@pytest.mark.parametrize("recon,flux", [(abi.RECON_SIMPLE, abi.FLUX_ROE), (abi.RECON_MUSCL, abi.FLUX_VANLEER),
                                        (abi.RECON_WENO, abi.FLUX_AUSM)])
def test_free_stream_preserved_exactly(recon, flux):
    c = cases.isentropic_vortex(N=16, layout="blocks8", beta=0.0, reconstruct=recon, flux_split=flux,
                                limiter=abi.LIMITER_MINMOD, rk_stages=3)
    o, (t, ra, rr, dt) = _run(c, 3)
    for b, q in enumerate(c.states):
        assert np.array_equal(o.get_state(b), q)
    assert ra[5] == 0.0


def test_multiblock_equals_single_block():
    c8 = cases.isentropic_vortex(N=32, layout="blocks8", rk_stages=4)
    c1 = cases.isentropic_vortex(N=32, layout="single", rk_stages=4)
    o8, _ = _run(c8, 2)
    o1, _ = _run(c1, 2)
    q8 = cases.assemble(c8, [o8.get_state(b) for b in range(8)])
    q1 = o1.get_state(0)
    assert np.array_equal(q8, q1)


def test_conservation_periodic():
    c = cases.isentropic_vortex(N=16, layout="blocks8", rk_stages=3, reconstruct=abi.RECON_MUSCL,
                                limiter=abi.LIMITER_VANALBADA, flux_split=abi.FLUX_ROE)
    tot0 = sum(q.sum(axis=(1, 2, 3)) for q in c.states)
    o, _ = _run(c, 5)
    tot1 = sum(o.get_state(b).sum(axis=(1, 2, 3)) for b in range(8))
    np.testing.assert_allclose(tot1, tot0, rtol=1e-12)


def test_residual_formula():
    c = cases.riemann2d(n=17, seed=2, dt=1e-3)
    o, (t, ra, rr, dt) = _run(c, 2)
    rhs = o.get_rhs(0)
    res2 = (rhs ** 2).reshape(5, -1).mean(axis=1)
    np.testing.assert_allclose(ra[:5], np.sqrt(res2), rtol=1e-13)
    np.testing.assert_allclose(ra[5], np.sqrt(res2.mean()), rtol=1e-13)
    assert t == pytest.approx(2e-3)


def test_riemann_symmetry():
    # x<->y symmetric quadrant data stays symmetric (to rounding)
    c = cases.riemann2d(n=24, seed=0, dt=1e-3)
    st = [(1.0, 0.1, 0.1, 0.0, 1.0), (0.5, 0.2, -0.1, 0.0, 0.4), (0.8, -0.2, -0.2, 0.0, 0.9),
          (0.5, -0.1, 0.2, 0.0, 0.4)]
    dx = c.meta["dx"]
    x = dx * np.arange(24)
    X, Y = np.meshgrid(x, x, indexing="xy")
    rho, u, v, w, p = cases._quadrant_fill(X, Y, 0.5, 0.5, st)
    c.states[0] = cases.prim_to_cons(rho, u, v, w, p)[:, None]
    o, _ = _run(c, 10)
    q = o.get_state(0)[:, 0]
    np.testing.assert_allclose(q[0], q[0].T, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(q[1], q[2].T, rtol=1e-12, atol=1e-12)


def test_reference_case_planes_identical():
    c = cases.riemann2d_reference()
    o, (t, ra, rr, dt) = _run(c, 5)
    q = o.get_state(0)
    assert np.array_equal(q[:, 0], q[:, 1])
    assert np.isfinite(ra).all() and ra[5] > 0
    assert t == pytest.approx(5 * 2e-4)


def test_cfl_dt_formula():
    c = cases.isentropic_vortex(N=16, layout="single", timestep_set=abi.DT_CFL, cfl=0.5)
    o, (t, ra, rr, dt) = _run(c, 1)
    q = c.states[0]
    rho, u, v, w, p = cases.cons_to_prim(q)
    cs = np.sqrt(1.4 * p / rho)
    dx = c.meta["dx"]
    s = (np.abs(u) + cs) / dx + (np.abs(v) + cs) / dx + (np.abs(w) + cs) / dx
    assert dt == pytest.approx(0.5 / s.max(), rel=1e-14)


def test_vortex_converges_to_exact():
    # textbook WENO5 + AUSM on the vortex: error drops with resolution
    errs = []
    for N in (16, 32):
        c = cases.isentropic_vortex(N=N, layout="single", compat=abi.COMPAT_TEXTBOOK, timestep_set=abi.DT_FIXED,
                                    dt=0.02 * 16 / N)
        o, (t, *_r) = _run(c, int(0.4 / (0.02 * 16 / N)))
        ex = cases.vortex_exact(c, t)[0]
        errs.append(np.abs(o.get_state(0)[0] - ex[0]).mean())
    assert errs[1] < 0.5 * errs[0]


def test_reference_weno_blast_nan_and_textbook_fallback():
    # the reference reconstructs conservative variables without a positivity
    # limit: on a strong blast its face states go negative and the residual
    # becomes NaN (its converged() then stops with "Error: ABSRES NaN");
    # TEXTBOOK compat falls back to first-order states there
    c = cases.blast((20, 20, 20), seed=0, reconstruct=abi.RECON_WENO, flux_split=abi.FLUX_AUSM)
    _, (t, ra, rr, dt) = _run(c, 2)
    assert np.isnan(ra[5])
    c = cases.blast((20, 20, 20), seed=0, reconstruct=abi.RECON_WENO, flux_split=abi.FLUX_AUSM,
                    compat=abi.COMPAT_TEXTBOOK)
    o, (t, ra, rr, dt) = _run(c, 3)
    assert np.isfinite(ra).all() and np.isfinite(o.get_state(0)).all()
