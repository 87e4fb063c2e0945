"""GPU path vs the CPU oracle through the C ABI.

Exact-FP64 mode must be bit-identical to the oracle (same operation order,
no FMA contraction). The fast FP64 form is held to 1e-12 relative max-norm on
smooth flows and a stated L1 bound across shocks; the FP32-flux form to an L1
density error of 1e-6 against the FP64 oracle on the smooth vortex."""
import numpy as np
import pytest

import oracle as orc
from fvm3d import abi, cases
from fvm3d.solver import Solver

pytestmark = pytest.mark.gpu


def run_both(case, steps, gpu_over=None, **over):
    cfg_o = case.config(**over)
    g_over = dict(over)
    g_over.update(gpu_over or {})
    g = case.apply(Solver(case.config(store_rhs=1, **g_over)))
    o = case.apply(orc.Oracle(cfg_o))
    rg = g.step(steps)
    ro = o.step(steps)
    return g, o, rg, ro


def states(x, n):
    return [x.get_state(b) for b in range(n)]


RECON_FLUX = [(r, f) for r in (abi.RECON_SIMPLE, abi.RECON_MUSCL, abi.RECON_WENO)
              for f in (abi.FLUX_ROE, abi.FLUX_VANLEER, abi.FLUX_AUSM)]


@pytest.mark.parametrize("recon,flux", RECON_FLUX)
@pytest.mark.parametrize("nk", [1, 2])
def test_2d_exact_bitwise(recon, flux, nk):
    c = cases.riemann2d(n=37, seed=11, nk=nk, reconstruct=recon, flux_split=flux, dt=1.5e-3)
    g, o, (tg, rag, rrg), (to, rao, rro, _) = run_both(c, 4)
    assert np.array_equal(g.get_state(0), o.get_state(0))
    assert np.array_equal(g.get_rhs(0), o.get_rhs(0))
    assert tg == to
    np.testing.assert_allclose(rag, rao, rtol=1e-12, atol=0)
    np.testing.assert_allclose(rrg, rro, rtol=1e-12, atol=0)


@pytest.mark.parametrize("lim", [abi.LIMITER_NONE, abi.LIMITER_MINMOD, abi.LIMITER_VANLEER,
                                 abi.LIMITER_VANALBADA, abi.SCHEME_NULL])
def test_limiters_exact_bitwise(lim):
    c = cases.riemann2d(n=40, seed=4, limiter=lim, kappa=0.33333, dt=1e-3)
    g, o, _, _ = run_both(c, 3)
    assert np.array_equal(g.get_state(0), o.get_state(0))


def test_reference_case_exact():
    c = cases.riemann2d_reference()
    g, o, rg, ro = run_both(c, 20)
    assert np.array_equal(g.get_state(0), o.get_state(0))
    np.testing.assert_allclose(rg[1], ro[1], rtol=1e-12)


@pytest.mark.parametrize("recon,flux,stages,compat", [
    (abi.RECON_WENO, abi.FLUX_AUSM, 4, abi.COMPAT_REFERENCE),
    (abi.RECON_WENO, abi.FLUX_AUSM, 4, abi.COMPAT_TEXTBOOK),
    (abi.RECON_WENO, abi.FLUX_ROE, 3, abi.COMPAT_REFERENCE),
    (abi.RECON_MUSCL, abi.FLUX_ROE, 3, abi.COMPAT_REFERENCE),
    (abi.RECON_MUSCL, abi.FLUX_VANLEER, 4, abi.COMPAT_TEXTBOOK),
    (abi.RECON_SIMPLE, abi.FLUX_AUSM, 3, abi.COMPAT_REFERENCE),
])
def test_3d_multiblock_exact_bitwise(recon, flux, stages, compat):
    c = cases.isentropic_vortex(N=32, layout="blocks8", reconstruct=recon, flux_split=flux, rk_stages=stages,
                                compat=compat, limiter=abi.LIMITER_MINMOD, kappa=1.0 / 3.0)
    g, o, (tg, rag, _), (to, rao, _, _) = run_both(c, 3)
    for b in range(8):
        assert np.array_equal(g.get_state(b), o.get_state(b)), f"block {b}"
        assert np.array_equal(g.get_rhs(b), o.get_rhs(b)), f"rhs block {b}"
    assert tg == to
    np.testing.assert_allclose(rag, rao, rtol=1e-12)


@pytest.mark.parametrize("tile,zchunk", [(0, 5), (1, 8), (0, 0), (3, 7), (3, 0)])
def test_tiling_does_not_change_state(tile, zchunk):
    c = cases.isentropic_vortex(N=32, layout="blocks8")
    o = c.apply(orc.Oracle(c.config()))
    o.step(2)
    g = Solver(c.config())
    c.apply(g, states=False)
    g.lib.fvm_step  # noqa: B018
    from fvm3d import tuning

    tuning.set_tuning(g, 0, tile, zchunk)
    for b, q in enumerate(c.states):
        g.set_state(b, q)
    g.step(2)
    for b in range(8):
        assert np.array_equal(g.get_state(b), o.get_state(b))


@pytest.mark.parametrize("split", [2, 4])
def test_tail_split_does_not_change_state(split):
    # 16x8 tiles with 4-plane z chunks on the 96^3 vortex in 8 blocks give
    # 1728 tasks, more than the stage kernel's resident CTAs, so the work
    # queue has a partial last round whose tasks are cut into `split` pieces
    from fvm3d import tuning
    from fvm3d.solver import FvmError

    c = cases.isentropic_vortex(N=96, layout="blocks8")
    o = c.apply(orc.Oracle(c.config()))
    ro = o.step(2)
    g = Solver(c.config())
    c.apply(g, states=False)
    tuning.set_tuning(g, 0, 3, 4)
    tuning.set_tail_split(g, 0, split)
    with pytest.raises(FvmError) as e:
        tuning.set_tail_split(g, 0, 0)
    assert e.value.code == 1  # FVM_ERR_INVALID
    for b, q in enumerate(c.states):
        g.set_state(b, q)
    rg = g.step(2)
    for b in range(8):
        assert np.array_equal(g.get_state(b), o.get_state(b))
    # the residual norms sum the same cells over a different partition
    np.testing.assert_allclose(rg[1], ro[1], rtol=1e-12)


@pytest.mark.parametrize("recon,flux", [(abi.RECON_MUSCL, abi.FLUX_ROE), (abi.RECON_WENO, abi.FLUX_VANLEER)])
def test_tma_tile_rk3_exact(recon, flux):
    # the 16x8 tile (plane, z window and RK operands by tensor copies) in the
    # exact form, SSP-RK3 (q_in operand), 8 uneven periodic blocks
    from fvm3d import tuning

    c = cases.isentropic_vortex(N=24, layout="blocks8", rk_stages=3, reconstruct=recon, flux_split=flux,
                                limiter=abi.LIMITER_VANALBADA, kappa=1.0 / 3.0)
    o = c.apply(orc.Oracle(c.config()))
    o.step(3)
    g = Solver(c.config())
    c.apply(g, states=False)
    tuning.set_tuning(g, 0, 3, 5)
    for b, q in enumerate(c.states):
        g.set_state(b, q)
    g.step(3)
    for b in range(8):
        assert np.array_equal(g.get_state(b), o.get_state(b)), f"block {b}"


@pytest.mark.parametrize("compat", [abi.COMPAT_REFERENCE, abi.COMPAT_TEXTBOOK])
def test_long_run_exact_bitwise(compat):
    # 300 CFL steps of the 8-block vortex: the exact form stays bit-identical
    # to the oracle (dt history, ghost exchange and residual state included)
    c = cases.isentropic_vortex(N=16, layout="blocks8", compat=compat)
    g, o, (tg, _, _), (to, _, _, _) = run_both(c, 300)
    assert tg == to
    for b in range(8):
        assert np.array_equal(g.get_state(b), o.get_state(b)), f"block {b}"


def test_local_timestep_exact():
    c = cases.isentropic_vortex(N=16, layout="blocks8", timestep_set=abi.DT_CFL_LOCAL, rk_stages=3,
                                reconstruct=abi.RECON_MUSCL, limiter=abi.LIMITER_VANLEER, flux_split=abi.FLUX_ROE)
    g, o, _, _ = run_both(c, 3)
    for b in range(8):
        assert np.array_equal(g.get_state(b), o.get_state(b))


def test_navier_stokes_tgv_exact():
    c = cases.taylor_green(N=16)
    g, o, (tg, rag, _), (to, rao, _, _) = run_both(c, 3)
    assert np.array_equal(g.get_state(0), o.get_state(0))
    np.testing.assert_allclose(rag, rao, rtol=1e-12)


def test_navier_stokes_fast_fp64_1e12():
    # the FP64 form's viscous terms multiply by reciprocal cell sizes instead
    # of dividing: within 1e-12 of the oracle's exact form on the smooth TGV
    c = cases.taylor_green(N=16)
    g, o, _, _ = run_both(c, 3, gpu_over=dict(precision=abi.PREC_FP64))
    a, r = g.get_state(0), o.get_state(0)
    assert np.abs(a - r).max() <= 1e-12 * np.abs(r).max()


def test_navier_stokes_fp32_flux_l1():
    # FP32 flux form (FP32 reconstruction, flux and viscous terms, FP64
    # state and RK): relative L1 error against the exact oracle after three
    # steps of the TGV, per conserved variable (momenta relative to their sum)
    c = cases.taylor_green(N=24)
    g, o, _, _ = run_both(c, 3, gpu_over=dict(precision=abi.PREC_FP32_FLUX))
    a, r = g.get_state(0), o.get_state(0)
    d = np.abs(a - r).reshape(5, -1).sum(axis=1)
    mom = np.abs(r[1:4]).sum()
    assert d[0] <= 1e-6 * np.abs(r[0]).sum()
    assert d[4] <= 1e-6 * np.abs(r[4]).sum()
    assert d[1:4].max() <= 1e-5 * mom


def test_navier_stokes_blocks_exact():
    # 8 uneven periodic blocks: connected faces and the layer-1 edge ghosts of
    # the viscous stencil, partial viscous tiles
    c = cases.isentropic_vortex(N=20, layout="blocks8", equation=abi.EQ_NAVIER_STOKES, mu=0.02, rk_stages=3,
                                reconstruct=abi.RECON_MUSCL, limiter=abi.LIMITER_VANALBADA, flux_split=abi.FLUX_ROE)
    g, o, _, _ = run_both(c, 3)
    for b in range(8):
        assert np.array_equal(g.get_state(b), o.get_state(b))


def test_navier_stokes_2d_exact():
    # 2D viscous path, transmissive regions, two independent k planes
    c = cases.riemann2d(n=27, seed=3, nk=2, dt=1e-3, equation=abi.EQ_NAVIER_STOKES, mu=5e-3)
    g, o, _, _ = run_both(c, 3)
    assert np.array_equal(g.get_state(0), o.get_state(0))


def test_fast_fp64_smooth_1e12():
    c = cases.isentropic_vortex(N=32, layout="blocks8")
    g, o, _, _ = run_both(c, 5, gpu_over=dict(precision=abi.PREC_FP64))
    for b in range(8):
        a, r = g.get_state(b), o.get_state(b)
        assert np.abs(a - r).max() <= 1e-12 * np.abs(r).max()


def test_fast_fp64_shock_l1():
    c = cases.riemann2d(n=96, seed=1, dt=2e-3)
    g, o, _, _ = run_both(c, 40, gpu_over=dict(precision=abi.PREC_FP64))
    d = np.abs(g.get_state(0) - o.get_state(0))
    assert d[0].mean() <= 1e-10


def test_fp32_flux_vortex_l1():
    c = cases.isentropic_vortex(N=32, layout="blocks8")
    g, o, _, _ = run_both(c, 10, gpu_over=dict(precision=abi.PREC_FP32_FLUX))
    err = np.mean([np.abs(g.get_state(b)[0] - o.get_state(b)[0]).mean() for b in range(8)])
    assert err <= 1e-6, err


def _oracle_and_forms(case, steps):
    o = case.apply(orc.Oracle(case.config()))
    o.step(steps)
    out = {}
    for name, prec in (("fp64", abi.PREC_FP64), ("fp32", abi.PREC_FP32_FLUX)):
        g = case.apply(Solver(case.config(precision=prec)))
        g.step(steps)
        out[name] = [g.get_state(b) for b in range(len(case.blocks))]
        g.close()
    return [o.get_state(b) for b in range(len(case.blocks))], out


FAST_SCHEMES = [(r, f, abi.COMPAT_REFERENCE) for r, f in RECON_FLUX] + \
    [(abi.RECON_WENO, abi.FLUX_AUSM, abi.COMPAT_TEXTBOOK), (abi.RECON_WENO, abi.FLUX_ROE, abi.COMPAT_TEXTBOOK)]


@pytest.mark.parametrize("recon,flux,compat", FAST_SCHEMES)
def test_fast_forms_every_scheme_3d(recon, flux, compat):
    # every reconstruction x flux kernel of the FP64 and FP32-flux forms on
    # the smooth 8-block vortex (Van Albada: no limiter branch to flip on a
    # rounding difference), SSP-RK3, against the exact oracle
    c = cases.isentropic_vortex(N=24, layout="blocks8", reconstruct=recon, flux_split=flux, compat=compat,
                                rk_stages=3, limiter=abi.LIMITER_VANALBADA, kappa=1.0 / 3.0)
    ref, got = _oracle_and_forms(c, 5)
    for b in range(8):
        assert np.abs(got["fp64"][b] - ref[b]).max() <= 1e-11 * np.abs(ref[b]).max(), f"fp64 block {b}"
    err32 = np.mean([np.abs(got["fp32"][b][0] - ref[b][0]).mean() for b in range(8)])
    assert err32 <= 1e-6, err32


@pytest.mark.parametrize("recon,flux", [(abi.RECON_MUSCL, abi.FLUX_ROE), (abi.RECON_WENO, abi.FLUX_AUSM),
                                        (abi.RECON_SIMPLE, abi.FLUX_VANLEER)])
def test_fast_forms_2d(recon, flux):
    # the 2D kernels of the FP64 and FP32-flux forms (per-thread staged
    # planes, no tensor copies) on the four-quadrant Riemann problem
    c = cases.riemann2d(n=40, seed=2, reconstruct=recon, flux_split=flux, limiter=abi.LIMITER_VANALBADA,
                        kappa=1.0 / 3.0, dt=1e-3)
    ref, got = _oracle_and_forms(c, 3)
    assert np.abs(got["fp64"][0][0] - ref[0][0]).mean() <= 1e-10
    assert np.abs(got["fp32"][0][0] - ref[0][0]).mean() <= 1e-5


def test_primitive_download():
    c = cases.riemann2d(n=20, seed=0, dt=1e-3)
    g, o, _, _ = run_both(c, 2)
    assert np.array_equal(g.get_primitive(0), o.get_primitive(0))


def test_textbook_positivity_fallback_exact():
    # a strong blast where the reference's WENO + AUSM produces NaN (see the
    # oracle test); TEXTBOOK compat falls back to first-order face states
    c = cases.blast((20, 20, 20), seed=0, reconstruct=abi.RECON_WENO, flux_split=abi.FLUX_AUSM,
                    compat=abi.COMPAT_TEXTBOOK)
    g, o, (tg, rag, _), (to, rao, _, _) = run_both(c, 3)
    assert np.array_equal(g.get_state(0), o.get_state(0))
    assert np.isfinite(rag).all()


def test_reference_blast_reports_nonfinite():
    from fvm3d.solver import FvmError

    c = cases.blast((20, 20, 20), seed=0, reconstruct=abi.RECON_WENO, flux_split=abi.FLUX_AUSM)
    g = c.apply(Solver(c.config()))
    with pytest.raises(FvmError) as e:
        g.step(2)
    assert e.value.code == 4 and "NaN" in e.value.msg


def test_tgv_kinetic_energy_history():
    # Navier-Stokes Taylor-Green vortex: the kinetic-energy history of the
    # exact FP64 path equals the oracle's bit for bit; the FP32 flux form
    # tracks it to 1e-6 relative
    c = cases.taylor_green(N=24)
    dV = c.meta["dx"] ** 3
    g = c.apply(Solver(c.config()))
    f = c.apply(Solver(c.config(precision=abi.PREC_FP32_FLUX)))
    o = c.apply(orc.Oracle(c.config()))
    for _ in range(4):
        g.step(1)
        f.step(1)
        o.step(1)
        kg = cases.kinetic_energy(g.get_state(0), dV)
        ko = cases.kinetic_energy(o.get_state(0), dV)
        kf = cases.kinetic_energy(f.get_state(0), dV)
        assert kg == ko
        assert abs(kf - ko) <= 1e-6 * ko
