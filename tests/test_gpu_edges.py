"""Edge cases of the GPU path against the oracle: degenerate and ragged
block shapes, the smallest periodic box, tiles that do not divide the block,
and the error paths of the C ABI."""
import numpy as np
import pytest

import oracle as orc
from fvm3d import abi, cases, tuning
from fvm3d.solver import FvmError, Solver

pytestmark = pytest.mark.gpu


def both(case, steps, **over):
    g = case.apply(Solver(case.config(**over)))
    o = case.apply(orc.Oracle(case.config(**over)))
    g.step(steps)
    o.step(steps)
    return g, o


@pytest.mark.parametrize("n", [(1, 1, 1), (2, 3, 1), (7, 1, 5), (1, 9, 4), (5, 3, 2)])
@pytest.mark.parametrize("recon,flux", [(abi.RECON_WENO, abi.FLUX_AUSM), (abi.RECON_MUSCL, abi.FLUX_ROE)])
def test_degenerate_blocks_exact(n, recon, flux):
    c = cases.shock_tube(n, seed=5, reconstruct=recon, flux_split=flux, limiter=abi.LIMITER_VANLEER,
                         compat=abi.COMPAT_TEXTBOOK, rk_stages=3, timestep_set=abi.DT_FIXED, dt=1e-3)
    g, o = both(c, 3)
    assert np.array_equal(g.get_state(0), o.get_state(0))


def test_smallest_periodic_box_exact():
    # 3 cells per axis: every ghost layer of the 3-deep halo wraps onto the
    # block itself
    c = cases.isentropic_vortex(N=3, layout="single")
    g, o = both(c, 2)
    assert np.array_equal(g.get_state(0), o.get_state(0))


@pytest.mark.parametrize("tile", [0, 1, 2, 3])
def test_ragged_block_every_tile_exact(tile):
    c = cases.shock_tube((37, 19, 11), seed=2, reconstruct=abi.RECON_WENO, flux_split=abi.FLUX_ROE,
                         compat=abi.COMPAT_REFERENCE, rk_stages=4, timestep_set=abi.DT_CFL, cfl=0.4)
    o = c.apply(orc.Oracle(c.config()))
    o.step(3)
    for prec in (abi.PREC_FP64_EXACT,):
        g = Solver(c.config(precision=prec))
        c.apply(g, states=False)
        tuning.set_tuning(g, 0, tile, 0)
        g.set_state(0, c.states[0])
        g.step(3)
        assert np.array_equal(g.get_state(0), o.get_state(0))


def test_ragged_block_fp32_l1():
    c = cases.shock_tube((37, 19, 11), seed=2, reconstruct=abi.RECON_WENO, flux_split=abi.FLUX_AUSM,
                         compat=abi.COMPAT_TEXTBOOK, rk_stages=3, timestep_set=abi.DT_FIXED, dt=5e-4)
    o = c.apply(orc.Oracle(c.config()))
    o.step(5)
    for tile in range(4):
        g = Solver(c.config(precision=abi.PREC_FP32_FLUX))
        c.apply(g, states=False)
        tuning.set_tuning(g, 0, tile, 0)
        g.set_state(0, c.states[0])
        g.step(5)
        err = np.abs(g.get_state(0)[0] - o.get_state(0)[0]).mean()
        assert err <= 1e-6, (tile, err)


def test_error_paths():
    c = cases.shock_tube((8, 8, 8), seed=0, reconstruct=abi.RECON_MUSCL, flux_split=abi.FLUX_ROE,
                         limiter=abi.LIMITER_MINMOD, timestep_set=abi.DT_FIXED, dt=1e-3)
    s = Solver(c.config())
    b = s.add_block((8, 8, 8), (0.125, 0.125, 0.125))
    with pytest.raises(FvmError) as e:
        s.step(1)  # nothing uploaded
    assert e.value.code == 7  # FVM_ERR_STATE
    with pytest.raises(FvmError) as e:
        s.set_state(b + 5, np.zeros((5, 8, 8, 8)))
    assert e.value.code == 1  # FVM_ERR_INVALID
    s.set_state(b, c.states[0])
    s.step(1)
    with pytest.raises(FvmError) as e:
        s.set_boundary(b, 7, abi.BC_PERIODIC)
    assert e.value.code == 1
    # a state with zero density is reported, not propagated silently
    bad = c.states[0].copy()
    bad[0, 4, 4, 4] = 0.0
    s.set_state(b, bad)
    with pytest.raises(FvmError) as e:
        s.step(2)
    assert e.value.code == 4  # FVM_ERR_NONFINITE


def test_fast_fp64_reciprocals_within_2ulp():
    # the non-exact FP64 forms' reciprocal and reciprocal square root
    # (hardware approximation + one third-order correction) against correctly
    # rounded references (long double), over normal arguments whose results
    # are normal too
    import ctypes

    lib = abi.load_library()
    lib.fvm_test_fast_math.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]
    rng = np.random.default_rng(5)
    x = np.concatenate([10.0 ** rng.uniform(-300, 300, 200_000), rng.uniform(0.5, 2.0, 200_000),
                        np.nextafter(1.0, 2.0) + rng.uniform(0, 1e-12, 1000), 2.0 ** np.arange(-900, 901, 7),
                        [1.0, 1.4, 0.4, 1e-6, 3.0, 7.0]])
    r = np.empty_like(x)
    rs = np.empty_like(x)
    assert lib.fvm_test_fast_math(x.ctypes.data, x.size, r.ctypes.data, rs.ctypes.data) == 0
    xl = x.astype(np.longdouble)
    ref_r = (np.longdouble(1) / xl).astype(np.float64)
    ref_rs = (np.longdouble(1) / np.sqrt(xl)).astype(np.float64)
    ulp_r = np.abs(r - ref_r) / np.spacing(ref_r)
    ulp_rs = np.abs(rs - ref_rs) / np.spacing(ref_rs)
    assert ulp_r.max() <= 2.0, ulp_r.max()
    assert ulp_rs.max() <= 2.0, ulp_rs.max()


def test_multi_block_state_calls_match_per_block():
    # fvm_set_states / fvm_get_states (copies of consecutive blocks overlap the
    # unpacking) give exactly what per-block fvm_set_state / fvm_get_state
    # give, with the blocks in any order, repeated calls, and bad arguments
    # rejected before any copy
    c = cases.isentropic_vortex(N=24, layout="blocks8", precision=abi.PREC_FP32_FLUX)
    a = c.apply(Solver(c.config()))
    b = Solver(c.config())
    c.apply(b, states=False)
    order = [5, 0, 7, 2, 1, 6, 3, 4]
    b.set_states({k: c.states[k] for k in order})
    for s in (a, b):
        s.step(2)
    got = b.get_states(order)
    for k, g in zip(order, got):
        assert np.array_equal(g, a.get_state(k))
    b.set_states({k: got[i] for i, k in enumerate(order)})
    again = b.get_states(list(range(8)))
    for k in range(8):
        assert np.array_equal(again[k], a.get_state(k))
    with pytest.raises(FvmError) as e:
        b.get_states_ptr([0, 99], [again[0].ctypes.data, again[1].ctypes.data])
    assert e.value.code == 1
    b.set_states({})
    a.close()
    b.close()


def test_run_continues_from_the_current_step():
    # fvm_run's max_step counts the context's steps from its first one (the
    # reference's iteration counter): a second call continues, and a limit
    # already reached returns at once with no step
    c = cases.riemann2d(n=24, seed=1, dt=1e-3)
    g = c.apply(Solver(c.config()))
    o = c.apply(orc.Oracle(c.config()))
    assert g.run(max_step=3, total_time=1.0) == (3, abi.STOP_MAX_STEP)
    assert g.run(max_step=5, total_time=1.0) == (2, abi.STOP_MAX_STEP)
    assert g.run(max_step=4, total_time=1.0) == (0, abi.STOP_MAX_STEP)
    assert g.time()[2] == 5
    # a time limit already passed stops before any step as well
    assert g.run(total_time=1e-3) == (0, abi.STOP_MAX_TIME)
    n, why = g.run(total_time=7e-3)
    assert why == abi.STOP_MAX_TIME and g.time()[2] == 5 + n
    o.step(5 + n)
    assert np.array_equal(g.get_state(0), o.get_state(0))
