"""Batched cases in one engine and the continuous-batching server."""
import numpy as np
import pytest

import oracle as orc
from fvm3d import abi, cases, serving
from fvm3d.solver import FvmError, Solver

pytestmark = pytest.mark.gpu


def alone(case, steps):
    s = case.apply(Solver(case.config()))
    s.step(steps)
    out = [s.get_state(b) for b in range(len(case.blocks))]
    s.close()
    return out


def trio():
    a = cases.blast((24, 20, 16), seed=1, reconstruct=abi.RECON_MUSCL, flux_split=abi.FLUX_ROE,
                    limiter=abi.LIMITER_MINMOD, kappa=1.0 / 3.0)
    b = cases.shock_tube((16, 24, 20), seed=2, reconstruct=abi.RECON_WENO, flux_split=abi.FLUX_AUSM)
    c = cases.isentropic_vortex(N=16, layout="blocks8", rk_stages=3, reconstruct=abi.RECON_SIMPLE,
                                flux_split=abi.FLUX_VANLEER)
    return [a, b, c]


def test_batch_equals_alone_and_oracle():
    cs = trio()
    s = Solver(cs[0].config())
    s.remove_case(0)
    ids = []
    for c in cs:
        cid = s.add_case(c.config())
        c.apply(s, case_id=cid)
        ids.append(list(c.block_ids))
    s.step(4)
    for c, bid in zip(cs, ids):
        ref = alone(c, 4)
        o = c.apply(orc.Oracle(c.config()))
        o.step(4)
        for b, g in enumerate(bid):
            got = s.get_state(g)
            assert np.array_equal(got, ref[b])
            assert np.array_equal(got, o.get_state(b))
    s.close()


def test_add_and_remove_between_steps():
    a, b, c = trio()
    s = Solver(a.config())
    s.remove_case(0)
    ca = s.add_case(a.config())
    a.apply(s, case_id=ca)
    cb = s.add_case(b.config())
    b.apply(s, case_id=cb)
    ids_b = list(b.block_ids)
    s.step(3)
    s.remove_case(ca)
    cc = s.add_case(c.config())
    c.apply(s, case_id=cc)
    ids_c = list(c.block_ids)
    s.step(2)
    ref_b = alone(b, 5)
    ref_c = alone(c, 2)
    for i, g in enumerate(ids_b):
        assert np.array_equal(s.get_state(g), ref_b[i])
    for i, g in enumerate(ids_c):
        assert np.array_equal(s.get_state(g), ref_c[i])
    assert s.case_state(cb)["step"] == 5 and s.case_state(cc)["step"] == 2
    s.close()


def test_reserved_budget_is_enforced():
    a, b, _ = trio()
    need = sum(abi.block_cells(3, n) for n, _ in a.blocks)
    s = Solver(a.config())
    s.remove_case(0)
    s.reserve(need)
    ca = s.add_case(a.config())
    a.apply(s, case_id=ca)
    cb = s.add_case(b.config())
    with pytest.raises(FvmError) as e:
        b.apply(s, case_id=cb)  # the upload plans the arena: no room
    assert e.value.code == 3
    s.close()


def _families_stream(n, seed, rate=1000.0):
    # the served families of the three solver configurations (2D Riemann,
    # 8-block vortex with RK4, Navier-Stokes TGV) and the batched blasts /
    # shock tubes, small grids, a few steps each
    fam = serving.config_families(precision=abi.PREC_FP32_FLUX, sizes=(12, 20))
    mix = serving.mixed_family(precision=abi.PREC_FP32_FLUX, sizes=(12, 24))
    make = lambda rng, i: fam(rng, i) if i % 3 else mix(rng, i)  # noqa: E731
    return serving.poisson_stream(n, rate=rate, seed=seed, make_case=make, steps=(3, 12))


def test_server_results_same_alone_and_in_the_mix():
    stream = _families_stream(9, seed=3)
    kinds = {r.case.name.split("_")[0] for r in stream}
    assert {"riemann2d", "vortex", "tgv"} <= kinds, kinds
    budget = 3 * max(sum(abi.block_cells(int(r.case.cfg.get("idimension", 3)), n) for n, _ in r.case.blocks)
                     for r in stream)
    srv = serving.Server(budget_cells=budget, chunk=4)
    stats = srv.run(stream, realtime=False)
    srv.close()
    assert stats["requests"] == 9 and stats["failed"] == 0
    assert stats["p99_s"] >= stats["p50_s"] > 0
    for r in stream:
        ref = alone(r.case, r.nsteps)
        for got, want in zip(r.result, ref):
            assert np.array_equal(got, want), f"request {r.rid} ({r.case.name})"


def test_server_admission_cap():
    stream = _families_stream(8, seed=4)
    srv0 = serving.Server(budget_cells=1 << 20)
    cells = [srv0.cells_of(r.case) for r in stream]
    srv0.close()
    cap = 2 * max(cells)
    srv = serving.Server(budget_cells=10 * max(cells), chunk=2, max_active_cells=cap)
    stats = srv.run(stream, realtime=False)
    peak = srv.stats()["peak_active_cells"]
    srv.close()
    assert stats["requests"] == 8 and stats["failed"] == 0
    assert 0 < peak <= cap


def test_server_error_codes():
    # FVM_ERR_NOT_FOUND for unknown / released ids, FVM_ERR_INVALID for a
    # request above the whole budget, FVM_ERR_BUSY for a full queue and for
    # reading an unfinished request
    a = cases.taylor_green(N=24)
    b = cases.blast((12, 12, 12), seed=0, limiter=abi.LIMITER_MINMOD, kappa=1.0 / 3.0)
    srv0 = serving.Server(budget_cells=1 << 20)
    ca, cb = srv0.cells_of(a), srv0.cells_of(b)
    srv0.close()
    srv = serving.Server(budget_cells=ca, chunk=1, max_queued=1)
    with pytest.raises(FvmError) as e:
        srv.poll(777)
    assert e.value.code == 10
    with pytest.raises(FvmError) as e:
        srv.submit(cases.taylor_green(N=40), 1)
    assert e.value.code == 1
    ra = srv.submit(a, 3000)
    import time

    t0 = time.time()
    while srv.poll(ra)["state"] == abi.REQ_QUEUED and time.time() - t0 < 30:
        time.sleep(0.001)
    assert srv.poll(ra)["state"] == abi.REQ_RUNNING
    assert cb <= ca
    rb = srv.submit(b, 2)                      # waits: the running TGV holds the whole budget
    with pytest.raises(FvmError) as e:
        srv.submit(b, 2)                       # max_queued = 1
    assert e.value.code == 9
    with pytest.raises(FvmError) as e:
        srv.fetch(ra, a)                       # still running
    assert e.value.code == 9
    assert srv.wait(ra) == abi.REQ_DONE, srv.poll(ra)
    assert srv.wait(rb) == abi.REQ_DONE, srv.poll(rb)
    assert srv.poll(ra)["steps_done"] == 3000
    srv.release(ra)
    with pytest.raises(FvmError) as e:
        srv.poll(ra)
    assert e.value.code == 10
    srv.close()


def test_navier_stokes_mixed_precisions_batched():
    # one engine holding a Navier-Stokes case of each precision form (three
    # viscous task lists, three viscous kernels) plus a 2D one: every case
    # matches its own run alone bit for bit, the exact one also the oracle
    forms = [abi.PREC_FP64_EXACT, abi.PREC_FP64, abi.PREC_FP32_FLUX]
    cs = [cases.taylor_green(N=16 + 4 * i, precision=p) for i, p in enumerate(forms)]
    cs.append(cases.riemann2d(n=27, seed=3, nk=2, dt=1e-3, equation=abi.EQ_NAVIER_STOKES, mu=5e-3))
    s = Solver(cs[0].config())
    s.remove_case(0)
    ids = []
    for c in cs:
        cid = s.add_case(c.config())
        c.apply(s, case_id=cid)
        ids.append(list(c.block_ids))
    s.step(3)
    for c, bid in zip(cs, ids):
        ref = alone(c, 3)
        for b, g in enumerate(bid):
            assert np.array_equal(s.get_state(g), ref[b])
    o = cs[0].apply(orc.Oracle(cs[0].config()))
    o.step(3)
    assert np.array_equal(s.get_state(ids[0][0]), o.get_state(0))
    s.close()


def test_running_case_unchanged_when_another_joins():
    # a case that is stepping keeps the dt its last step computed when the
    # engine re-plans for a joining case: 3 + 3 steps with a case added in
    # between equal 6 steps alone (CFL time step, FP64 and FP32 forms)
    for prec in (abi.PREC_FP64, abi.PREC_FP32_FLUX):
        a = cases.isentropic_vortex(N=16, layout="blocks8", rk_stages=3, precision=prec,
                                    timestep_set=abi.DT_CFL, cfl=0.5)
        b = cases.blast((16, 16, 16), seed=4, precision=prec)
        ref = alone(a, 6)
        s = Solver(a.config())
        s.remove_case(0)
        ca = s.add_case(a.config())
        a.apply(s, case_id=ca)
        ids = list(a.block_ids)
        s.step(3)
        cb = s.add_case(b.config())
        b.apply(s, case_id=cb)
        s.step(3)
        for k, g in enumerate(ids):
            assert np.array_equal(s.get_state(g), ref[k]), (prec, k)
        s.close()


def test_server_failing_request_does_not_disturb_the_others():
    # a request whose residual goes NaN (the reference WENO5 + AUSM on a
    # strong blast) ends FAILED with FVM_ERR_NONFINITE while the requests
    # served beside it finish and equal their runs alone
    bad = cases.blast((20, 20, 20), seed=0, reconstruct=abi.RECON_WENO, flux_split=abi.FLUX_AUSM)
    good = [cases.taylor_green(N=16), cases.riemann2d(n=40, seed=2, dt=1e-3)]
    srv = serving.Server(budget_cells=1 << 22, chunk=2)
    ids = [srv.submit(c, 6) for c in [good[0], bad, good[1]]]
    states = [srv.wait(i) for i in ids]
    assert states == [abi.REQ_DONE, abi.REQ_FAILED, abi.REQ_DONE], states
    assert srv.poll(ids[1])["status"] == 4
    for i, c in ((ids[0], good[0]), (ids[2], good[1])):
        got = srv.fetch(i, c)
        ref = alone(c, 6)
        for g, r in zip(got, ref):
            assert np.array_equal(g, r)
    srv.close()
