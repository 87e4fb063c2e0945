"""Golden fixtures (tests/golden/*.npz, written by tests/golden/make_golden.py
from the oracle): the oracle itself (CPU) and the GPU path's exact FP64 form
(through the C ABI) must reproduce each fixture's per-step time and residual
history, final state and last-stage rhs bit for bit.

tests/golden/riemann2d_reference_devlog.json holds what the reference's own
run of case/Riemann-2D.nml logged (its case/dev.log): the flow time after each
of 269 steps, printed to 17 significant digits, and the per-step structure of
the trace. The oracle and every GPU precision form must reach the same
doubles, and the configuration the tests rebuild for that case file must take
the steps the run took."""
import json
import os

import numpy as np
import pytest

import oracle as orc
from fvm3d import abi, cases
from fvm3d.solver import Solver

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

BUILDERS = {
    "riemann2d_reference": lambda: cases.riemann2d_reference(),
    "vortex16_blocks8": lambda: cases.isentropic_vortex(N=16, layout="blocks8"),
    "tgv12": lambda: cases.taylor_green(N=12),
}


def load(name):
    z = np.load(os.path.join(HERE, name + ".npz"))
    return json.loads(str(z["meta"])), {k: z[k] for k in z.files if k != "meta"}


def replay(case, steps, target, res_exact):
    """Steps `target` like the generator and compares as it goes."""
    _, gold = load(case._golden)
    for s in range(steps):
        r = target.step(1)
        assert r[0] == gold["t"][s], f"t at step {s + 1}"
        if res_exact:
            assert np.array_equal(np.asarray(r[1]), gold["res_abs"][s]), f"residuals at step {s + 1}"
        else:
            np.testing.assert_allclose(r[1], gold["res_abs"][s], rtol=1e-12, atol=0)
        if "kinetic_energy" in gold:
            q = target.get_state(0)
            dx = case.meta["dx"]
            assert cases.kinetic_energy(q, dx ** 3) == gold["kinetic_energy"][s]
            assert cases.enstrophy(q, dx) == gold["enstrophy"][s]
    for b in range(len(case.blocks)):
        assert np.array_equal(target.get_state(b), gold[f"q{b}"]), f"state of block {b}"
        assert np.array_equal(target.get_rhs(b), gold[f"rhs{b}"]), f"rhs of block {b}"


def build(name):
    meta, _ = load(name)
    case = BUILDERS[name]()
    case._golden = name
    cfg = case.config()
    for k, v in meta["config"].items():
        assert getattr(cfg, k) == v, f"{name}: config field {k} {getattr(cfg, k)} != {v}"
    return case, meta["steps"]


@pytest.mark.parametrize("name", sorted(BUILDERS))
def test_oracle_reproduces_golden(name):
    case, steps = build(name)
    o = case.apply(orc.Oracle(case.config()))
    replay(case, steps, o, res_exact=True)
    o.close()


def test_golden_riemann_matches_reference_case_file():
    # the fixture's configuration is the reference's case/Riemann-2D.nml
    # (gridSize 21, 21; MUSCL kappa 0.33333, minmod; Roe, entropy fix 0.2;
    # fixed dt 2e-4), with nk = 2 as the reference's 2D grid has
    meta, gold = load("riemann2d_reference")
    c = meta["config"]
    assert c["idimension"] == 2 and c["reconstruct"] == abi.RECON_MUSCL and c["limiter"] == abi.LIMITER_MINMOD
    assert c["kappa"] == 0.33333 and c["flux_split"] == abi.FLUX_ROE and c["entropy_fix"] == 0.2
    assert c["timestep_set"] == abi.DT_FIXED and c["dt"] == 2.0e-4 and c["rk_stages"] == 3
    assert gold["q0"].shape == (5, 2, 21, 21)
    assert np.isfinite(gold["res_abs"]).all()


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(BUILDERS))
def test_gpu_exact_reproduces_golden(name):
    case, steps = build(name)
    g = case.apply(Solver(case.config(store_rhs=1)))
    # the GPU sums residual norms in a different (deterministic) order
    replay(case, steps, g, res_exact=False)
    g.close()


def load_devlog():
    with open(os.path.join(HERE, "riemann2d_reference_devlog.json")) as f:
        return json.load(f)


def test_devlog_fixture_is_self_consistent():
    fx = load_devlog()
    # 17 significant digits: each printed string names exactly the double stored beside it
    assert [float(s) for s in fx["printed_time"]] == fx["time"]
    assert len(fx["time"]) == 269
    assert all(b > a for a, b in zip(fx["time"], fx["time"][1:]))


def test_reference_case_takes_the_steps_its_run_logged():
    # class_time_discret.f90:177,187 log each RK stage and block; class_space_discret.f90:132-173
    # each direction with its reconstruction and flux-split names
    fx = load_devlog()
    case = cases.riemann2d_reference()
    cfg = case.config()
    assert cfg.rk_stages == fx["rk_stages_per_step"] == 3
    assert cfg.idimension == len(fx["directions_per_stage"]) == 2
    assert fx["reconstruction"] == ["MUSCL"] and cfg.reconstruct == abi.RECON_MUSCL
    assert fx["flux_split"] == ["Roe"] and cfg.flux_split == abi.FLUX_ROE
    assert len(case.blocks) == len(fx["blocks"]) == 1
    assert fx["residual_computed_per_step"] == 1
    assert cfg.timestep_set == abi.DT_FIXED and cfg.dt == float(fx["dt_namelist"])


def test_oracle_time_history_matches_reference_run():
    # ClassTimeDiscret%solve: time = time + dt, then set_realtime logs it (class_time_discret.f90:142-144)
    fx = load_devlog()
    case = cases.riemann2d_reference()
    o = case.apply(orc.Oracle(case.config()))
    for s, want in enumerate(fx["time"]):
        t = o.step(1)[0]
        assert t == want, f"step {s}: {t!r} != {fx['printed_time'][s]}"
    o.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [abi.PREC_FP64_EXACT, abi.PREC_FP64, abi.PREC_FP32_FLUX])
def test_gpu_time_history_matches_reference_run(prec):
    fx = load_devlog()
    case = cases.riemann2d_reference()
    g = case.apply(Solver(case.config(precision=prec)))
    for s, want in enumerate(fx["time"]):
        t = g.step(1)[0]
        assert t == want, f"step {s}: {t!r} != {fx['printed_time'][s]}"
    g.close()
