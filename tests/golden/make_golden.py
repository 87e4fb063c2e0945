"""Writes the golden fixtures of tests/golden/ from the CPU oracle.

    python tests/golden/make_golden.py

Each fixture is a seeded case run on the oracle (the C++ restatement of the
reference's explicit step, oracle/fvm_oracle.cpp) with its per-step time and
residual history and its final state (and last-stage rhs). The tests check
that the oracle and the GPU path's exact FP64 form still reproduce them bit
for bit, so a change that moved both together would not pass unnoticed.

Cases:
  * riemann2d_reference: the reference's own case file case/Riemann-2D.nml
    (21 x 21 nodes, nk = 2, MUSCL kappa 0.33333 / minmod, Roe with entropy fix
    0.2, fixed dt 2e-4) with the initial condition hard-coded in
    class_flow_field.f90:207-243; 100 steps. When the reference tree is
    present, the configuration is parsed from that file with the namelist
    front end and must equal the one the tests rebuild without it.
  * vortex16_blocks8: the isentropic vortex on 16^3 cells in the 8 uneven
    periodic blocks, WENO5 (reference variant) + AUSM, classic RK4, CFL 0.5;
    10 steps.
  * tgv12: the Navier-Stokes Taylor-Green vortex on 12^3 cells, MUSCL /
    Van Albada + Roe, central viscous fluxes, SSP-RK3, CFL 0.5; 8 steps, with
    kinetic-energy and enstrophy histories.

One fixture comes from the reference itself rather than the oracle:
  * riemann2d_reference_devlog.json: what the reference's own run of
    case/Riemann-2D.nml logged in case/dev.log (written by global_devlog from
    class_flow_field.f90:321 and class_time_discret.f90:177,187): the flow
    time after each step as printed (17 significant digits, so each string
    names one double), and the trace lines counted per step (RK stages,
    directions, reconstruction and flux-split names, blocks). It is written
    only when the reference tree is present.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "fvm-3d-f90_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as orc  # noqa: E402
from fvm3d import cases  # noqa: E402
from fvm3d.namelist import parse_case  # noqa: E402

REFERENCE_CASE = "/root/reference/case/Riemann-2D.nml"
REFERENCE_DEVLOG = "/root/reference/case/dev.log"

# name -> (case builder, steps)
FIXTURES = {
    "riemann2d_reference": (lambda: cases.riemann2d_reference(), 100),
    "vortex16_blocks8": (lambda: cases.isentropic_vortex(N=16, layout="blocks8"), 10),
    "tgv12": (lambda: cases.taylor_green(N=12), 8),
}

CFG_FIELDS = ("idimension", "equation", "reconstruct", "limiter", "flux_split", "time_scheme", "rk_stages",
              "timestep_set", "compat", "precision", "kappa", "entropy_fix", "gamma", "dt", "cfl", "mu", "prandtl")


def config_dict(cfg) -> dict:
    return {k: getattr(cfg, k) for k in CFG_FIELDS}


def run(case, steps, target):
    """Per-step (t, res_abs[6]) history, then final states / rhs; for a
    single-block periodic case also the kinetic energy and enstrophy."""
    hist_t, hist_r, ke, en = [], [], [], []
    for _ in range(steps):
        r = target.step(1)
        hist_t.append(r[0])
        hist_r.append(np.asarray(r[1], dtype=np.float64))
        if case.name.startswith("tgv"):
            q = target.get_state(0)
            dx = case.meta["dx"]
            ke.append(cases.kinetic_energy(q, dx ** 3))
            en.append(cases.enstrophy(q, dx))
    nb = len(case.blocks)
    out = {"t": np.array(hist_t), "res_abs": np.array(hist_r)}
    for b in range(nb):
        out[f"q{b}"] = target.get_state(b)
        out[f"rhs{b}"] = target.get_rhs(b)
    if ke:
        out["kinetic_energy"] = np.array(ke)
        out["enstrophy"] = np.array(en)
    return out


def devlog_fixture(path):
    """The reference run's log as a fixture: printed flow times, in step
    order, and the per-step structure of its trace lines."""
    with open(path) as f:
        lines = [ln.strip() for ln in f.read().splitlines()]
    times = [ln.split("Flowfield real time", 1)[1].strip() for ln in lines if "Flowfield real time" in ln]
    steps = [int(ln.split("Print residual step", 1)[1]) for ln in lines if "Print residual step" in ln]
    assert steps == list(range(len(times))), "one time line per printed step"
    # the trace of one complete step (step 0, up to the next step's header)
    first = lines.index("-- Print residual step 0")
    nxt = lines.index("-- Print residual step 1")
    step0 = [ln for ln in lines[first:nxt] if ln != "--"]
    return {
        "source": "case/dev.log of the reference (its own run of case/Riemann-2D.nml)",
        "dt_namelist": "2.0E-4",
        "printed_time": times,
        "time": [float(t) for t in times],
        "rk_stages_per_step": sum(1 for ln in step0 if ln.startswith("-- RK stage")),
        "directions_per_stage": sorted({int(ln.split(":")[1]) for ln in step0 if ln.startswith("-- Direction:")}),
        "reconstruction": sorted({ln.split("(")[1].rstrip(")") for ln in step0 if ln.startswith("-- Reconstruction")}),
        "flux_split": sorted({ln.split("(")[1].rstrip(")") for ln in step0 if ln.startswith("-- Flux split")}),
        "blocks": sorted({ln.rsplit(" ", 1)[1] for ln in step0 if ln.startswith("-- Time Stepping")}),
        "residual_computed_per_step": sum(1 for ln in step0 if ln == "-- Compute residual"),
    }


def main():
    if os.path.exists(REFERENCE_DEVLOG):
        fx = devlog_fixture(REFERENCE_DEVLOG)
        path = os.path.join(HERE, "riemann2d_reference_devlog.json")
        with open(path, "w") as f:
            json.dump(fx, f, indent=1)
            f.write("\n")
        print(f"{path}: {len(fx['time'])} printed flow times")
    if os.path.exists(REFERENCE_CASE):
        with open(REFERENCE_CASE) as f:
            spec = parse_case(f.read())
        want = config_dict(cases.riemann2d_reference().config())
        got = config_dict(spec.config)
        assert got == want, (got, want)
        assert spec.nvert == (21, 21, 2), spec.nvert
        print("Riemann-2D.nml parses to the riemann2d_reference configuration")
    for name, (build, steps) in FIXTURES.items():
        case = build()
        o = case.apply(orc.Oracle(case.config()))
        out = run(case, steps, o)
        o.close()
        meta = {"case": case.name, "steps": steps, "config": config_dict(case.config()),
                "generator": "oracle/fvm_oracle.cpp via tests/golden/make_golden.py"}
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, meta=np.array(json.dumps(meta)), **out)
        print(f"{path}: {os.path.getsize(path)} bytes, t = {out['t'][-1]:.6g}")


if __name__ == "__main__":
    main()
