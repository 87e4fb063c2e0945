"""Command-line front end: run a reference case file the way the reference's
executable does.

    python -m fvm3d --input=path/to/case.nml [--precision=exact|fp64|fp32]
                    [--output-dir=DIR] [--no-devlog]

The reference's main program (solver_sub.f90:80-207) takes the case file from
`--input` (class_input.f90:55-86), logs developer trace lines to dev.log in
the case file's directory (global_devlog.f90:48-80), prints a residual table
to the terminal every step (class_output.f90:414-463) and writes the flow
field at the output times. This front end does the same on the GPU path: the
steps run through libfvm3d.so, one step per call so the table and the trace
see every step; the flow field goes to VTK files (the CGNS library is not
available here) through fvm3d.output.

The dev.log lines that carry data are the reference's, character for
character: "Print residual step N" before each step and after the last one,
and "Flowfield real time T" with T printed as fortran-stdlib's to_string
prints a double (the library the reference formats numbers with; not part of
the reference tree). The stage lines name what runs on the GPU instead of
the reference's per-direction calls: one fused launch per RK stage for every
block, then the residual.
"""
from __future__ import annotations

import argparse
import datetime
import math
import os
import sys

from . import abi, namelist, output


def dp_to_string(x: float) -> str:
    """A double as the reference's dev.log prints it (fortran-stdlib
    to_string of a real(dp)): "0." then 17 significant digits, "E", the
    decimal exponent with its sign and no leading zeros, e.g.
    0.20000000000000001E-3 for 2e-4. The reference's case/dev.log pins this
    form for the positive values below one it holds."""
    if x == 0.0:
        return "0.0000000000000000E+0"
    if not math.isfinite(x):
        return "NaN" if math.isnan(x) else ("Infinity" if x > 0 else "-Infinity")
    mant, exp = f"{abs(x):.16e}".split("e")
    digits = mant.replace(".", "")
    e = int(exp) + 1
    return f"{'-' if x < 0 else ''}0.{digits}E{'-' if e < 0 else '+'}{abs(e)}"


class DevLog:
    """dev.log in the reference's line format: a list-directed write of
    "-- " and the message (a leading blank, then the text)."""

    def __init__(self, path: str | None):
        self.f = open(path, "w") if path else None

    def print(self, message: str = "") -> None:
        if self.f:
            self.f.write(f" -- {message}\n")

    def start(self) -> None:
        self.print()
        self.print("START SIMULATION: " + datetime.datetime.now().strftime("%Y%m%d %H:%M:%S"))
        self.print()

    def close(self) -> None:
        if self.f:
            self.f.close()
            self.f = None


# residual names of the Euler system and the total (ClassIteration's res_name,
# class_iteration.f90:122-129, from EqnResName, type_defs_equation.f90:163-184)
RES_NAMES = ["R_mass", "R_momx", "R_momy", "R_momz", "R_energy", "R_total"]


def residual_table(step: int, res, idimension: int, header: bool, out=sys.stdout) -> None:
    """The terminal residual table of the reference: a header at step 0, then
    the step and each residual as es18.10 (R_momz left out in 2D)."""
    keep = [i for i in range(6) if not (idimension == 2 and RES_NAMES[i] == "R_momz")]
    if header:
        cols = [f" {'Iter':>10}"] + [f" {RES_NAMES[i]:>14}" if j == 0 else f" {RES_NAMES[i]:>18}"
                                     for j, i in enumerate(keep)]
        out.write("".join(cols) + "\n")
    out.write(f" {step:>10}" + "".join(f" {float(res[i]):18.10E}" for i in keep) + "\n")


def run(argv=None, solver_cls=None, out=sys.stdout) -> int:
    ap = argparse.ArgumentParser(prog="python -m fvm3d", description=__doc__.split("\n\n")[0])
    ap.add_argument("--input", required=True, help="the case file (namelist)")
    ap.add_argument("--precision", choices=["exact", "fp64", "fp32"], default="exact",
                    help="exact: the reference's operation order, bit for bit (default); fp64: reassociated "
                         "FP64; fp32: FP32 reconstruction and fluxes, FP64 state")
    ap.add_argument("--output-dir", default=None, help="where dev.log and the flow field go (default: the "
                                                        "case file's directory)")
    ap.add_argument("--no-devlog", action="store_true")
    args = ap.parse_args(argv)

    from .solver import FvmError, Solver

    with open(args.input) as f:
        text = f.read()
    spec = namelist.parse_case(text)
    spec.config.precision = {"exact": abi.PREC_FP64_EXACT, "fp64": abi.PREC_FP64,
                             "fp32": abi.PREC_FP32_FLUX}[args.precision]
    outdir = args.output_dir or os.path.dirname(os.path.abspath(args.input))
    os.makedirs(outdir, exist_ok=True)
    log = DevLog(None if args.no_devlog else os.path.join(outdir, "dev.log"))
    log.start()
    recon = {abi.RECON_SIMPLE: "simple", abi.RECON_MUSCL: "MUSCL", abi.RECON_WENO: "WENO"}[spec.config.reconstruct]
    flux = {abi.FLUX_ROE: "Roe", abi.FLUX_VANLEER: "VanLeer", abi.FLUX_AUSM: "AUSM"}[spec.config.flux_split]

    s = (solver_cls or Solver)(spec.config)
    writer = None
    try:
        s.add_block(spec.nvert, spec.dr)
        s.set_state(0, namelist.initial_state(spec))
        if spec.output_vars:
            name = spec.solnfile or spec.name
            writer = output.SolutionWriter(os.path.join(outdir, name), spec.output_vars, spec.dr)
            writer.snapshot(s, 0.0, [0])
        time_out = spec.output_time
        step = 0

        def print_residual(res):
            log.print()
            log.print(f"Print residual step {step}")
            log.print()
            residual_table(step, res, spec.config.idimension, header=(step == 0), out=out)

        print_residual([0.0] * 6)
        reason = abi.STOP_NONE
        while reason == abi.STOP_NONE:
            # one step; a non-finite or diverged residual raises FvmError with
            # the reference's messages
            t, res_abs, res_rel = s.step(1)
            step += 1
            log.print(f"Flowfield real time {dp_to_string(t)}")
            for m in range(1, spec.config.rk_stages + 1):
                log.print(f"RK stage {m}")
                log.print(f"Fused stage launch: Reconstruction ({recon}), Flux split ({flux}), Update RHS, "
                          f"Time Stepping (Runge-Kutta), blocks 1..1")
            log.print("Compute residual")
            print_residual(res_abs)
            if writer and spec.output_time > 0 and abs(t - time_out) <= 1e-9:
                writer.snapshot(s, t, [0])
                time_out += spec.output_time
            elif writer and spec.output_time > 0 and t > time_out + 1e-9:
                time_out = float("inf")   # missed: the reference writes nothing more
            # ClassIteration%converged (class_iteration.f90:145-192), in its order
            if t > spec.total_time - 1.0e-10:
                reason = abi.STOP_MAX_TIME
            elif res_abs[5] < spec.absolute_residual:
                reason = abi.STOP_ABS_RESIDUAL
            elif res_rel[5] < spec.relative_residual:
                reason = abi.STOP_REL_RESIDUAL
    except FvmError as e:
        out.write(f"Error: {e}\n")
        return 1
    finally:
        if writer:
            writer.close()
        log.close()
        s.close()
    out.write({abi.STOP_MAX_TIME: " >> Reached the total time\n", abi.STOP_ABS_RESIDUAL: " >> Converged (absolute)\n",
               abi.STOP_REL_RESIDUAL: " >> Converged (relative)\n"}.get(reason, ""))
    return 0
