"""Command-line front end (python -m fvm3d --input=case.nml): the reference's
dev.log line format and number printing, checked against the log of the
reference's own run of case/Riemann-2D.nml (tests/golden/
riemann2d_reference_devlog.json), and, on the GPU, a whole run of that case
file through the CLI whose logged step and time lines must equal the
reference's."""
import io
import json
import os

import pytest

from fvm3d import cli

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "riemann2d_reference_devlog.json")

# The reference's case/Riemann-2D.nml settings (21 x 21 nodes, MUSCL kappa
# 0.33333 / minmod, Roe with entropy fix 0.2, fixed dt 2e-4), with the total
# time cut to the 269 steps its log records
RIEMANN_CASE = """
&General
  name = "Riemann-2D"
  dimension = "2D"
  dimensionless = .true.
  equation = "Euler"
  gasModel = "ideal"
/
&Geometry
  type = "uniform"
  geoType = "square"
  geoSize = 1.0
  gridType = "nodal-centered"
  gridSize = 21, 21
  writeGrid = .false.
/
&Inviscid_Flux
  reconstruct = "MUSCL"
  kappa = 0.33333
  limiter = "minmod_"
  flux_split = "Roe"
  entropy_fix = 0.2
/
&Viscous_Flux
/
&Time_Stepping
  time_scheme = "Runge-Kutta"
  timestep_set = "fixed"
  fix_timestep = 2.0E-4
  total_time = 0.0538
  output_time = 0.01
  absolute_residual = 1.0E-8
  relative_residual = 1.0E-6
/
&Boundary_Condition
/
&Initial_Condition
/
&Output
  format = "CGNS"
  Density = .true.
  VelocityX = .true.
  VelocityY = .true.
  Pressure = .true.
/
"""


def load():
    with open(GOLD) as f:
        return json.load(f)


def test_number_printing_matches_reference_log():
    fx = load()
    assert [cli.dp_to_string(t) for t in fx["time"]] == fx["printed_time"]
    assert cli.dp_to_string(-2.0e-4) == "-0.20000000000000001E-3"
    assert cli.dp_to_string(12.5) == "0.12500000000000000E+2"


def test_devlog_line_format(tmp_path):
    log = cli.DevLog(str(tmp_path / "dev.log"))
    log.print()
    log.print("Print residual step 0")
    log.close()
    assert (tmp_path / "dev.log").read_text() == " -- \n -- Print residual step 0\n"


def test_residual_table_layout():
    out = io.StringIO()
    cli.residual_table(0, [1.0, 2.0, 3.0, 4.0, 5.0, 6.0], 2, header=True, out=out)
    head, row = out.getvalue().splitlines()
    assert head.split() == ["Iter", "R_mass", "R_momx", "R_momy", "R_energy", "R_total"]   # no R_momz in 2D
    assert row.split() == ["0", "1.0000000000E+00", "2.0000000000E+00", "3.0000000000E+00", "5.0000000000E+00",
                           "6.0000000000E+00"]
    assert len(row) == 11 + 5 * 19


def test_cli_needs_input():
    with pytest.raises(SystemExit):
        cli.run([])


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["exact", "fp32"])
def test_cli_run_logs_the_reference_steps_and_times(tmp_path, precision):
    case = tmp_path / "Riemann-2D.nml"
    case.write_text(RIEMANN_CASE)
    out = io.StringIO()
    assert cli.run([f"--input={case}", f"--precision={precision}"], out=out) == 0
    fx = load()
    want = []
    for n, t in enumerate(fx["printed_time"]):
        want += [f" -- Print residual step {n}", f" -- Flowfield real time {t}"]
    got = [ln for ln in (tmp_path / "dev.log").read_text().splitlines()
           if "Print residual step" in ln or "Flowfield real time" in ln]
    assert got[:len(want)] == want
    assert got[len(want)] == " -- Print residual step 269"   # the run stops at the total time
    lines = (tmp_path / "dev.log").read_text().splitlines()
    step1 = lines[lines.index(" -- Print residual step 0") + 2:lines.index(" -- Print residual step 1") - 1]
    assert sum(1 for ln in step1 if ln.startswith(" -- RK stage")) == fx["rk_stages_per_step"]
    assert step1.count(" -- Compute residual") == 1
    table = out.getvalue().splitlines()
    assert table[0].split()[0] == "Iter" and table[-1].startswith(" >> Reached the total time")
    assert table[-2].split()[0] == "269"
    # the flow field at t = 0 and each output time 0.01 .. 0.05 it hits to 1e-9
    assert len([p for p in tmp_path.iterdir() if p.suffix == ".vts"]) == 6
    assert (tmp_path / "Riemann-2D.pvd").exists()
