"""Namelist front end: the reference's parser rules and key mapping."""
import pytest

from fvm3d import abi
from fvm3d.namelist import NamelistError, parse_case, read_group

CASE = """
! a 2D four-quadrant case in the reference's case-file format
&General
  name          = "Quadrants"
  dimension     = "2D"
  dimensionless = .true.
  equation      = "Euler"
  gasModel      = "ideal"
/

&Geometry
  type      = "uniform"
  geoType   = "square"
  geoSize   = 1.0
  gridType  = "nodal-centered"
  gridSize  = 33, &
              33
  writeGrid = .false.
/

&Inviscid_Flux
  reconstruct   = "MUSCL"
  kappa         = 0.5
  limiter       = "vanAlbada_"
  flux_split    = "AUSM"
  entropy_fix   = 0.1
/

&Viscous_Flux
/

&Time_Stepping
  time_scheme  = "Runge-Kutta"
  timestep_set = "fixed"
  fix_timestep = 1.0E-3
  total_time   = 0.005
  output_time  = 0.01
  absolute_residual = 1.0E-12
  relative_residual = 1.0E-9
/

&Output
  format    = "CGNS"
  Density   = .true.
/
"""


def test_parse_maps_keys_to_config():
    spec = parse_case(CASE)
    c = spec.config
    assert spec.name == "Quadrants"
    assert c.idimension == 2 and c.equation == abi.EQ_EULER
    assert c.reconstruct == abi.RECON_MUSCL and c.limiter == abi.LIMITER_VANALBADA and c.kappa == 0.5
    assert c.flux_split == abi.FLUX_AUSM and c.entropy_fix == 0.1
    assert c.time_scheme == abi.TIME_RUNGE_KUTTA and c.timestep_set == abi.DT_FIXED and c.dt == 1e-3
    assert spec.nvert == (33, 33, 2)
    assert spec.dr == pytest.approx((1.0 / 32, 1.0 / 32, 1.0))
    assert spec.total_time == 0.005 and spec.absolute_residual == 1e-12 and spec.relative_residual == 1e-9


def test_continuation_and_quotes():
    g = read_group(CASE, "Geometry")
    assert g.get("gridSize").replace(" ", "") == "33,33"
    assert g.get("type") == "uniform"
    assert g.get("missing") == ""


def test_unused_key_is_an_error():
    bad = CASE.replace('  kappa         = 0.5', '  kappa         = 0.5\n  kapa = 1')
    with pytest.raises(NamelistError, match="Variable not defined in namelist: kapa"):
        parse_case(bad)


def test_format_error():
    bad = CASE.replace('  entropy_fix   = 0.1', '  entropy_fix 0.1')
    with pytest.raises(NamelistError, match="Format Error"):
        parse_case(bad)


def test_unknown_scheme_is_rejected():
    with pytest.raises(NamelistError, match="Invalid flux split scheme"):
        parse_case(CASE.replace('"AUSM"', '"Godunov"'))


def test_initial_state_outside_unit_square_is_rejected():
    from fvm3d.namelist import initial_state

    with pytest.raises(NamelistError, match="unit square"):
        initial_state(parse_case(CASE.replace("geoSize   = 1.0", "geoSize   = 2.0")))


def test_extension_group():
    ext = CASE + '\n&B200\n  precision = "fp32_flux"\n  compat = "textbook"\n  rk_stages = 4\n  nk = 1\n/\n'
    spec = parse_case(ext)
    assert spec.config.precision == abi.PREC_FP32_FLUX and spec.config.compat == abi.COMPAT_TEXTBOOK
    assert spec.config.rk_stages == 4 and spec.nvert[2] == 1


@pytest.mark.gpu
def test_run_case_matches_oracle():
    import numpy as np

    import oracle as orc
    from fvm3d.namelist import initial_state, run_case

    s, spec, steps, reason = run_case(CASE)
    assert reason == abi.STOP_MAX_TIME and steps == 5
    o = orc.Oracle(spec.config)
    o.add_block(spec.nvert, spec.dr)
    o.set_state(0, initial_state(spec))
    o.step(steps)
    assert np.array_equal(s.get_state(0), o.get_state(0))
