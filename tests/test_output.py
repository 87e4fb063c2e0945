"""Solution output (the reference's CGNS snapshots, written as VTK XML)."""
import numpy as np
import pytest

from fvm3d import abi, output
from fvm3d.namelist import parse_case

from test_namelist import CASE


def test_output_variables_follow_the_group():
    spec = parse_case(CASE)  # the test case switches on Density only
    assert spec.output_vars == ("Density",)
    g = {"Density": ".true.", "VelocityX": ".false.", "Pressure": "T", "Temperature": ".TRUE."}
    assert output.output_variables(g) == ["Density", "Pressure", "Temperature"]


def test_vts_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    prim = rng.uniform(0.5, 2.0, size=(5, 3, 4, 6))
    path = str(tmp_path / "b.vts")
    names = ["Density", "VelocityY", "Pressure", "Temperature"]
    output.write_vts(path, prim, names, dr=(0.1, 0.2, 0.3), origin=(1.0, 0.0, -1.0))
    back = output.read_vts(path)
    assert np.array_equal(back["Density"], prim[0])
    assert np.array_equal(back["VelocityY"], prim[2])
    assert np.array_equal(back["Pressure"], prim[4])
    assert np.array_equal(back["Temperature"], prim[4] / prim[0])
    pts = back["Points"]
    assert pts.shape == (3, 4, 6, 3)
    assert pts[2, 3, 5, 0] == pytest.approx(1.0 + 0.5) and pts[2, 3, 5, 1] == pytest.approx(0.6)
    assert pts[2, 3, 5, 2] == pytest.approx(-1.0 + 0.6)
    text = open(path, "rb").read()
    assert text.startswith(b'<?xml version="1.0"?>') and text.rstrip().endswith(b"</VTKFile>")


class _FakeSolver:
    def __init__(self, prims):
        self.prims = prims

    def get_primitive(self, b):
        return self.prims[b]


def test_writer_collection(tmp_path):
    prims = [np.full((5, 2, 2, 2), float(b + 1)) for b in range(2)]
    w = output.SolutionWriter(str(tmp_path / "run" / "case"), ["Density"], (1.0, 1.0, 1.0))
    w.snapshot(_FakeSolver(prims), 0.0, [0, 1])
    w.snapshot(_FakeSolver(prims), 0.25, [0, 1])
    pvd = w.close()
    text = open(pvd).read()
    assert text.count("<DataSet") == 4 and 'timestep="0.25" part="1" file="case_b1_0001.vts"' in text
    assert np.array_equal(output.read_vts(str(tmp_path / "run" / "case_b1_0001.vts"))["Density"], prims[1][0])


@pytest.mark.gpu
def test_run_case_writes_snapshots(tmp_path):
    from fvm3d.namelist import run_case

    text = CASE.replace("output_time  = 0.01", "output_time  = 0.002").replace(
        "Density   = .true.", "Density   = .true.\n  Pressure  = .true.")
    s, spec, steps, reason = run_case(text, output_prefix=str(tmp_path / "q"))
    assert reason == abi.STOP_MAX_TIME and steps == 5
    pvd = open(tmp_path / "q.pvd").read()
    # t = 0, 0.002, 0.004 (0.006 is past the end)
    assert pvd.count("<DataSet") == 3
    last = output.read_vts(str(tmp_path / "q_b0_0002.vts"))
    assert set(last) == {"Density", "Pressure", "Points"}
    assert np.isfinite(last["Density"]).all() and (last["Density"] > 0).all()
