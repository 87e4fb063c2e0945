"""The library from a plain-C host: the header compiles as C99, a C program
links against libfvm3d.so, and (on a GPU) its results equal those of the
same run made through the Python bindings, bit for bit in exact mode."""
import os
import subprocess

import numpy as np
import pytest

from fvm3d import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c_driver", "fvm_c_driver.c")
LIBDIR = os.path.dirname(abi.LIB_PATH)


def build(tmp_path) -> str:
    exe = str(tmp_path / "fvm_c_driver")
    cmd = ["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-O2", "-I", os.path.join(ROOT, "include"),
           SRC, "-o", exe, "-L", LIBDIR, "-lfvm3d", "-lm", f"-Wl,-rpath,{LIBDIR}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_header_is_c99_and_a_c_host_links(tmp_path):
    build(tmp_path)


def parse(out: str):
    runs = {}
    lines = out.split()
    i = 0
    while i < len(lines):
        assert lines[i] == "case"
        case, what = int(lines[i + 1]), lines[i + 2]
        i += 3
        if what == "init":
            n = 5 * 20 * 12 * 9
            runs.setdefault(case, {})["init"] = np.array([float.fromhex(x) for x in lines[i:i + n]])
            i += n
        else:
            assert what == "t"
            r = runs[case]
            r["t"] = float.fromhex(lines[i])
            i += 1
            res = []
            for _ in range(6):
                assert lines[i] == "res"
                res.append(float.fromhex(lines[i + 1]))
                i += 2
            r["res"] = np.array(res)
            n = 5 * 20 * 12 * 9
            r["final"] = np.array([float.fromhex(x) for x in lines[i:i + n]])
            i += n
    return runs


@pytest.mark.gpu
def test_c_host_matches_python_bindings(tmp_path):
    from fvm3d.solver import Solver

    exe = build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    runs = parse(r.stdout)
    for pulse in (0, 1):
        cfg = abi.make_config(idimension=3, reconstruct=abi.RECON_WENO if pulse else abi.RECON_MUSCL,
                              limiter=abi.LIMITER_MINMOD, flux_split=abi.FLUX_AUSM if pulse else abi.FLUX_ROE,
                              rk_stages=4 if pulse else 3, timestep_set=abi.DT_CFL, cfl=0.4,
                              precision=abi.PREC_FP64_EXACT)
        s = Solver(cfg)
        b = s.add_block((20, 12, 9), (1.0 / 20, 1.0 / 12, 1.0 / 9))
        if pulse:
            for region in range(1, 7):
                s.set_boundary(b, region, abi.BC_PERIODIC)
        s.set_state(b, runs[pulse]["init"].reshape(5, 9, 12, 20))
        t, ra, _ = s.step(4)
        got = s.get_state(b).reshape(-1)
        s.close()
        assert t == runs[pulse]["t"]
        assert np.array_equal(ra, runs[pulse]["res"])
        assert np.array_equal(got, runs[pulse]["final"])


def test_fortran_module_binds_header_functions():
    # every bind(c) interface of the Fortran module names a function of
    # include/fvm3d.h and has the C prototype's number of arguments (no
    # Fortran compiler here, so the module is checked against the header)
    import re

    f90 = open(os.path.join(ROOT, "fvm-3d-f90_b200", "fortran", "fvm3d_c.f90")).read()
    hdr = open(os.path.join(ROOT, "include", "fvm3d.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    protos = {m.group(1): m.group(2) for m in re.finditer(r"\bint\s+(fvm_\w+)\s*\(([^)]*)\)\s*;", hdr)}
    binds = re.findall(r"function\s+(\w+)\s*\(([^)]*)\)\s*&?\s*(?:\n\s*)?bind\(c,\s*name=\"(\w+)\"\)", f90)
    assert len(binds) >= 15
    for fname, fargs, cname in binds:
        assert fname == cname
        assert cname in protos, cname
        n_f = len([a for a in fargs.split(",") if a.strip()])
        c_args = protos[cname].strip()
        n_c = 0 if c_args in ("", "void") else len(c_args.split(","))
        assert n_f == n_c, (cname, n_f, n_c)


SERVE_SRC = os.path.join(ROOT, "tests", "c_driver", "fvm_c_serve.c")


def build_serve(tmp_path) -> str:
    exe = str(tmp_path / "fvm_c_serve")
    cmd = ["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-O2", "-I", os.path.join(ROOT, "include"),
           SERVE_SRC, "-o", exe, "-L", LIBDIR, "-lfvm3d", "-lm", f"-Wl,-rpath,{LIBDIR}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_serving_c_host_links(tmp_path):
    build_serve(tmp_path)


@pytest.mark.gpu
def test_c_host_serves_three_requests(tmp_path):
    # fvm_case_submit / fvm_wait / fvm_poll / fvm_fetch_state / fvm_release
    # from C: an Euler RK3, an Euler RK4 (second engine) and a Navier-Stokes
    # request served together, each bit-identical to its run alone
    exe = build_serve(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "served 3 requests" in r.stdout
