"""C ABI checks that need no GPU: the library loads, exports every symbol
include/fvm3d.h declares, and validates configuration and topology on the
host before any CUDA call (the reference's mpi%stop("Invalid ...") checks)."""
import ctypes
import os
import subprocess

import pytest

from fvm3d import abi
from fvm3d.solver import FvmError, Solver

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fvm3d.h")


def test_library_exports_every_declared_symbol():
    lib = abi.load_library()
    declared = abi.declared_symbols(HEADER)
    assert "fvm_step" in declared and "fvm_connect" in declared
    out = subprocess.check_output(["nm", "-D", "--defined-only", abi.LIB_PATH]).decode()
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [s for s in declared if s not in exported]
    assert not missing, missing
    for s in declared:
        getattr(lib, s)


def test_abi_version_and_defaults():
    lib = abi.load_library()
    assert lib.fvm_abi_version() == 1
    c = abi.FvmConfig()
    assert lib.fvm_config_default(ctypes.byref(c)) == 0
    assert c.struct_size == ctypes.sizeof(abi.FvmConfig)
    assert c.kappa == -1.0 and c.entropy_fix == 0.05 and c.gamma == 1.4
    assert c.limiter == abi.SCHEME_NULL and c.rk_stages == 3


@pytest.mark.parametrize("kw,code", [
    (dict(idimension=1), 1),
    (dict(reconstruct=abi.RECON_WCNS), 8),
    (dict(reconstruct=999), 1),
    (dict(flux_split=abi.FLUX_HLLC), 8),
    (dict(flux_split=abi.SCHEME_NULL), 1),
    (dict(limiter=254), 1),
    (dict(time_scheme=abi.TIME_BDF1), 8),
    (dict(rk_stages=2), 1),
    (dict(timestep_set=abi.DT_CFL, cfl=0.0), 1),
    (dict(dt=-1.0), 1),
    (dict(gamma=1.0), 1),
    (dict(precision=7), 1),
    (dict(equation=abi.EQ_NAVIER_STOKES, prandtl=0.0), 1),
])
def test_config_validation(kw, code):
    with pytest.raises(FvmError) as e:
        Solver(**kw)
    assert e.value.code == code


def test_struct_size_checked():
    lib = abi.load_library()
    c = abi.make_config()
    c.struct_size = 12
    h = ctypes.c_void_p()
    assert lib.fvm_create(ctypes.byref(c), ctypes.byref(h)) == 1


def test_topology_validation_without_gpu():
    s = Solver(idimension=3)
    b0 = s.add_block((8, 8, 8), (0.1, 0.1, 0.1))
    b1 = s.add_block((8, 4, 8), (0.1, 0.1, 0.1))
    with pytest.raises(FvmError):
        s.add_block((0, 8, 8), (0.1, 0.1, 0.1))
    with pytest.raises(FvmError):
        s.add_block((8, 8, 8), (0.1, -1.0, 0.1))
    with pytest.raises(FvmError):
        s.set_boundary(b0, 7, abi.BC_PERIODIC)
    with pytest.raises(FvmError):
        s.set_boundary(5, 1, abi.BC_PERIODIC)
    s.set_boundary(b0, 1, abi.BC_PERIODIC)
    # donor type must be a signed permutation
    with pytest.raises(FvmError):
        s.connect(b0, ((8, 10), (0, 7), (0, 7)), b1, ((0, 2), (0, 7), (0, 7)), (1, 1, 3))
    # extent mismatch
    with pytest.raises(FvmError):
        s.connect(b0, ((8, 10), (0, 3), (0, 7)), b1, ((0, 2), (0, 2), (0, 7)), (1, 2, 3))
    # donor outside its real cells
    with pytest.raises(FvmError):
        s.connect(b0, ((8, 10), (0, 7), (0, 7)), b1, ((0, 2), (0, 7), (0, 7)), (1, 2, 3))
    # not a ghost box
    with pytest.raises(FvmError):
        s.connect(b0, ((0, 2), (0, 3), (0, 7)), b1, ((0, 2), (0, 3), (0, 7)), (1, 2, 3))
    # beyond three ghost layers
    with pytest.raises(FvmError):
        s.connect(b0, ((8, 11), (0, 3), (0, 7)), b1, ((0, 3), (0, 3), (0, 7)), (1, 2, 3))
    # a valid one (axis reversal along j)
    s.connect(b0, ((8, 10), (0, 3), (0, 7)), b1, ((0, 2), (3, 0), (0, 7)), (1, -2, 3))
    s.close()


def test_2d_k_regions_stay_transmissive():
    s = Solver(idimension=2)
    b = s.add_block((8, 8, 1), (0.1, 0.1, 1.0))
    with pytest.raises(FvmError):
        s.set_boundary(b, 5, abi.BC_PERIODIC)
    s.set_boundary(b, 1, abi.BC_PERIODIC)
    s.close()


def test_last_error_message():
    with pytest.raises(FvmError) as e:
        Solver(reconstruct=abi.RECON_WCNS)
    assert "WCNS" in e.value.msg


def test_struct_layouts_match_the_header(tmp_path):
    # the ctypes mirrors of the header's structs have the C compiler's sizes
    # and field offsets
    src = tmp_path / "layout.c"
    fields = {
        "fvm_config": (abi.FvmConfig, ["struct_size", "store_rhs", "kappa", "prandtl"]),
        "fvm_server_config": (abi.ServerConfig, ["chunk_steps", "budget_cells", "max_active_cells", "max_queued"]),
        "fvm_connection": (abi.Connection, ["donor", "range", "donor_range", "donor_type"]),
        "fvm_request": (abi.Request, ["nblocks", "cfg", "nvert", "dr", "q", "nbc", "nconn", "bc", "conn", "steps"]),
    }
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "fvm3d.h"', "int main(void) {"]
    for st, (_, fs) in fields.items():
        lines.append(f'  printf("{st} size %zu\\n", sizeof({st}));')
        for f in fs:
            lines.append(f'  printf("{st} {f} %zu\\n", offsetof({st}, {f}));')
    lines.append("  return 0;\n}")
    src.write_text("\n".join(lines))
    exe = str(tmp_path / "layout")
    subprocess.check_call(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", exe])
    out = subprocess.check_output([exe]).decode().split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for st, (cls, fs) in fields.items():
        assert got[(st, "size")] == ctypes.sizeof(cls), st
        for f in fs:
            assert got[(st, f)] == getattr(cls, f).offset, (st, f)
