"""ctypes binding of the CPU oracle (oracle/lib/libfvm_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py, as the checker. The product never imports it.
The oracle restates the reference's Fortran hot path; see fvm_oracle.cpp.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libfvm_oracle.so")
sys.path.insert(0, os.path.join(os.path.dirname(_HERE), "fvm-3d-f90_b200"))
from fvm3d.abi import FvmConfig, make_config  # noqa: E402

_lib = None


def build() -> str:
    subprocess.check_call(["make", "-s", "-C", _HERE], stdout=subprocess.DEVNULL)
    return LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        vp, i64, dbl, i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, ctypes.c_int32
        L.orc_create.restype = vp
        L.orc_create.argtypes = [P(FvmConfig)]
        L.orc_destroy.argtypes = [vp]
        L.orc_last_error.restype = ctypes.c_char_p
        L.orc_last_error.argtypes = [vp]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_max_threads.restype = ctypes.c_int
        L.orc_add_block.argtypes = [vp, P(i64), P(dbl)]
        L.orc_set_boundary.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_connect.argtypes = [vp, ctypes.c_int, P(i64), ctypes.c_int, P(i64), P(i32)]
        for n in ("orc_set_state", "orc_get_state", "orc_get_rhs", "orc_get_primitive",
                  "orc_get_ghost_state"):
            getattr(L, n).argtypes = [vp, ctypes.c_int, P(dbl)]
        L.orc_prepare.argtypes = [vp]
        L.orc_step.argtypes = [vp, ctypes.c_int, P(dbl), P(dbl), P(dbl), P(dbl)]
        L.orc_muscl_point.restype = dbl
        L.orc_muscl_point.argtypes = [dbl, dbl, dbl, ctypes.c_int, ctypes.c_int, dbl]
        L.orc_weno_point.restype = dbl
        L.orc_weno_point.argtypes = [P(dbl), ctypes.c_int]
        L.orc_flux_point.argtypes = [ctypes.c_int, ctypes.c_int, dbl, dbl, ctypes.c_int,
                                     P(dbl), P(dbl), P(dbl)]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def max_threads() -> int:
    return int(lib().orc_max_threads())


class Oracle:
    """A multi-block case on the CPU oracle, same calls as the product's Solver."""

    def __init__(self, cfg: FvmConfig | None = None, **kw):
        self.cfg = cfg if cfg is not None else make_config(**kw)
        self.L = lib()
        self.h = self.L.orc_create(ctypes.byref(self.cfg))
        self.shapes: list[tuple[int, int, int]] = []
        self._prepared = False

    def close(self):
        if self.h:
            self.L.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc):
        if rc != 0:
            raise RuntimeError(f"oracle error {rc}: {self.L.orc_last_error(self.h).decode()}")

    def add_block(self, nvert, dr) -> int:
        n = (ctypes.c_int64 * 3)(*[int(x) for x in nvert])
        d = (ctypes.c_double * 3)(*[float(x) for x in dr])
        b = self.L.orc_add_block(self.h, n, d)
        if b < 0:
            self._chk(-b)
        self.shapes.append(tuple(int(x) for x in nvert))
        return b

    def set_boundary(self, blk, region, kind):
        self._chk(self.L.orc_set_boundary(self.h, blk, region, kind))

    def connect(self, blk, rng, donor, drng, dtype):
        r = (ctypes.c_int64 * 6)(*[int(x) for pair in rng for x in pair])
        d = (ctypes.c_int64 * 6)(*[int(x) for pair in drng for x in pair])
        t = (ctypes.c_int32 * 3)(*[int(x) for x in dtype])
        self._chk(self.L.orc_connect(self.h, blk, r, donor, d, t))

    def set_state(self, blk, q: np.ndarray):
        """q: (5, nk, nj, ni) C-order == Fortran (ni,nj,nk,5)."""
        ni, nj, nk = self.shapes[blk]
        a = np.ascontiguousarray(q, dtype=np.float64).reshape(5, nk, nj, ni)
        self._chk(self.L.orc_set_state(self.h, blk, _dp(a)))
        self._prepared = False

    def _get(self, fn, blk):
        ni, nj, nk = self.shapes[blk]
        out = np.empty((5, nk, nj, ni), dtype=np.float64)
        self._chk(fn(self.h, blk, _dp(out)))
        return out

    def get_state(self, blk):
        return self._get(self.L.orc_get_state, blk)

    def get_rhs(self, blk):
        return self._get(self.L.orc_get_rhs, blk)

    def get_primitive(self, blk):
        self._prepare()
        return self._get(self.L.orc_get_primitive, blk)

    def get_ghost_state(self, blk):
        self._prepare()
        ni, nj, nk = self.shapes[blk]
        out = np.empty((5, nk + 6, nj + 6, ni + 6), dtype=np.float64)
        self._chk(self.L.orc_get_ghost_state(self.h, blk, _dp(out)))
        return out

    def _prepare(self):
        if not self._prepared:
            self._chk(self.L.orc_prepare(self.h))
            self._prepared = True

    def step(self, nsteps: int = 1):
        """Returns (t, res_abs[6], res_rel[6], dt_last)."""
        self._prepare()
        t = ctypes.c_double()
        dt = ctypes.c_double()
        ra = np.zeros(6)
        rr = np.zeros(6)
        self._chk(self.L.orc_step(self.h, int(nsteps), ctypes.byref(t), _dp(ra), _dp(rr),
                                  ctypes.byref(dt)))
        return t.value, ra, rr, dt.value


def muscl_point(p1, p2, p3, wind, limiter, kappa):
    return lib().orc_muscl_point(p1, p2, p3, wind, limiter, kappa)


def weno_point(u, compat=0):
    a = np.ascontiguousarray(u, dtype=np.float64)
    return lib().orc_weno_point(_dp(a), compat)


def flux_point(flux, dir, gamma, fix, L, R, compat=0):
    a = np.ascontiguousarray(L, dtype=np.float64)
    b = np.ascontiguousarray(R, dtype=np.float64)
    F = np.zeros(5)
    lib().orc_flux_point(flux, dir, gamma, fix, compat, _dp(a), _dp(b), _dp(F))
    return F
