"""Python mirror of the reference's solver objects over the C ABI.

``Solver`` plays the part of the reference's ``ClassSolver`` aggregate for the
explicit path (class_solver.f90: geometry / flowfield / spaceDiscr /
timeDiscr / iteration): blocks are added with their cell size, ghost regions
are transmissive, periodic or connected, the conservative state goes in and
out in the layout of ``ClassBlockData%get_q()`` and ``step`` replaces
``ClassTimeDiscret%solve`` (class_time_discret.f90:125-156). Every call goes
through libfvm3d.so; there is no Python or CPU compute path.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import abi


class FvmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{abi.STATUS.get(code, code)}: {msg}")
        self.code = code
        self.msg = msg


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Solver:
    """One case (a set of blocks with one scheme configuration) on the GPU."""

    def __init__(self, cfg: abi.FvmConfig | None = None, **kw):
        self.lib = abi.load_library()
        self.cfg = cfg if cfg is not None else abi.make_config(**kw)
        h = ctypes.c_void_p()
        rc = self.lib.fvm_create(ctypes.byref(self.cfg), ctypes.byref(h))
        if rc != 0:
            buf = ctypes.create_string_buffer(512)
            self.lib.fvm_last_error(None, buf, 512)
            raise FvmError(rc, buf.value.decode())
        self.h = h
        self.shapes: list[tuple[int, int, int]] = []

    # -- lifetime
    def close(self):
        if getattr(self, "h", None):
            self.lib.fvm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _chk(self, rc: int):
        if rc != 0:
            buf = ctypes.create_string_buffer(512)
            self.lib.fvm_last_error(self.h, buf, 512)
            raise FvmError(rc, buf.value.decode())

    # -- topology
    def add_block(self, nvert, dr) -> int:
        n = (ctypes.c_int64 * 3)(*[int(x) for x in nvert])
        d = (ctypes.c_double * 3)(*[float(x) for x in dr])
        b = ctypes.c_int()
        self._chk(self.lib.fvm_add_block(self.h, n, d, ctypes.byref(b)))
        while len(self.shapes) <= b.value:
            self.shapes.append(None)
        self.shapes[b.value] = tuple(int(x) for x in nvert)
        return b.value

    def set_boundary(self, blk: int, region: int, kind: int):
        self._chk(self.lib.fvm_set_boundary(self.h, blk, region, kind))

    def connect(self, blk, rng, donor, drng, dtype):
        r = (ctypes.c_int64 * 6)(*[int(x) for pair in rng for x in pair])
        d = (ctypes.c_int64 * 6)(*[int(x) for pair in drng for x in pair])
        t = (ctypes.c_int32 * 3)(*[int(x) for x in dtype])
        self._chk(self.lib.fvm_connect(self.h, blk, r, donor, d, t))

    # -- batched / served cases
    def reserve(self, cells: int):
        """Fix the state arena at `cells` padded cells per variable slab."""
        self._chk(self.lib.fvm_reserve(self.h, int(cells)))

    def add_case(self, cfg: abi.FvmConfig | None = None, **kw) -> int:
        c = cfg if cfg is not None else abi.make_config(**kw)
        cid = ctypes.c_int()
        self._chk(self.lib.fvm_add_case(self.h, ctypes.byref(c), ctypes.byref(cid)))
        return cid.value

    def add_case_block(self, case_id: int, nvert, dr) -> int:
        n = (ctypes.c_int64 * 3)(*[int(x) for x in nvert])
        d = (ctypes.c_double * 3)(*[float(x) for x in dr])
        b = ctypes.c_int()
        self._chk(self.lib.fvm_add_case_block(self.h, int(case_id), n, d, ctypes.byref(b)))
        while len(self.shapes) <= b.value:
            self.shapes.append(None)
        self.shapes[b.value] = tuple(int(x) for x in nvert)
        return b.value

    def remove_case(self, case_id: int):
        self._chk(self.lib.fvm_remove_case(self.h, int(case_id)))

    def case_state(self, case_id: int) -> dict:
        t = ctypes.c_double()
        dt = ctypes.c_double()
        st = ctypes.c_int64()
        ra = np.zeros(6)
        rr = np.zeros(6)
        status = ctypes.c_int()
        self._chk(self.lib.fvm_case_state(self.h, int(case_id), ctypes.byref(t), ctypes.byref(dt),
                                          ctypes.byref(st), _dp(ra), _dp(rr), ctypes.byref(status)))
        return {"t": t.value, "dt": dt.value, "step": st.value, "res_abs": ra, "res_rel": rr,
                "status": status.value}

    # -- state
    def _shape(self, blk: int):
        if not (0 <= blk < len(self.shapes)) or self.shapes[blk] is None:
            raise FvmError(1, "bad block id")  # FVM_ERR_INVALID, as the ABI reports it
        return self.shapes[blk]

    def set_state(self, blk: int, q: np.ndarray):
        """q: (5, nk, nj, ni) C-order, i.e. Fortran (ni,nj,nk,5)."""
        ni, nj, nk = self._shape(blk)
        a = np.ascontiguousarray(q, dtype=np.float64).reshape(5, nk, nj, ni)
        self._chk(self.lib.fvm_set_state(self.h, blk, _dp(a)))

    def set_state_ptr(self, blk: int, ptr: int):
        """Upload from a raw host pointer (e.g. pinned memory)."""
        self._chk(self.lib.fvm_set_state(self.h, blk, ctypes.cast(ptr, ctypes.POINTER(ctypes.c_double))))

    def get_state_ptr(self, blk: int, ptr: int):
        self._chk(self.lib.fvm_get_state(self.h, blk, ctypes.cast(ptr, ctypes.POINTER(ctypes.c_double))))

    def _many(self, fn, blks, ptrs):
        n = len(blks)
        ids = (ctypes.c_int * n)(*blks)
        arr = (ctypes.POINTER(ctypes.c_double) * n)(*[ctypes.cast(p, ctypes.POINTER(ctypes.c_double)) for p in ptrs])
        self._chk(fn(self.h, n, ids, arr))

    def set_states_ptr(self, blks, ptrs):
        """Upload several blocks in one call (fvm_set_states) from raw host
        pointers, e.g. pinned memory; copies overlap the unpacking."""
        self._many(self.lib.fvm_set_states, list(blks), list(ptrs))

    def get_states_ptr(self, blks, ptrs):
        """Download several blocks in one call (fvm_get_states)."""
        self._many(self.lib.fvm_get_states, list(blks), list(ptrs))

    def set_states(self, qs: dict):
        """Upload {block: q} with q as set_state takes it, in one call."""
        arrs = {}
        for blk, q in qs.items():
            ni, nj, nk = self._shape(blk)
            arrs[blk] = np.ascontiguousarray(q, dtype=np.float64).reshape(5, nk, nj, ni)
        self.set_states_ptr(list(arrs), [a.ctypes.data for a in arrs.values()])

    def get_states(self, blks) -> list:
        """The conservative states of blocks `blks`, in one call."""
        outs = []
        for blk in blks:
            ni, nj, nk = self._shape(blk)
            outs.append(np.empty((5, nk, nj, ni), dtype=np.float64))
        self.get_states_ptr(list(blks), [o.ctypes.data for o in outs])
        return outs

    def _get(self, fn, blk):
        ni, nj, nk = self._shape(blk)
        out = np.empty((5, nk, nj, ni), dtype=np.float64)
        self._chk(fn(self.h, blk, _dp(out)))
        return out

    def get_state(self, blk: int) -> np.ndarray:
        return self._get(self.lib.fvm_get_state, blk)

    def get_primitive(self, blk: int) -> np.ndarray:
        return self._get(self.lib.fvm_get_primitive, blk)

    def get_rhs(self, blk: int) -> np.ndarray:
        return self._get(self.lib.fvm_get_rhs, blk)

    # -- time stepping
    def step(self, nsteps: int = 1):
        """Advance nsteps; returns (t, res_abs[6], res_rel[6])."""
        t = ctypes.c_double()
        ra = np.zeros(6)
        rr = np.zeros(6)
        self._chk(self.lib.fvm_step(self.h, int(nsteps), ctypes.byref(t), _dp(ra), _dp(rr)))
        return t.value, ra, rr

    def run(self, max_step=10**10, total_time=0.0, absolute_residual=0.0, relative_residual=0.0):
        """Loop until ClassIteration%converged fires; returns (steps, reason)."""
        n = ctypes.c_int64()
        why = ctypes.c_int()
        self._chk(self.lib.fvm_run(self.h, int(max_step), float(total_time), float(absolute_residual),
                                   float(relative_residual), ctypes.byref(n), ctypes.byref(why)))
        return n.value, why.value

    def time(self):
        """(t, dt of the last step, step count)."""
        t = ctypes.c_double()
        dt = ctypes.c_double()
        s = ctypes.c_int64()
        self._chk(self.lib.fvm_get_time(self.h, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(s)))
        return t.value, dt.value, s.value
