"""Tile-shape / z-chunk / tail-split autotuner of the fused stage kernel.

The stage kernel is compiled for a small set of tile shapes (TX x TY column
tiles) and marches each tile over a z chunk of runtime length; in 3D the
tasks of the work queue's last, partial round can be cut into shorter
pieces (tail split). The best combination depends on the scheme, the
precision and the block sizes; tuning times one full graph-captured step per
candidate on the case itself and caches the winner per (scheme, precision,
size bucket), so the tiling of a case never depends on the other cases it
is batched with.
"""
from __future__ import annotations

import ctypes
import json
import os

from . import abi

_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "csrc", "lib", "tuning_cache.json")


def _lib():
    lib = abi.load_library()
    if not hasattr(lib, "_fvm_tuning_declared"):
        lib.fvm_tune_set.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        lib.fvm_tune_set_tail_split.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        lib.fvm_tune_time_step.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
        lib.fvm_profile_step.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float),
                                         ctypes.POINTER(ctypes.c_int32), ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        lib.fvm_kernel_launches_per_step.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
        lib._fvm_tuning_declared = True
    return lib


def set_tuning(solver, case_id: int, tile: int, zchunk: int) -> None:
    rc = _lib().fvm_tune_set(solver.h, case_id, tile, zchunk)
    solver._chk(rc)


def set_tail_split(solver, case_id: int, split: int) -> None:
    solver._chk(_lib().fvm_tune_set_tail_split(solver.h, case_id, split))


def time_step(solver, reps: int = 5) -> float:
    ms = ctypes.c_float()
    solver._chk(_lib().fvm_tune_time_step(solver.h, reps, ctypes.byref(ms)))
    return ms.value


KIND_NAMES = {1: "stage", 2: "gather", 3: "viscous", 4: "finalize"}


def profile_step(solver):
    """One step launched kernel by kernel; returns [(kind_name, ms)]."""
    cap = 256
    ms = (ctypes.c_float * cap)()
    kinds = (ctypes.c_int32 * cap)()
    n = ctypes.c_int()
    solver._chk(_lib().fvm_profile_step(solver.h, ms, kinds, cap, ctypes.byref(n)))
    return [(KIND_NAMES.get(kinds[i], "?"), ms[i]) for i in range(n.value)]


def launches_per_step(solver) -> int:
    n = ctypes.c_int()
    solver._chk(_lib().fvm_kernel_launches_per_step(solver.h, ctypes.byref(n)))
    return n.value


def size_bucket(ncells: int) -> int:
    b = 0
    while (1 << (b + 1)) <= max(1, ncells):
        b += 1
    return b


def key(cfg, ncells: int) -> str:
    return f"{cfg.idimension}:{cfg.reconstruct}:{cfg.flux_split}:{cfg.compat}:{cfg.precision}:{size_bucket(ncells)}"


def load_cache() -> dict:
    try:
        with open(_CACHE) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def save_cache(c: dict) -> None:
    os.makedirs(os.path.dirname(_CACHE), exist_ok=True)
    with open(_CACHE, "w") as f:
        json.dump(c, f, indent=1, sort_keys=True)


def autotune(solver, ncells: int, zchunks=(0, 8, 16, 32, 64), tiles=(0, 1, 2, 3), splits=(1, 2, 3, 4), reps: int = 3,
             use_cache=True):
    """Pick (tile, zchunk, tail split) for case 0 of `solver` (state already
    uploaded). Returns (tile, zchunk, ms_per_step, split). Stepping during the
    search advances the state; callers re-upload it afterwards."""
    k = key(solver.cfg, ncells)
    cache = load_cache() if use_cache else {}
    if k in cache:
        t, z, ms = cache[k][:3]
        sp = cache[k][3] if len(cache[k]) > 3 else 1
        set_tuning(solver, 0, t, z)
        set_tail_split(solver, 0, sp)
        return t, z, ms, sp
    best = None
    three_d = solver.cfg.idimension == 3
    for t in tiles:
        for z in (zchunks if three_d else (0,)):
            for sp in (splits if three_d else (1,)):
                set_tuning(solver, 0, t, z)
                set_tail_split(solver, 0, sp)
                time_step(solver, 1)  # warm-up
                ms = time_step(solver, reps)
                if best is None or ms < best[2]:
                    best = (t, z, ms, sp)
    set_tuning(solver, 0, best[0], best[1])
    set_tail_split(solver, 0, best[3])
    if use_cache:
        cache[k] = list(best)
        save_cache(cache)
    return best
