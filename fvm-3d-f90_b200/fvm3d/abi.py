"""ctypes view of include/fvm3d.h and the loader of the in-tree CUDA library.

The library is ``csrc/lib/libfvm3d.so`` next to this package, built by
``__graft_entry__.build()`` (or ``make -C fvm-3d-f90_b200/csrc``).  Loading
fails loudly when it is missing: there is no CPU fallback for the product.
"""
from __future__ import annotations

import ctypes
import os

# ---- ids of include/fvm3d.h (TypeDefs%SchemeIndex, type_defs_scheme.f90:12-35)
SCHEME_NULL = -1
TIME_RUNGE_KUTTA = 101
TIME_BDF1 = 102
RECON_SIMPLE = 200
RECON_MUSCL = 201
RECON_WENO = 202
RECON_WCNS = 203
LIMITER_NONE = 250
LIMITER_MINMOD = 251
LIMITER_VANLEER = 252
LIMITER_VANALBADA = 253
FLUX_ROE = 300
FLUX_VANLEER = 301
FLUX_HLLC = 302
FLUX_AUSM = 303

DT_FIXED, DT_CFL, DT_CFL_LOCAL = 0, 1, 2
EQ_EULER, EQ_NAVIER_STOKES = 0, 1
COMPAT_REFERENCE, COMPAT_TEXTBOOK = 0, 1
PREC_FP64_EXACT, PREC_FP64, PREC_FP32_FLUX = 0, 1, 2
BC_TRANSMISSIVE, BC_PERIODIC, BC_CONNECTED = 0, 1, 2

STOP_NONE, STOP_MAX_STEP, STOP_MAX_TIME, STOP_ABS_RESIDUAL, STOP_REL_RESIDUAL = range(5)

STATUS = {
    0: "FVM_OK",
    1: "FVM_ERR_INVALID",
    2: "FVM_ERR_CUDA",
    3: "FVM_ERR_NOMEM",
    4: "FVM_ERR_NONFINITE",
    5: "FVM_ERR_DIVERGED",
    6: "FVM_ERR_TIMEOUT",
    7: "FVM_ERR_STATE",
    8: "FVM_ERR_UNSUPPORTED",
    9: "FVM_ERR_BUSY",
    10: "FVM_ERR_NOT_FOUND",
    11: "FVM_ERR_NEGATIVE",
}

# Namelist string -> id, exactly TypeDefs%SchemeIndex (type_defs_scheme.f90:41-84).
SCHEME_INDEX = {
    "Runge-Kutta": TIME_RUNGE_KUTTA,
    "BDF1": 102,
    "BDF2": 103,
    "BDF3": 104,
    "MEBDF4": 105,
    "SSPRK3": 106,
    "simple": RECON_SIMPLE,
    "MUSCL": RECON_MUSCL,
    "WENO": RECON_WENO,
    "WCNS": RECON_WCNS,
    "none_": LIMITER_NONE,
    "minmod_": LIMITER_MINMOD,
    "VanLeer_": LIMITER_VANLEER,
    "vanAlbada_": LIMITER_VANALBADA,
    "Roe": FLUX_ROE,
    "VanLeer": FLUX_VANLEER,
    "HLLC": FLUX_HLLC,
    "AUSM": FLUX_AUSM,
}


def scheme_index(name: str) -> int:
    """TypeDefs%SchemeIndex: unknown names give SCHEME_NULL (-1)."""
    return SCHEME_INDEX.get(name.strip(), SCHEME_NULL)


class FvmConfig(ctypes.Structure):
    """struct fvm_config of include/fvm3d.h."""

    _fields_ = [
        ("struct_size", ctypes.c_int32),
        ("idimension", ctypes.c_int32),
        ("equation", ctypes.c_int32),
        ("reconstruct", ctypes.c_int32),
        ("limiter", ctypes.c_int32),
        ("flux_split", ctypes.c_int32),
        ("time_scheme", ctypes.c_int32),
        ("rk_stages", ctypes.c_int32),
        ("timestep_set", ctypes.c_int32),
        ("compat", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("store_rhs", ctypes.c_int32),
        ("kappa", ctypes.c_double),
        ("entropy_fix", ctypes.c_double),
        ("gamma", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("cfl", ctypes.c_double),
        ("mu", ctypes.c_double),
        ("prandtl", ctypes.c_double),
    ]


def make_config(**kw) -> FvmConfig:
    """A config holding the reference's defaults (ClassSpaceDiscret:
    kappa -1, limiter NULL, entropy_fix 0.05; ClassFlowField gamma 1.4;
    3 RK stages, fixed dt), overridden by keyword arguments."""
    c = FvmConfig()
    c.struct_size = ctypes.sizeof(FvmConfig)
    c.idimension = 3
    c.equation = EQ_EULER
    c.reconstruct = RECON_MUSCL
    c.limiter = SCHEME_NULL
    c.flux_split = FLUX_ROE
    c.time_scheme = TIME_RUNGE_KUTTA
    c.rk_stages = 3
    c.timestep_set = DT_FIXED
    c.compat = COMPAT_REFERENCE
    c.precision = PREC_FP64_EXACT
    c.store_rhs = 0
    c.kappa = -1.0
    c.entropy_fix = 0.05
    c.gamma = 1.4
    c.dt = 0.0
    c.cfl = 0.5
    c.mu = 0.0
    c.prandtl = 0.71
    for k, v in kw.items():
        if not hasattr(c, k):
            raise KeyError(f"fvm_config has no field {k!r}")
        setattr(c, k, v)
    return c


class ServerConfig(ctypes.Structure):
    """struct fvm_server_config of include/fvm3d.h."""

    _fields_ = [
        ("struct_size", ctypes.c_int32),
        ("chunk_steps", ctypes.c_int32),
        ("budget_cells", ctypes.c_int64),
        ("max_active_cells", ctypes.c_int64),
        ("max_queued", ctypes.c_int32),
        ("pad_", ctypes.c_int32),
    ]


class Connection(ctypes.Structure):
    """struct fvm_connection of include/fvm3d.h."""

    _fields_ = [
        ("blk", ctypes.c_int32),
        ("donor", ctypes.c_int32),
        ("range", (ctypes.c_int64 * 2) * 3),
        ("donor_range", (ctypes.c_int64 * 2) * 3),
        ("donor_type", ctypes.c_int32 * 3),
        ("pad_", ctypes.c_int32),
    ]


class Request(ctypes.Structure):
    """struct fvm_request of include/fvm3d.h."""

    _fields_ = [
        ("struct_size", ctypes.c_int32),
        ("nblocks", ctypes.c_int32),
        ("cfg", ctypes.POINTER(FvmConfig)),
        ("nvert", ctypes.POINTER(ctypes.c_int64)),
        ("dr", ctypes.POINTER(ctypes.c_double)),
        ("q", ctypes.POINTER(ctypes.POINTER(ctypes.c_double))),
        ("nbc", ctypes.c_int32),
        ("nconn", ctypes.c_int32),
        ("bc", ctypes.POINTER(ctypes.c_int32)),
        ("conn", ctypes.POINTER(Connection)),
        ("steps", ctypes.c_int64),
    ]


REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED = 0, 1, 2, 3

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "csrc", "lib", "libfvm3d.so")

_lib = None


def load_library(path: str | None = None) -> ctypes.CDLL:
    """Load libfvm3d.so and declare its prototypes. Raises if it is absent.
    The environment variable FVM3D_LIB, when set, names another build of the
    library to load instead of the in-tree one."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or os.environ.get("FVM3D_LIB") or LIB_PATH
    if not os.path.exists(p):
        raise OSError(
            f"libfvm3d.so not found at {p}; build it with "
            "`python -c 'import __graft_entry__ as g; g.build()'`"
        )
    lib = ctypes.CDLL(p)
    i32, i64, dbl, vp = ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p
    P = ctypes.POINTER
    proto = {
        "fvm_config_default": (ctypes.c_int, [P(FvmConfig)]),
        "fvm_abi_version": (ctypes.c_int, []),
        "fvm_create": (ctypes.c_int, [P(FvmConfig), P(vp)]),
        "fvm_add_block": (ctypes.c_int, [vp, P(i64), P(dbl), P(ctypes.c_int)]),
        "fvm_set_boundary": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
        "fvm_connect": (ctypes.c_int, [vp, ctypes.c_int, P(i64), ctypes.c_int, P(i64), P(i32)]),
        "fvm_set_state": (ctypes.c_int, [vp, ctypes.c_int, P(dbl)]),
        "fvm_get_state": (ctypes.c_int, [vp, ctypes.c_int, P(dbl)]),
        "fvm_set_states": (ctypes.c_int, [vp, ctypes.c_int, P(ctypes.c_int), P(P(dbl))]),
        "fvm_get_states": (ctypes.c_int, [vp, ctypes.c_int, P(ctypes.c_int), P(P(dbl))]),
        "fvm_get_primitive": (ctypes.c_int, [vp, ctypes.c_int, P(dbl)]),
        "fvm_get_rhs": (ctypes.c_int, [vp, ctypes.c_int, P(dbl)]),
        "fvm_step": (ctypes.c_int, [vp, ctypes.c_int, P(dbl), P(dbl), P(dbl)]),
        "fvm_run": (ctypes.c_int, [vp, i64, dbl, dbl, dbl, P(i64), P(ctypes.c_int)]),
        "fvm_get_time": (ctypes.c_int, [vp, P(dbl), P(dbl), P(i64)]),
        "fvm_last_error": (ctypes.c_int, [vp, ctypes.c_char_p, ctypes.c_size_t]),
        "fvm_destroy": (ctypes.c_int, [vp]),
        "fvm_residual_norms": (ctypes.c_int, [vp, P(i64), vp, vp]),
        "fvm_reserve": (ctypes.c_int, [vp, i64]),
        "fvm_block_cells": (ctypes.c_int, [ctypes.c_int, P(i64), P(i64)]),
        "fvm_add_case": (ctypes.c_int, [vp, P(FvmConfig), P(ctypes.c_int)]),
        "fvm_add_case_block": (ctypes.c_int, [vp, ctypes.c_int, P(i64), P(dbl), P(ctypes.c_int)]),
        "fvm_remove_case": (ctypes.c_int, [vp, ctypes.c_int]),
        "fvm_case_state": (ctypes.c_int, [vp, ctypes.c_int, P(dbl), P(dbl), P(i64), P(dbl), P(dbl),
                                          P(ctypes.c_int)]),
        "fvm_server_config_default": (ctypes.c_int, [P(ServerConfig)]),
        "fvm_server_create": (ctypes.c_int, [P(ServerConfig), P(vp)]),
        "fvm_case_submit": (ctypes.c_int, [vp, P(Request), P(i64)]),
        "fvm_poll": (ctypes.c_int, [vp, i64, P(ctypes.c_int), P(i64), P(dbl), P(dbl), P(ctypes.c_int)]),
        "fvm_wait": (ctypes.c_int, [vp, i64, dbl, P(ctypes.c_int)]),
        "fvm_fetch_state": (ctypes.c_int, [vp, i64, ctypes.c_int, P(dbl)]),
        "fvm_release": (ctypes.c_int, [vp, i64]),
        "fvm_server_last_error": (ctypes.c_int, [vp, ctypes.c_char_p, ctypes.c_size_t]),
        "fvm_server_destroy": (ctypes.c_int, [vp]),
        "fvm_server_stats": (ctypes.c_int, [vp, P(i64), P(i64), P(ctypes.c_int), P(ctypes.c_int)]),
    }
    for name, (res, args) in proto.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _lib = lib
    return lib


def block_cells(idimension: int, nvert) -> int:
    """Arena cells (per variable slab) a block of this shape occupies."""
    lib = load_library()
    out = ctypes.c_int64()
    rc = lib.fvm_block_cells(int(idimension), (ctypes.c_int64 * 3)(*[int(x) for x in nvert]), ctypes.byref(out))
    if rc != 0:
        raise ValueError(f"fvm_block_cells failed ({rc})")
    return out.value


def block_bytes(cfg: FvmConfig, nvert) -> int:
    """Device bytes the state of one block takes (all RK roles, viscous slab)."""
    slabs = (4 if cfg.rk_stages == 4 else 3) + (1 if cfg.equation == EQ_NAVIER_STOKES else 0)
    return block_cells(cfg.idimension, nvert) * 5 * 8 * slabs


def declared_symbols(header: str) -> list[str]:
    """Names of the functions include/fvm3d.h declares (for export checks)."""
    import re

    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fvm_[a-z0-9_]+)\s*\(", text)))
