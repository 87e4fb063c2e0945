"""Namelist front end: the reference's case files drive the B200 path.

Parsing follows ClassNamelist (src/base/method_namelist.f90:152-259):
  * a group opens on a line that is exactly ``&Name`` and closes on ``/``;
  * blank lines and lines starting with ``!`` are skipped;
  * a line ending in ``&`` continues on the next one (the ``&`` becomes a
    blank), and every assignment must contain ``=`` ("Format Error");
  * ``get`` returns the value with double quotes removed, ``""`` when the key
    is absent;
  * ``check`` fails on any key of the group nobody asked for ("Variable not
    defined in namelist").
The keys read per group are those of ClassInput%read_casefile
(src/solve/class_input.f90:89-183); strings map to ids as TypeDefs does
(type_defs_scheme.f90:41-84, type_defs_dimension.f90, type_defs_equation.f90,
type_defs_gas.f90).

Settings the reference has no key for (precision, compat, RK stage count, CFL
number, viscosity) live in an extra group ``&B200`` the reference never
reads, so one file drives both codes.
"""
from __future__ import annotations

from dataclasses import dataclass, field

from . import abi, output

# the keys ClassInput%read_casefile asks for, per group (class_input.f90:109-177)
GROUP_KEYS = {
    "General": ["name", "dimension", "dimensionless", "equation", "gasModel"],
    "Geometry": ["type", "gridfile", "geoType", "gridType", "geoSize", "gridSize", "writeGrid"],
    "Inviscid_Flux": ["reconstruct", "kappa", "limiter", "limiter_coeff", "flux_split", "entropy_fix"],
    "Time_Stepping": ["time_scheme", "timestep_set", "fix_timestep", "total_time", "output_time",
                      "absolute_residual", "relative_residual"],
    "Output": ["format", "solnfile", "Density", "VelocityX", "VelocityY", "VelocityZ", "Pressure", "Temperature"],
    "B200": ["precision", "compat", "rk_stages", "cfl", "mu", "prandtl", "nk"],
}


class NamelistError(ValueError):
    pass


@dataclass
class Namelist:
    name: str
    members: dict = field(default_factory=dict)   # key -> raw value
    used: set = field(default_factory=set)

    def get(self, key: str) -> str:
        """ClassNamelist%get: value without double quotes, "" if absent."""
        if key in self.members:
            self.used.add(key)
            return self.members[key].replace('"', "").strip()
        return ""

    def check(self):
        for k, v in self.members.items():
            if k not in self.used:
                raise NamelistError(f"Variable not defined in namelist: {k} = {v}")


def read_group(text: str, name: str) -> Namelist | None:
    """read_nml_sub: the group `name` of `text`, or None when absent."""
    nml = Namelist(name)
    inside = False
    found = False
    pending = ""
    for idx, raw in enumerate(text.splitlines(), start=1):
        line = raw.strip()
        if not line or line.startswith("!"):
            continue
        if line == "&" + name:
            inside = True
            found = True
            continue
        if inside and line == "/":
            break
        if not inside:
            continue
        pending = pending + line
        if line.endswith("&"):
            continue
        if "=" not in pending:
            raise NamelistError(f"Format Error -- line {idx}: {raw}")
        pending = pending.replace("&", " ")
        k, v = pending.split("=", 1)
        nml.members[k.strip()] = v.strip()
        pending = ""
    return nml if found else None


def _num(s: str, default: float) -> float:
    s = s.strip()
    if not s:
        return default
    return float(s.replace("d", "e").replace("D", "E"))


def _ints(s: str) -> list[int]:
    return [int(float(x)) for x in s.replace(",", " ").split()]


@dataclass
class CaseSpec:
    """What a case file asks the B200 path for."""
    name: str
    config: abi.FvmConfig
    nvert: tuple
    dr: tuple
    geo_size: float
    total_time: float
    absolute_residual: float
    relative_residual: float
    output_time: float
    output_vars: tuple = ()
    solnfile: str = ""


DIMENSION = {"2D": 2, "3D": 3}
EQUATION = {"Euler": abi.EQ_EULER, "NavierStokes": abi.EQ_NAVIER_STOKES}


def parse_case(text: str) -> CaseSpec:
    """ClassInput%read_casefile + check_casefile on the groups the B200 path
    needs. Raises NamelistError with the reference's message on bad input."""
    groups = {}
    for g in GROUP_KEYS:
        nml = read_group(text, g)
        if nml is None:
            if g == "B200":
                continue
            raise NamelistError(f"namelist &{g} not found")
        vals = {k: nml.get(k) for k in GROUP_KEYS[g]}
        nml.check()
        groups[g] = vals
    gen, geo, inv, ts = groups["General"], groups["Geometry"], groups["Inviscid_Flux"], groups["Time_Stepping"]
    out = groups["Output"]
    ext = groups.get("B200", {})

    idim = DIMENSION.get(gen["dimension"])
    if idim is None:
        raise NamelistError("Invalid dimension.")
    if gen["equation"] not in EQUATION:
        raise NamelistError("Invalid equation type.")
    if gen["gasModel"] not in ("ideal", "Calorically Perfect"):
        raise NamelistError("Invalid gas model.")
    if geo["type"] != "uniform" or geo["geoType"] != "square":
        raise NamelistError("only the uniform square grid of method_gridgen.f90 is generated")
    L = _num(geo["geoSize"], 1.0)
    sizes = _ints(geo["gridSize"])
    if len(sizes) < idim:
        raise NamelistError("gridSize needs one entry per dimension")
    # method_gridgen.f90:99-131: nodal-centred, dx = L/(n-1), "square" forces
    # Ly = Lx and Lz = 1; a 2D grid has 2 node planes in k
    nvert = [sizes[0], sizes[1], sizes[2] if idim == 3 else 2]
    if ext.get("nk"):
        nvert[2] = int(ext["nk"])
    geo_sz = [L, L, L if idim == 3 else 1.0]
    dr = tuple(geo_sz[a] / (max(nvert[a], 2) - 1) for a in range(3))

    recon = abi.scheme_index(inv["reconstruct"])
    flux = abi.scheme_index(inv["flux_split"])
    if recon == abi.SCHEME_NULL:
        raise NamelistError("Invalid reconstruct scheme.")
    if flux == abi.SCHEME_NULL:
        raise NamelistError("Invalid flux split scheme.")
    tscheme = abi.scheme_index(ts["time_scheme"])
    if tscheme == abi.SCHEME_NULL:
        raise NamelistError("Invalid time discretization scheme.")
    tset = {"fixed": abi.DT_FIXED, "CFL": abi.DT_CFL, "CFL_local": abi.DT_CFL_LOCAL}.get(ts["timestep_set"])
    if tset is None:
        raise NamelistError("Invalid timestep type.")
    prec = {"": abi.PREC_FP64_EXACT, "fp64_exact": abi.PREC_FP64_EXACT, "fp64": abi.PREC_FP64,
            "fp32_flux": abi.PREC_FP32_FLUX}[ext.get("precision", "")]
    compat = {"": abi.COMPAT_REFERENCE, "reference": abi.COMPAT_REFERENCE,
              "textbook": abi.COMPAT_TEXTBOOK}[ext.get("compat", "")]
    cfg = abi.make_config(
        idimension=idim, equation=EQUATION[gen["equation"]], reconstruct=recon,
        limiter=abi.scheme_index(inv["limiter"]) if inv["limiter"] else abi.SCHEME_NULL,
        kappa=_num(inv["kappa"], -1.0), flux_split=flux, entropy_fix=_num(inv["entropy_fix"], 0.05),
        time_scheme=tscheme, rk_stages=int(_num(ext.get("rk_stages", ""), 3)), timestep_set=tset,
        dt=_num(ts["fix_timestep"], 0.0), cfl=_num(ext.get("cfl", ""), 0.5), precision=prec, compat=compat,
        mu=_num(ext.get("mu", ""), 0.0), prandtl=_num(ext.get("prandtl", ""), 0.71))
    return CaseSpec(name=gen["name"], config=cfg, nvert=tuple(nvert), dr=dr, geo_size=L,
                    total_time=_num(ts["total_time"], 0.0),
                    absolute_residual=_num(ts["absolute_residual"], 0.0),
                    relative_residual=_num(ts["relative_residual"], 0.0),
                    output_time=_num(ts["output_time"], 0.0),
                    output_vars=tuple(output.output_variables(out)), solnfile=out["solnfile"])


def initial_state(spec: CaseSpec):
    """The initial condition the reference hard-codes for every case file
    (the 2D Riemann quadrants of class_flow_field.f90:207-243) on the grid
    the file describes). Its four regions cover [0,1]^2 only; a larger grid
    would keep zero density outside them, so it is rejected."""
    import numpy as np

    from . import cases

    ni, nj, nk = spec.nvert
    if spec.dr[0] * (ni - 1) > 1.0 + 1e-12 or spec.dr[1] * (nj - 1) > 1.0 + 1e-12:
        raise NamelistError("the reference initial condition covers the unit square only (geoSize <= 1)")
    x = spec.dr[0] * np.arange(ni)
    y = spec.dr[1] * np.arange(nj)
    X, Y = np.meshgrid(x, y, indexing="xy")
    states = [(1.5, 0.0, 0.0, 0.0, 1.5), (0.5323, 1.206, 0.0, 0.0, 0.3), (0.138, 1.206, 1.206, 0.0, 0.029),
              (0.5323, 0.0, 1.206, 0.0, 0.3)]
    rho, u, v, w, p = cases._quadrant_fill(X, Y, 0.8, 0.8, states)
    q = cases.prim_to_cons(rho, u, v, w, p)
    return np.broadcast_to(q[:, None], (5, nk, nj, ni)).copy()


def run_case(text: str, solver_cls=None, output_prefix: str | None = None):
    """Run a reference case file end to end: parse, build the block, upload
    the reference IC, step until ClassIteration%converged fires. With
    `output_prefix`, the flow field is written at t = 0 and whenever the time
    hits the next multiple of output_time to 1e-9, as write_flowfield_sub
    does (class_output.f90:204-237): once a time is missed, no later output
    follows, as in the reference."""
    from .solver import Solver

    spec = parse_case(text)
    s = (solver_cls or Solver)(spec.config)
    s.add_block(spec.nvert, spec.dr)
    s.set_state(0, initial_state(spec))
    stop = dict(absolute_residual=spec.absolute_residual, relative_residual=spec.relative_residual)
    if output_prefix is None or not spec.output_vars:
        steps, reason = s.run(total_time=spec.total_time, **stop)
        return s, spec, steps, reason
    w = output.SolutionWriter(output_prefix, spec.output_vars, spec.dr)
    w.snapshot(s, 0.0, [0])
    time_out, steps = spec.output_time, 0
    while True:
        chunked = spec.output_time > 0 and time_out < spec.total_time - 1e-10
        n, reason = s.run(total_time=time_out if chunked else spec.total_time, **stop)
        steps += n
        t = s.time()[0]
        if spec.output_time > 0 and abs(t - time_out) <= 1e-9:
            w.snapshot(s, t, [0])
            time_out += spec.output_time
        elif chunked:
            time_out = float("inf")   # missed: the reference writes nothing more
        if not (chunked and reason == abi.STOP_MAX_TIME):
            break
    w.close()
    return s, spec, steps, reason
