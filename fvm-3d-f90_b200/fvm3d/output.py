"""Solution output: the flow-field snapshots the reference writes at its
output times, as VTK XML structured grids.

The reference writes one CGNS file (class_output.f90:204-263 through
interface_cgns_write.f90:143-421): the grid coordinates once, then at t = 0
and at every multiple of `output_time` the realtime hits (to 1e-9) one
FlowSolution per block with the variables the &Output group switches on
(Density, VelocityX/Y/Z, Pressure; type_defs_variables.f90 names them after
the CGNS SIDS identifiers). CGNS needs the CGNS/HDF5 libraries, which this
image does not have; the same content goes to one `.vts` file per block and
output time, named with the same variable names, plus a `.pvd` collection
that lists the files with their times (what the CGNS iterative data holds).

Snapshots are downloaded as primitives through `fvm_get_primitive` and
written by a background thread, so the solver advances while the previous
snapshot is being written.
"""
from __future__ import annotations

import os
import threading
from concurrent.futures import ThreadPoolExecutor

import numpy as np

# type_defs_variables.f90: the names the &Output group switches on, in the
# order ClassInput%read_casefile reads them (class_input.f90:164-177)
VARIABLES = ("Density", "VelocityX", "VelocityY", "VelocityZ", "Pressure", "Temperature")
# component of the primitive vector (rho, u, v, w, p) each name reads;
# Temperature is p / rho (the reference names it but get_data_fun fills
# nothing for it)
_COMPONENT = {"Density": 0, "VelocityX": 1, "VelocityY": 2, "VelocityZ": 3, "Pressure": 4}


def fortran_true(value: str) -> bool:
    """A Fortran logical literal as namelist input gives it."""
    v = value.strip().lower().strip(".")
    return v in ("true", "t")


def output_variables(group: dict) -> list[str]:
    """The variables an &Output group switches on, in the reference's order."""
    return [name for name in VARIABLES if fortran_true(group.get(name, "") or "")]


def _field(prim: np.ndarray, name: str) -> np.ndarray:
    if name == "Temperature":
        return prim[4] / prim[0]
    return prim[_COMPONENT[name]]


def write_vts(path: str, prim: np.ndarray, variables, dr, origin=(0.0, 0.0, 0.0)) -> None:
    """One block's primitives (5, nk, nj, ni) as a VTK XML StructuredGrid with
    raw appended Float64 data; point i sits at origin + i * dr."""
    _, nk, nj, ni = prim.shape
    arrays = [np.ascontiguousarray(_field(prim, v), dtype="<f8") for v in variables]
    z, y, x = np.meshgrid(origin[2] + dr[2] * np.arange(nk), origin[1] + dr[1] * np.arange(nj),
                          origin[0] + dr[0] * np.arange(ni), indexing="ij")
    pts = np.ascontiguousarray(np.stack([x, y, z], axis=-1), dtype="<f8")
    ext = f"0 {ni - 1} 0 {nj - 1} 0 {nk - 1}"
    head = ['<?xml version="1.0"?>',
            '<VTKFile type="StructuredGrid" version="1.0" byte_order="LittleEndian" header_type="UInt64">',
            f'  <StructuredGrid WholeExtent="{ext}">',
            f'    <Piece Extent="{ext}">',
            f'      <PointData Scalars="{variables[0] if variables else ""}">']
    off = 0
    blobs = []
    for name, a in zip(variables, arrays):
        head.append(f'        <DataArray type="Float64" Name="{name}" format="appended" offset="{off}"/>')
        blobs.append(a)
        off += 8 + a.nbytes
    head += ['      </PointData>', '      <Points>',
             f'        <DataArray type="Float64" Name="Points" NumberOfComponents="3" format="appended" '
             f'offset="{off}"/>', '      </Points>', '    </Piece>', '  </StructuredGrid>',
             '  <AppendedData encoding="raw">']
    blobs.append(pts)
    tmp = path + ".tmp"
    with open(tmp, "wb") as f:
        f.write(("\n".join(head) + "\n   _").encode())
        for b in blobs:
            f.write(np.uint64(b.nbytes).tobytes())
            f.write(b.tobytes())
        f.write(b"\n  </AppendedData>\n</VTKFile>\n")
    os.replace(tmp, path)


def read_vts(path: str) -> dict:
    """Arrays of a file written by write_vts, by name (Points included),
    shaped (nk, nj, ni[, 3])."""
    import re

    raw = open(path, "rb").read()
    start = raw.index(b'<AppendedData encoding="raw">')
    head = raw[:start].decode()
    data = raw[raw.index(b"_", start) + 1:]
    ext = [int(v) for v in re.search(r'WholeExtent="([^"]+)"', head).group(1).split()]
    shape = (ext[5] + 1, ext[3] + 1, ext[1] + 1)
    out = {}
    for m in re.finditer(r'Name="([^"]+)"(?: NumberOfComponents="(\d)")? format="appended" offset="(\d+)"', head):
        name, ncomp, off = m.group(1), int(m.group(2) or 1), int(m.group(3))
        n = int(np.frombuffer(data[off:off + 8], dtype="<u8")[0])
        a = np.frombuffer(data[off + 8:off + 8 + n], dtype="<f8")
        out[name] = a.reshape(shape + ((ncomp,) if ncomp > 1 else ()))
    return out


class SolutionWriter:
    """Snapshots of a multi-block case: `<prefix>_b<block>_<n>.vts` files and
    a `<prefix>.pvd` collection with their times."""

    def __init__(self, prefix: str, variables, dr, origins=None, workers: int = 1):
        self.prefix = prefix
        self.variables = list(variables)
        self.dr = dr
        self.origins = origins
        self.entries = []           # (time, block, file)
        self.nsoln = 0
        self._pool = ThreadPoolExecutor(max_workers=workers)
        self._pending = []
        self._lock = threading.Lock()
        d = os.path.dirname(prefix)
        if d:
            os.makedirs(d, exist_ok=True)

    def snapshot(self, solver, t: float, blocks) -> None:
        """Download the primitives of `blocks` now and write them in the
        background."""
        for b in blocks:
            prim = solver.get_primitive(b)
            dr = self.dr[b] if isinstance(self.dr, (list, tuple)) and isinstance(self.dr[0], (list, tuple)) \
                else self.dr
            org = self.origins[b] if self.origins else (0.0, 0.0, 0.0)
            name = f"{self.prefix}_b{b}_{self.nsoln:04d}.vts"
            self._pending.append(self._pool.submit(write_vts, name, prim, self.variables, dr, org))
            with self._lock:
                self.entries.append((t, b, os.path.basename(name)))
        self.nsoln += 1

    def close(self) -> str:
        """Wait for the writes and write the collection file; returns its path."""
        for f in self._pending:
            f.result()
        self._pending.clear()
        self._pool.shutdown(wait=True)
        pvd = self.prefix + ".pvd"
        lines = ['<?xml version="1.0"?>', '<VTKFile type="Collection" version="1.0" byte_order="LittleEndian">',
                 "  <Collection>"]
        for t, b, f in self.entries:
            lines.append(f'    <DataSet timestep="{t:.17g}" part="{b}" file="{f}"/>')
        lines += ["  </Collection>", "</VTKFile>", ""]
        with open(pvd, "w") as fh:
            fh.write("\n".join(lines))
        return pvd
