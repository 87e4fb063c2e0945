"""Serving: continuous batching of solver requests on one GPU.

Requests (a seeded case plus a number of RK steps) arrive over time and are
submitted to the library's server (fvm_server_* of include/fvm3d.h). Its
worker thread keeps every admitted case's state resident in engines whose
state arenas are reserved up front (the HBM budget); a request is admitted,
first come first served, as soon as its blocks fit into the free arena, and it
joins the running batch at the next step boundary: all admitted cases advance
together, one persistent launch per scheme group and stage. A finished case
is read back and removed, which frees its arena range for the queue.
Time-to-solution is measured from submission (at arrival) to the moment its
final state is in host memory.

The one-at-a-time baseline serves the same stream in arrival order with one
engine per request.

The engine keeps a case's tiling, time step and residual sums independent of
its neighbours, so a case's final state is the same alone and in the mix.
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import abi, cases
from .solver import FvmError, Solver


@dataclass
class Request:
    rid: int
    case: cases.Case
    nsteps: int
    arrival: float                # seconds after the stream starts
    cells: int = 0                # arena cells the request needs
    case_id: int = -1
    req_id: int = -1              # the library server's request id
    remaining: int = 0
    admitted: float = math.nan
    submitted: float = math.nan
    finished: float = math.nan
    result: list = field(default_factory=list)
    status: int = 0

    @property
    def latency(self) -> float:
        return self.finished - self.arrival

    @property
    def work(self) -> int:
        """cell-stage updates the request asks for"""
        return self.case.ncells * int(self.case.cfg.get("rk_stages", 3)) * self.nsteps


def poisson_stream(n: int, rate: float, seed: int, make_case, steps=(200, 2000)):
    """n requests with exponential inter-arrival times (mean 1/rate seconds);
    make_case(rng, i) builds the i-th case; step counts uniform in `steps`."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        c = make_case(rng, i)
        out.append(Request(rid=i, case=c, nsteps=int(rng.integers(steps[0], steps[1] + 1)), arrival=t))
    return out


def mixed_family(precision=abi.PREC_FP32_FLUX, sizes=(32, 96)):
    """Case builder for the serving stream: blasts and oblique shock tubes of
    random cube size, random Roe / AUSM and MUSCL / WENO5, SSP-RK3, TEXTBOOK
    compat (its positivity fallback keeps WENO5 alive on the strong blasts
    that drive the reference's scheme to NaN)."""
    def make(rng, i):
        n = int(round(sizes[0] * (sizes[1] / sizes[0]) ** rng.uniform()))
        n = max(8, n)
        recon = [abi.RECON_MUSCL, abi.RECON_WENO][int(rng.integers(2))]
        flux = [abi.FLUX_ROE, abi.FLUX_AUSM][int(rng.integers(2))]
        fam = cases.blast if rng.uniform() < 0.5 else cases.shock_tube
        return fam((n, n, n), seed=int(rng.integers(1 << 30)), reconstruct=recon, flux_split=flux,
                   limiter=abi.LIMITER_MINMOD, kappa=1.0 / 3.0, precision=precision, rk_stages=3,
                   compat=abi.COMPAT_TEXTBOOK)
    return make


def config_families(precision=abi.PREC_FP32_FLUX, sizes=(32, 96)):
    """Case builder for the served stream of the three solver configurations'
    families, drawn with equal probability, grid edge N log-uniform in
    `sizes` (a 2D case takes edge round(N^1.5), the same cell count as N^3):
      * four-quadrant 2D Riemann problem, MUSCL / minmod + Roe (fix 0.2),
        SSP-RK3, CFL 0.5, seeded quadrant states;
      * 3D Euler isentropic vortex in the 8 uneven periodic blocks, WENO5 +
        AUSM, classic RK4, CFL 0.5;
      * 3D Navier-Stokes Taylor-Green vortex (Re 1600, Ma 0.1), MUSCL / Van
        Albada + Roe + central viscous fluxes, SSP-RK3, CFL 0.5."""
    def make(rng, i):
        n = int(round(sizes[0] * (sizes[1] / sizes[0]) ** rng.uniform()))
        n = max(8, n)
        fam = int(rng.integers(3))
        if fam == 0:
            return cases.riemann2d(n=int(round(n ** 1.5)), seed=int(rng.integers(1 << 30)), precision=precision,
                                   timestep_set=abi.DT_CFL, cfl=0.5)
        if fam == 1:
            return cases.isentropic_vortex(N=n, layout="blocks8", precision=precision)
        return cases.taylor_green(N=n, precision=precision)
    return make


class Server:
    """Continuous-batching server of the library (fvm_server_* in
    include/fvm3d.h): requests are submitted to a worker thread inside
    libfvm3d.so that admits them first come, first served, into a reserved
    state arena (the HBM budget), advances all admitted cases together and
    retires each one when its steps are done. This class only converts cases
    to requests and reads results back."""

    def __init__(self, budget_cells: int, chunk: int = 8, max_active_cells: int | None = 1 << 20,
                 max_queued: int = 4096):
        """budget_cells: the state arena (HBM budget) in fvm_block_cells
        units. max_active_cells: stop admitting once the running set holds
        this many cells (None = no cap; one request is always admitted into
        an empty set). Past the point where the running set keeps the GPU
        busy, admitting more only shares it among more requests, which
        lengthens every running request's latency."""
        self.lib = abi.load_library()
        cfg = abi.ServerConfig()
        self.lib.fvm_server_config_default(ctypes.byref(cfg))
        cfg.chunk_steps = int(chunk)
        cfg.budget_cells = int(budget_cells)
        cfg.max_active_cells = 0 if max_active_cells is None else int(max_active_cells)
        cfg.max_queued = int(max_queued)
        self.h = ctypes.c_void_p()
        rc = self.lib.fvm_server_create(ctypes.byref(cfg), ctypes.byref(self.h))
        if rc:
            raise FvmError(rc, "fvm_server_create failed")
        self.budget = budget_cells

    def close(self):
        if getattr(self, "h", None):
            self.lib.fvm_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc: int):
        if rc:
            buf = ctypes.create_string_buffer(512)
            self.lib.fvm_server_last_error(self.h, buf, 512)
            raise FvmError(rc, buf.value.decode())

    def cells_of(self, c: cases.Case) -> int:
        idim = int(c.cfg.get("idimension", 3))
        return sum(abi.block_cells(idim, n) for n, _ in c.blocks)

    def submit(self, case: cases.Case, nsteps: int) -> int:
        """fvm_case_submit: the library copies everything before it returns."""
        nb = len(case.blocks)
        cfg = case.config()
        nvert = (ctypes.c_int64 * (3 * nb))(*[int(x) for n, _ in case.blocks for x in n])
        dr = (ctypes.c_double * (3 * nb))(*[float(x) for _, d in case.blocks for x in d])
        qs = [np.ascontiguousarray(q, dtype=np.float64) for q in case.states]
        qp = (ctypes.POINTER(ctypes.c_double) * nb)(*[q.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for q in qs])
        bc = (ctypes.c_int32 * max(1, 3 * len(case.bcs)))(*[int(x) for b in case.bcs for x in b])
        conn = (abi.Connection * max(1, len(case.conns)))()
        for i, (blk, rng, donor, drng, dtype) in enumerate(case.conns):
            c = conn[i]
            c.blk, c.donor = int(blk), int(donor)
            for a in range(3):
                c.range[a][0], c.range[a][1] = int(rng[a][0]), int(rng[a][1])
                c.donor_range[a][0], c.donor_range[a][1] = int(drng[a][0]), int(drng[a][1])
                c.donor_type[a] = int(dtype[a])
        r = abi.Request()
        r.struct_size = ctypes.sizeof(abi.Request)
        r.nblocks = nb
        r.cfg = ctypes.pointer(cfg)
        r.nvert = nvert
        r.dr = dr
        r.q = qp
        r.nbc = len(case.bcs)
        r.bc = bc
        r.nconn = len(case.conns)
        r.conn = conn
        r.steps = int(nsteps)
        rid = ctypes.c_int64()
        self._chk(self.lib.fvm_case_submit(self.h, ctypes.byref(r), ctypes.byref(rid)))
        return rid.value

    def poll(self, rid: int) -> dict:
        st, status = ctypes.c_int(), ctypes.c_int()
        done, t, lat = ctypes.c_int64(), ctypes.c_double(), ctypes.c_double()
        self._chk(self.lib.fvm_poll(self.h, rid, ctypes.byref(st), ctypes.byref(done), ctypes.byref(t),
                                    ctypes.byref(lat), ctypes.byref(status)))
        return {"state": st.value, "steps_done": done.value, "t": t.value, "latency_s": lat.value,
                "status": status.value}

    def wait(self, rid: int, timeout: float = 600.0) -> int:
        st = ctypes.c_int()
        self._chk(self.lib.fvm_wait(self.h, rid, float(timeout), ctypes.byref(st)))
        return st.value

    def fetch(self, rid: int, case: cases.Case) -> list:
        out = []
        for b, (n, _) in enumerate(case.blocks):
            q = np.empty((5, n[2], n[1], n[0]), dtype=np.float64)
            self._chk(self.lib.fvm_fetch_state(self.h, rid, b, q.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
            out.append(q)
        return out

    def release(self, rid: int):
        self._chk(self.lib.fvm_release(self.h, rid))

    def stats(self) -> dict:
        """Cells held by the running set now and at most so far, and the
        numbers of running and queued requests (fvm_server_stats)."""
        act, peak = ctypes.c_int64(), ctypes.c_int64()
        run, que = ctypes.c_int(), ctypes.c_int()
        self._chk(self.lib.fvm_server_stats(self.h, ctypes.byref(act), ctypes.byref(peak), ctypes.byref(run),
                                            ctypes.byref(que)))
        return {"active_cells": act.value, "peak_active_cells": peak.value, "running": run.value,
                "queued": que.value}

    def run(self, stream: list[Request], clock=time.perf_counter, realtime: bool = True):
        """Serve the stream: each request is submitted at its arrival time
        (wall clock) when `realtime`, else all at t = 0; then every result is
        awaited and read back. Time-to-solution is the library's own
        submission-to-completion time. Returns stats."""
        pending = sorted(stream, key=lambda r: r.arrival)
        for r in pending:
            r.cells = self.cells_of(r.case)
            if r.cells > self.budget:
                raise ValueError(f"request {r.rid} needs {r.cells} cells, more than the whole budget")
        t0 = clock()
        for r in pending:
            if realtime:
                wait = r.arrival - (clock() - t0)
                if wait > 0:
                    time.sleep(wait)
            r.submitted = clock() - t0
            r.req_id = self.submit(r.case, r.nsteps)
        for r in pending:
            self.wait(r.req_id)
            p = self.poll(r.req_id)
            r.status = p["status"]
            r.finished = r.submitted + p["latency_s"]
            if not realtime:
                r.arrival = 0.0
            r.result = self.fetch(r.req_id, r.case)
            self.release(r.req_id)
        makespan = max((r.finished for r in pending), default=0.0)
        return summarize(pending, makespan)


def serve_one_at_a_time(stream: list[Request], clock=time.perf_counter, realtime: bool = True, precision=None):
    """Baseline: one engine per request, strictly in arrival order (each
    request in its own precision form, or in `precision` when given)."""
    pending = sorted(stream, key=lambda r: r.arrival)
    done = []
    t0 = clock()
    for r in pending:
        now = clock() - t0
        if realtime and r.arrival > now:
            time.sleep(r.arrival - now)
        r.admitted = clock() - t0
        over = {} if precision is None else {"precision": precision}
        s = r.case.apply(Solver(r.case.config(**over)))
        s.step(r.nsteps)
        r.result = [s.get_state(b) for b in range(len(r.case.blocks))]
        r.status = s.case_state(0)["status"]
        s.close()
        r.finished = clock() - t0
        done.append(r)
    return summarize(done, clock() - t0)


def summarize(done: list[Request], makespan: float) -> dict:
    lat = np.array([r.latency for r in done]) if done else np.zeros(1)
    work = float(sum(r.work for r in done))
    return {
        "requests": len(done),
        "p50_s": float(np.percentile(lat, 50)),
        "p99_s": float(np.percentile(lat, 99)),
        "mean_s": float(lat.mean()),
        "makespan_s": makespan,
        "gcell_stage_per_s": work / makespan / 1e9 if makespan > 0 else 0.0,
        "failed": int(sum(1 for r in done if r.status != 0)),
    }
