#!/usr/bin/env python
"""Benchmark of the B200 explicit residual-and-update path.

Workload (the configuration the headline metric is quoted on): 3D Euler
isentropic vortex (strength 5, gamma 1.4, freestream rho = p = 1,
u = v = w = 1) on the periodic box [-5,5]^3 split into 8 uneven blocks
(2,097,152 cells, 3 ghost layers, non-conforming block interfaces), WENO5 +
AUSM, classic RK4, CFL 0.5. Inputs are the seeded analytic initial state
(no dataset exists for this solver).

One "step" is one RK4 time step (4 stages) over all blocks. value = cells x
stages x ranks / max-over-ranks device time, in Gcell-stage/s, for the FP64
plain form (the reference's arithmetic width); the FP32-flux form (FP32
reconstruction and flux, FP64 state and RK accumulation) and the exact FP64
form (the reference's operation order) are reported beside it, with the L1
density difference of the FP32 form against FP64 after the same steps and
the FP32 / FP64 speed ratio on every configuration.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "fvm-3d-f90_b200")
sys.path.insert(0, PKG)

METRIC = "Gcell-stage/s FP64 plain vs FP32-batched at L1 err<=1e-6; served p50/p99 latency"
UNIT = "Gcell-stage/s"
# DRAM bytes per stage launch on the 128^3 vortex (ncu dram__bytes_read.sum +
# dram__bytes_write.sum, mean of the 4 launches of one step), by (precision
# form, tile index, z chunk, tail split); tilings not captured report null
STAGE_TRAFFIC = {(1, 3, 32, 4): 368.4e6, (2, 2, 16, 2): 366.1e6}
# Tiling of the headline forms on the 128^3 vortex (tile index, z chunk, tail
# split), the autotuner's picks on a B200; fixed so that every run measures
# the same kernel configuration as its ncu capture (--autotune searches
# again). Precision ids: 1 FP64, 2 FP32 flux.
FIXED_TILING = {1: (3, 32, 4), 2: (2, 16, 2)}
# The arithmetic roof beside the HBM one: the stage kernel's busiest
# instruction pipe for the fixed tilings: the fraction of the kernel's active
# cycles that pipe was busy (ncu
# sm__pipe_<pipe>_cycles_active.avg.pct_of_peak_sustained_active, mean of the
# first two stages of a step); the FP64 form is bound by the FP64 pipe, the
# FP32-flux form by the FMA pipe (its WENO runs in f32x2 instructions, two
# pipe cycles each)
STAGE_PIPE = {(1, 3, 32, 4): ("fp64", 0.564), (2, 2, 16, 2): ("fma", 0.414)}
WORKLOAD = "isentropic vortex 3D Euler, periodic [-5,5]^3, 8 uneven blocks, 128^3 = 2,097,152 cells, WENO5 + AUSM, RK4, CFL 0.5"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="product", choices=["product", "reference"])
    ap.add_argument("--n", type=int, default=128, help="global grid edge (cells)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the 64-case batched leg")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving leg")
    ap.add_argument("--batch-cases", type=int, default=64)
    ap.add_argument("--serve-requests", type=int, default=24)
    ap.add_argument("--serve-full", action="store_true",
                    help="serving leg at the full sizes: edges 32..192, 200..2000 steps")
    ap.add_argument("--autotune", action="store_true",
                    help="search tile / z chunk / tail split for every form instead of the fixed headline tilings")
    ap.add_argument("--tile", type=int, default=None, help="fixed tile index (skips the autotuner)")
    ap.add_argument("--zchunk", type=int, default=0, help="fixed z chunk with --tile")
    ap.add_argument("--tail-split", type=int, default=1, help="fixed tail split with --tile (1 = none)")
    ap.add_argument("--forms", default="fp64,fp32,exact",
                    help="comma list of precision forms, the first is the headline: fp64, fp32, exact")
    ap.add_argument("--only", choices=["tgv", "riemann2d", "accuracy", "batched", "serve", "resid"], default=None,
                    help="run one secondary leg alone (its precision forms from --forms) and print its JSON")
    ap.add_argument("--accuracy-steps", type=int, default=1000, help="RK4 steps of the accuracy leg")
    return ap.parse_args()


# ---------------------------------------------------------------- distributed
class Dist:
    def __init__(self, gpus: int):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            # one process per GPU: the library uses the first visible device,
            # so each rank keeps only its own entry of the visible list
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            if vis is None:
                os.environ["CUDA_VISIBLE_DEVICES"] = str(self.local)
            elif vis.strip():
                devs = [d for d in vis.split(",") if d.strip()]
                os.environ["CUDA_VISIBLE_DEVICES"] = devs[self.local % len(devs)].strip()
            import datetime

            import torch.distributed as dist

            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch

        t = torch.tensor([x], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------- clocks
class Clocks:
    """Clock and throttle-reason sampling through NVML (read-only queries)
    in a background thread during the timed region."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4}

    def __init__(self, index: int = 0):
        self.rows = []
        self.ok = False
        try:
            import pynvml as nv

            nv.nvmlInit()
            self.nv = nv
            self.h, self.found_by = self._handle(nv, index)
            self.max_sm = nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)
            self.ok = True
        except Exception as e:  # noqa: BLE001
            self.err = str(e)
            return
        self.stop_flag = False
        self.th = threading.Thread(target=self._run, daemon=True)
        self.th.start()

    @staticmethod
    def _handle(nv, index):
        """The NVML device of CUDA device `index` of this process: NVML numbers
        the machine's GPUs and ignores CUDA_VISIBLE_DEVICES, so the device is
        matched by UUID, else by PCI bus id; physical index 0 only as a last
        resort (said so in the record)."""
        try:
            import torch

            p = torch.cuda.get_device_properties(index)
            try:
                return nv.nvmlDeviceGetHandleByUUID(("GPU-" + str(p.uuid)).encode()), "uuid"
            except Exception:  # noqa: BLE001
                bus = f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
                return nv.nvmlDeviceGetHandleByPciBusId(bus.encode()), "pci bus id"
        except Exception:  # noqa: BLE001
            return nv.nvmlDeviceGetHandleByIndex(0), "nvml index 0 (no match)"

    def _run(self):
        # SM clock and reasons every millisecond (the timed region of a short
        # run lasts tens of ms); the slower power query every fifth sample
        nv = self.nv
        pw = 0.0
        i = 0
        while not self.stop_flag:
            try:
                sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                try:
                    rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                except AttributeError:
                    rs = nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
                if i % 5 == 0:
                    pw = nv.nvmlDeviceGetPowerUsage(self.h) / 1000.0
                self.rows.append((sm, rs, pw))
                i += 1
            except Exception:  # noqa: BLE001
                pass
            time.sleep(0.001)

    def stop(self) -> dict:
        if not self.ok:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [f"nvml unavailable: {getattr(self, 'err', '')}"]}
        self.stop_flag = True
        self.th.join(timeout=2)
        sm = [r[0] for r in self.rows]
        reasons = sorted({n for r in self.rows for n, bit in self.REASONS.items() if r[1] & bit})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_sm,
                "power_w_max": max((r[2] for r in self.rows), default=None), "samples": len(self.rows),
                "reasons": reasons, "source": "NVML, 1 ms sampling during the timed steps",
                "device_matched_by": self.found_by}


def peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return {"hbm_gbs": d["hbm_gbs"], "src": "measured"}
    except (OSError, KeyError, ValueError):
        return {"hbm_gbs": 6650.0, "src": "fallback"}


# ---------------------------------------------------------------- product arm
def sig(x, n=4):
    """x rounded to n significant digits (keeps the JSON line short)."""
    if x is None or not isinstance(x, float) or x == 0.0 or not math.isfinite(x):
        return x
    return round(x, n - 1 - int(math.floor(math.log10(abs(x)))))


def timed_windows(solver, k, min_s=1.0, max_windows=64):
    """Device time per step of k graph-launched steps (CUDA events on the
    engine's stream, synchronised on both sides), repeated until about
    min_s seconds of timed work have run. Returns the per-window ms/step."""
    from fvm3d import tuning

    out = []
    while len(out) < max_windows and (not out or sum(out) * k < min_s * 1e3):
        out.append(tuning.time_step(solver, k))
    return out


def product(args, dist: Dist):
    import numpy as np

    from fvm3d import abi, cases, tuning
    from fvm3d.solver import Solver

    case = cases.isentropic_vortex(N=args.n, layout="blocks8")
    ncells = case.ncells
    stages = 4
    nblk = len(case.blocks)

    def fresh(prec, tile=None, z=None, sp=1):
        s = Solver(case.config(precision=prec))
        case.apply(s, states=False)
        if tile is not None:
            tuning.set_tuning(s, 0, tile, z)
            tuning.set_tail_split(s, 0, sp)
        for b, q in enumerate(case.states):
            s.set_state(b, q)
        return s

    def tune(prec):
        if args.tile is not None:
            return args.tile, args.zchunk, args.tail_split
        if not args.autotune and args.n == 128 and prec in FIXED_TILING:
            return FIXED_TILING[prec]
        s = fresh(prec)
        t, z, ms, sp = tuning.autotune(s, ncells, use_cache=False, reps=2)
        s.close()
        return t, z, sp

    def timed(prec, clocks=False):
        tile, z, sp = tune(prec)
        s = fresh(prec, tile, z, sp)
        s.step(args.warmup)
        dist.barrier()
        clk = Clocks(0) if (clocks and dist.rank == 0) else None
        win = timed_windows(s, args.steps)
        clk_rec = clk.stop() if clk else None
        ms = dist.max(statistics.median(win))
        prof = [tuning.profile_step(s) for _ in range(3)]
        launches = tuning.launches_per_step(s)
        return dict(s=s, ms=ms, win=win, clocks=clk_rec, prof=prof, launches=launches, tiling=(tile, z, sp))

    def gcs(ms):
        return ncells * stages * dist.world / (ms * 1e-3) / 1e9

    # L1 density difference between two precision forms after the same
    # number of steps (warm-up + one timing window) from the same initial
    # state: fresh contexts, since the timed runs take different step counts
    l1_steps = args.warmup + args.steps
    _rho = {}

    def rho_after(f):
        if f not in _rho:
            r = runs[f]
            s = fresh(r["prec"], *r["tiling"])
            s.step(l1_steps)
            _rho[f] = [s.get_state(i)[0] for i in range(nblk)]
            s.close()
        return _rho[f]

    def l1rho(fa, fb):
        a, b = rho_after(fa), rho_after(fb)
        return float(np.mean([np.abs(a[i] - b[i]).mean() for i in range(nblk)]))

    # roofline of the dominant kernel (the fused stage): algorithmic bytes are
    # the FP64 state arrays each stage must read or write. RK4 with q0 folded
    # into the accumulator touches 3, 5, 5, 3 arrays of 5 x 8 B per cell:
    # 640 B per cell-step, 160 B per cell-stage (the same in every precision
    # form: the state is FP64 in all of them).
    def roof(r, prec):
        prof = r["prof"]
        st = [ms for p in prof for k, ms in p if k == "stage"]
        per_step_ms = sum(st) / len(prof)
        alg = 640.0 * ncells
        ach = alg / (per_step_ms * 1e-3) / 1e9
        pk = peaks()
        share = per_step_ms / (sum(ms for p in prof for _, ms in p) / len(prof))
        key = (prec,) + tuple(r["tiling"])
        traffic = STAGE_TRAFFIC.get(key) if args.n == 128 else None
        pipe = STAGE_PIPE.get(key) if args.n == 128 else None
        return {"bound": "hbm", "achieved": sig(ach), "peak": pk["hbm_gbs"], "unit": "GB/s",
                "frac": sig(ach / pk["hbm_gbs"]), "traffic": traffic, "peak_src": pk["src"],
                "kernel": "stage_kernel", "stage_ms_per_step": sig(per_step_ms), "stage_share_of_step": sig(share),
                "alg_bytes_per_cell_step": 640, "alg_bytes_per_launch": round(160.0 * ncells),
                "alu_roof": ({"pipe": pipe[0], "busy_of_peak": pipe[1], "src": "ncu"} if pipe else None)}

    forms = args.forms.split(",")
    runs = {}
    for f in forms:
        prec = {"fp64": abi.PREC_FP64, "fp32": abi.PREC_FP32_FLUX, "exact": abi.PREC_FP64_EXACT}[f]
        runs[f] = timed(prec, clocks=(f == forms[0]))
        runs[f]["prec"] = prec
    head = runs[forms[0]]
    out = {"value": gcs(head["ms"]), "ms_per_step": head["ms"],
           "dtype": {"fp64": "f64", "fp32": "f32 recon/flux, f64 state + RK + dt + norms",
                     "exact": "f64 (reference operation order)"}[forms[0]],
           "gpu_launches": head["launches"] * args.steps * len(head["win"]),
           "roofline": roof(head, head["prec"]), "clocks": head["clocks"]}
    out["timing"] = {"windows": len(head["win"]), "steps_per_window": args.steps,
                     "ms_per_step_median": sig(statistics.median(head["win"])),
                     "ms_per_step_min": sig(min(head["win"])), "ms_per_step_max": sig(max(head["win"])),
                     "tiling": list(head["tiling"]),
                     "profile_ms": {k: sig(sum(ms for p in head["prof"] for kk, ms in p if kk == k) / 3)
                                    for k in ("stage", "gather", "finalize")}}

    # end to end through the C ABI with host buffers: every step uploads the
    # state from pinned host memory, advances one step (residuals come back)
    # and downloads the state, in the headline's precision form
    if not args.no_e2e:
        out["e2e"] = e2e_loop(args, dist, case, fresh, head["prec"], head["tiling"], stages)

    for f in forms[1:]:
        r = runs[f]
        rec = {"value": sig(gcs(r["ms"])), "ms_per_step": sig(r["ms"]), "tiling": list(r["tiling"]),
               "spread_ms": [sig(min(r["win"])), sig(max(r["win"]))]}
        if f == "fp32":
            rec["roofline"] = {k: v for k, v in roof(r, r["prec"]).items()
                               if k in ("achieved", "frac", "traffic", "stage_ms_per_step", "alu_roof")}
            ref = "fp64" if "fp64" in runs else ("exact" if "exact" in runs else None)
            if ref:
                rec["l1_density_vs_" + ref] = sig(l1rho(f, ref))
                rec["l1_steps"] = l1_steps
        out[{"fp64": "fp64_plain", "fp32": "fp32_flux", "exact": "fp64_exact"}[f]] = rec
    if "fp64" in runs and "exact" in runs and forms[0] == "fp64":
        out["fp64_exact"]["l1_density_vs_fp64"] = sig(l1rho("exact", "fp64"))
    if "fp64" in runs and "fp32" in runs:
        out["vortex_fp32_over_fp64"] = sig(runs["fp64"]["ms"] / runs["fp32"]["ms"])
    for r in runs.values():
        r["s"].close()
    return out


def e2e_loop(args, dist, case, fresh, prec, tiling, stages):
    """fvm_set_states (all blocks, pinned host memory) + fvm_step(1) +
    fvm_get_states per step, one context; then the same loop on two contexts
    from two host threads (one context per host thread, as the ABI allows),
    one's upload overlapping the other's download."""
    import threading

    import torch

    ncells = case.ncells

    def pinned():
        ps = []
        for q in case.states:
            t = torch.empty(q.size, dtype=torch.float64, pin_memory=True)
            t.numpy()[:] = q.reshape(-1)
            ps.append(t)
        return ps

    pins = pinned()
    s = fresh(prec, *tiling)
    blks = list(range(len(pins)))
    ptrs = [t.data_ptr() for t in pins]
    s.set_states_ptr(blks, ptrs)  # warm-up
    s.step(1)
    s.get_states_ptr(blks, ptrs)
    ke = max(3, min(args.steps, 10))
    dist.barrier()
    t0 = time.perf_counter()
    for _ in range(ke):
        s.set_states_ptr(blks, ptrs)
        s.step(1)
        s.get_states_ptr(blks, ptrs)
    sec = dist.max((time.perf_counter() - t0) / ke)
    s.close()
    rec = {"value": ncells * stages * dist.world / sec / 1e9, "unit": UNIT,
           "h2d_bytes_per_step": ncells * 40, "d2h_bytes_per_step": ncells * 40 + 2 * 6 * 8 + 8,
           "ms_per_step": sig(sec * 1e3), "path": "fvm_set_states + fvm_step(1) + fvm_get_states, pinned host"}
    pins2 = pinned()
    ctxs = [(fresh(prec, *tiling), ptrs), (fresh(prec, *tiling), [t.data_ptr() for t in pins2])]
    for c, p in ctxs:
        c.set_states_ptr(blks, p)
        c.step(1)
        c.get_states_ptr(blks, p)

    def loop(c, p):
        for _ in range(ke):
            c.set_states_ptr(blks, p)
            c.step(1)
            c.get_states_ptr(blks, p)

    ths = [threading.Thread(target=loop, args=cp) for cp in ctxs]
    dist.barrier()
    t0 = time.perf_counter()
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    sec2 = dist.max((time.perf_counter() - t0) / ke)
    rec["two_contexts"] = sig(2 * ncells * stages * dist.world / sec2 / 1e9)
    for c, _ in ctxs:
        c.close()
    # the reference's own pattern (solve_process): the state stays resident,
    # every step returns time and residuals to the host (fvm_step), and the
    # host reads the whole state back at output times only, here every 50
    # steps (the Riemann-2D case file writes every 0.01 s at dt 2e-4)
    s = fresh(prec, *tiling)
    s.set_states_ptr(blks, ptrs)
    s.step(1)
    nsteps = 50
    dist.barrier()
    t0 = time.perf_counter()
    for _ in range(nsteps):
        s.step(1)
    s.get_states_ptr(blks, ptrs)
    sec3 = dist.max((time.perf_counter() - t0) / nsteps)
    s.close()
    rec["state_resident_output_every_50_steps"] = sig(ncells * stages * dist.world / sec3 / 1e9)
    return rec


# ---------------------------------------------------------------- batched leg
def batched(args):
    """64 independent 3D Euler cases (seeded blasts / oblique shock tubes,
    grid edges round(32 * 4**u), u ~ U[0,1] per axis, random Roe / AUSM x
    MUSCL / WENO5, SSP-RK3, TEXTBOOK compat: the reference's WENO goes to NaN
    on the strongest blasts) advanced together: one persistent launch per
    scheme group and stage, one CUDA graph per step; in the FP32-flux and the
    FP64 forms. The FP32 batch is also compared with the same cases run one
    engine at a time (sum of their device times)."""
    import numpy as np

    from fvm3d import abi, cases, tuning
    from fvm3d.solver import Solver

    def build(prec):
        rng = np.random.default_rng(2024)
        cs = []
        for i in range(args.batch_cases):
            n = tuple(int(round(32 * 4 ** u)) for u in rng.uniform(size=3))
            recon = [abi.RECON_MUSCL, abi.RECON_WENO][int(rng.integers(2))]
            flux = [abi.FLUX_ROE, abi.FLUX_AUSM][int(rng.integers(2))]
            fam = cases.blast if rng.uniform() < 0.5 else cases.shock_tube
            cs.append(fam(n, seed=int(rng.integers(1 << 30)), reconstruct=recon, flux_split=flux,
                          limiter=abi.LIMITER_MINMOD, kappa=1.0 / 3.0, precision=prec,
                          compat=abi.COMPAT_TEXTBOOK))
        return cs

    steps = max(3, min(args.steps, 20))
    out = {"cases": args.batch_cases, "steps": steps, "unit": UNIT}
    for name, prec in (("fp64", abi.PREC_FP64), ("fp32_flux", abi.PREC_FP32_FLUX)):
        cs = build(prec)
        cells = sum(c.ncells for c in cs)
        s = Solver(cs[0].config())
        s.remove_case(0)
        for c in cs:
            cid = s.add_case(c.config())
            c.case_id = cid
            c.apply(s, case_id=cid, states=False)
        for c in cs:
            for b, q in enumerate(c.states):
                s.set_state(c.block_ids[b], q)
        s.step(2)
        win = timed_windows(s, steps, min_s=0.5)
        ms = statistics.median(win)
        failed = sum(1 for c in cs if s.case_state(c.case_id)["status"] != 0)
        out["cells"] = cells
        out["scheme_groups"] = len({(c.cfg["reconstruct"], c.cfg["flux_split"]) for c in cs})
        out[name] = {"value": sig(cells * 3 / (ms * 1e-3) / 1e9), "ms_per_step": sig(ms), "nonfinite": failed}
        s.close()
        if name == "fp32_flux":
            seq_ms = 0.0
            for c in cs:
                a = c.apply(Solver(c.config()))
                a.step(1)
                seq_ms += tuning.time_step(a, steps)
                a.close()
            out[name]["one_at_a_time"] = sig(cells * 3 / (seq_ms * 1e-3) / 1e9)
    out["fp32_over_fp64"] = sig(out["fp64"]["ms_per_step"] / out["fp32_flux"]["ms_per_step"])
    return out


# ---------------------------------------------------------------- Navier-Stokes leg
def tgv(args):
    """Compressible Taylor-Green vortex, 128^3, Ma 0.1, Re 1600, Pr 0.71,
    MUSCL / Van Albada + Roe + central viscous flux, SSP-RK3, CFL 0.5: FP64
    plain and FP32 flux (each autotuned), with the kinetic-energy difference
    after the steps."""
    from fvm3d import abi, cases, tuning
    from fvm3d.solver import Solver

    c = cases.taylor_green(N=128)
    steps = max(3, min(args.steps, 20))
    out = {"cells": c.ncells, "steps": steps}
    dV = c.meta["dx"] ** 3
    ke = {}
    forms = set(args.forms.split(",")) if args.only else {"fp64", "fp32"}
    for name, prec in (("fp64", abi.PREC_FP64), ("fp32_flux", abi.PREC_FP32_FLUX)):
        if name.split("_")[0] not in forms:
            continue
        s = c.apply(Solver(c.config(precision=prec)))
        t, z, _, sp = tuning.autotune(s, c.ncells, use_cache=False, reps=2)
        s.close()
        s = c.apply(Solver(c.config(precision=prec)))
        tuning.set_tuning(s, 0, t, z)
        tuning.set_tail_split(s, 0, sp)
        s.step(1)
        ms = tuning.time_step(s, steps)
        prof = tuning.profile_step(s)
        ke[name] = cases.kinetic_energy(s.get_state(0), dV)
        out[name] = {"value": sig(c.ncells * 3 / (ms * 1e-3) / 1e9), "ms_per_step": sig(ms), "tiling": [t, z, sp],
                     "viscous_ms": sig(sum(x for kk, x in prof if kk == "viscous"))}
        s.close()
    if len(ke) == 2:
        out["ke_rel_diff_fp32_vs_fp64"] = sig(abs(ke["fp32_flux"] - ke["fp64"]) / ke["fp64"])
        out["fp32_over_fp64"] = sig(out["fp64"]["ms_per_step"] / out["fp32_flux"]["ms_per_step"])
    out["unit"] = UNIT
    return out


# ---------------------------------------------------------------- accuracy leg
def accuracy_leg(args):
    """The vortex workload run for --accuracy-steps RK4 steps (CFL 0.5) in the
    exact, FP64 and FP32-flux forms and both compat modes: L1 (mean) and Linf
    density error against the exact solution (the vortex translated by the
    free stream to each run's own final time) and against the exact form,
    which is bit-identical to the oracle."""
    import numpy as np

    from fvm3d import abi, cases
    from fvm3d.solver import Solver

    c = cases.isentropic_vortex(N=args.n, layout="blocks8")
    steps = args.accuracy_steps
    out = {"cells": c.ncells, "steps": steps}
    for cname, compat in (("reference", abi.COMPAT_REFERENCE), ("textbook", abi.COMPAT_TEXTBOOK)):
        runs = {}
        for name, prec in (("exact", abi.PREC_FP64_EXACT), ("fp64", abi.PREC_FP64), ("fp32_flux", abi.PREC_FP32_FLUX)):
            s = c.apply(Solver(c.config(precision=prec, compat=compat)))
            t0 = time.perf_counter()
            t, _, _ = s.step(steps)
            sec = time.perf_counter() - t0
            rho = np.concatenate([s.get_state(b)[0].ravel() for b in range(len(c.blocks))])
            s.close()
            ex = np.concatenate([q[0].ravel() for q in cases.vortex_exact(c, t)])
            runs[name] = rho
            e = np.abs(rho - ex)
            out.setdefault(cname, {})[name] = {"t_end": t, "l1_vs_exact_solution": float(e.mean()),
                                               "linf_vs_exact_solution": float(e.max()), "wall_s": round(sec, 3)}
        for name in ("fp64", "fp32_flux"):
            d = np.abs(runs[name] - runs["exact"])
            out[cname][name]["l1_vs_exact_form"] = float(d.mean())
            out[cname][name]["linf_vs_exact_form"] = float(d.max())
    return out


# ---------------------------------------------------------------- 2D Riemann leg
def riemann2d_leg(args):
    """Four-quadrant 2D Riemann problem on 256 x 256 nodes of [0,1]^2, one
    block, transmissive regions, MUSCL / minmod (kappa 1/3) + Roe (entropy fix
    0.2), SSP-RK3, CFL 0.5: the reference's own kind of case at the size its
    case files use, in the three precision forms. A 2D plane counts its cells
    once."""
    from fvm3d import abi, cases, tuning
    from fvm3d.solver import Solver

    c = cases.riemann2d(n=256, seed=11, reconstruct=abi.RECON_MUSCL, limiter=abi.LIMITER_MINMOD,
                        kappa=1.0 / 3.0, flux_split=abi.FLUX_ROE, entropy_fix=0.2, rk_stages=3,
                        timestep_set=abi.DT_CFL, cfl=0.5)
    steps = max(20, args.steps * 10)
    out = {"cells": c.ncells, "steps": steps}
    forms = set(args.forms.split(",")) if args.only else {"fp64", "fp32", "exact"}
    for name, prec in (("fp64", abi.PREC_FP64), ("fp32_flux", abi.PREC_FP32_FLUX),
                       ("fp64_exact", abi.PREC_FP64_EXACT)):
        if {"fp64": "fp64", "fp32_flux": "fp32", "fp64_exact": "exact"}[name] not in forms:
            continue
        s = c.apply(Solver(c.config(precision=prec)))
        s.step(3)
        ms = statistics.median(timed_windows(s, steps, min_s=0.3))
        out[name] = {"value": sig(c.ncells * 3 / (ms * 1e-3) / 1e9), "ms_per_step": sig(ms)}
        s.close()
    if "fp64" in out and "fp32_flux" in out:
        out["fp32_over_fp64"] = sig(out["fp64"]["ms_per_step"] / out["fp32_flux"]["ms_per_step"])
    out["unit"] = UNIT
    return out


# ---------------------------------------------------------------- serving leg
def serve(args):
    """Poisson stream of seeded requests from the three solver
    configurations' families (2D four-quadrant Riemann problem, 8-block
    isentropic vortex with RK4, Navier-Stokes Taylor-Green vortex; grid edge
    log-uniform in 32..96, 100..400 steps; 32..192 and 200..2000 steps with
    --serve-full) in the FP32-flux form, served with continuous batching by
    the library's server, against the same stream served one request at a
    time in the plain FP64 form."""
    from fvm3d import abi, serving

    lo, hi, steps = (32, 192, (200, 2000)) if args.serve_full else (32, 96, (100, 400))
    make = serving.config_families(precision=abi.PREC_FP32_FLUX, sizes=(lo, hi))
    budget = int((16e9 if args.serve_full else 4e9) / (5 * 8 * 4))
    rate = 40.0 if not args.serve_full else 4.0
    out = {}

    def short(st):
        return {k: sig(float(st[k])) if isinstance(st[k], float) else st[k]
                for k in ("requests", "p50_s", "p99_s", "gcell_stage_per_s", "failed")}

    def stream():
        return serving.poisson_stream(args.serve_requests, rate=rate, seed=7, make_case=make, steps=steps)

    # warm-up, untimed: a short stream of every family, so the first timed
    # server does not pay the first use of each kernel and of the graph and
    # tensor-map machinery
    warm = serving.poisson_stream(6, rate=1000.0, seed=1, make_case=serving.config_families(
        precision=abi.PREC_FP32_FLUX, sizes=(lo, lo)), steps=(5, 10))
    srv = serving.Server(budget_cells=budget, chunk=8, max_active_cells=None)
    srv.run(warm, realtime=False)
    srv.close()
    serving.serve_one_at_a_time(warm, realtime=False, precision=abi.PREC_FP64)
    serving.serve_one_at_a_time(warm, realtime=False, precision=abi.PREC_FP32_FLUX)

    srv = serving.Server(budget_cells=budget, chunk=8, max_active_cells=None)
    out["continuous_batching"] = short(srv.run(stream()))
    srv.close()
    srv = serving.Server(budget_cells=budget, chunk=8, max_active_cells=1 << 22)
    out["continuous_batching_capped_4M_cells"] = short(srv.run(stream()))
    srv.close()
    out["one_at_a_time_fp64"] = short(serving.serve_one_at_a_time(stream(), precision=abi.PREC_FP64))
    out["arrival_rate_per_s"] = rate
    # at the arrival rate above the GPU is not saturated (the last request
    # arrives about 0.6 s into the stream), so the stream's throughput is
    # partly the arrival window's; the same requests all submitted at t = 0
    # measure the capacity of each way of serving them
    sat = {}
    srv = serving.Server(budget_cells=budget, chunk=8, max_active_cells=None)
    sat["continuous_batching"] = sig(srv.run(stream(), realtime=False)["gcell_stage_per_s"])
    srv.close()
    for name, prec in (("one_at_a_time_fp32", abi.PREC_FP32_FLUX), ("one_at_a_time_fp64", abi.PREC_FP64)):
        sat[name] = sig(serving.serve_one_at_a_time(stream(), realtime=False, precision=prec)["gcell_stage_per_s"])
    out["saturated_gcell_stage_per_s"] = sat
    out["workload"] = (f"C1-C3 families, edge {lo}..{hi}, {steps[0]}..{steps[1]} steps, FP32 flux, "
                       f"{budget * 160 / 1e9:.0f} GB budget")
    return out


# ---------------------------------------------------------------- residual norms leg
def resid_leg(args):
    """fvm_residual_norms and fvm_residual_norms_noalloc on one n^3 block's
    rhs already in device memory (the ClassIteration%compute_residual_sub
    step of a host that keeps rhs on the device): time per call, including
    the per-call scratch allocation of the first and the stream sync of both,
    and the rhs bytes read per second."""
    import ctypes

    import torch

    from fvm3d import abi

    lib = abi.load_library()
    lib.fvm_residual_norms_noalloc.argtypes = lib.fvm_residual_norms.argtypes
    n = args.n
    rhs = torch.randn(5 * n * n * n, dtype=torch.float64, device="cuda")
    res = torch.zeros(6, dtype=torch.float64, device="cuda")
    nv = (ctypes.c_int64 * 3)(n, n, n)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    out = {"cells": n ** 3, "unit": "GB/s"}
    for name in ("fvm_residual_norms", "fvm_residual_norms_noalloc"):
        fn = getattr(lib, name)
        for _ in range(3):
            assert fn(ctypes.c_void_p(rhs.data_ptr()), nv, ctypes.c_void_p(res.data_ptr()), st) == 0
        torch.cuda.synchronize()
        reps = 20
        t0 = time.perf_counter()
        for _ in range(reps):
            fn(ctypes.c_void_p(rhs.data_ptr()), nv, ctypes.c_void_p(res.data_ptr()), st)
        sec = (time.perf_counter() - t0) / reps
        out[name] = {"us_per_call": sig(sec * 1e6), "rhs_read_gbs": sig(40.0 * n ** 3 / sec / 1e9)}
    return out


# ---------------------------------------------------------------- CPU oracle
def cpu_oracle(n, steps, warmup, threads=None):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    from fvm3d import cases

    threads = threads or os.cpu_count() or 1
    orc.set_threads(threads)
    case = cases.isentropic_vortex(N=n, layout="blocks8")
    o = case.apply(orc.Oracle(case.config()))
    if warmup:
        o.step(warmup)
    t0 = time.perf_counter()
    o.step(steps)
    sec = time.perf_counter() - t0
    return case.ncells * 4 * steps / sec / 1e9, threads, sec


def main():
    args = parse()
    dist = Dist(args.gpus)
    base = {"metric": METRIC, "unit": UNIT, "n_gpus": dist.world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "data": "synthetic",
            "config": {"workload": WORKLOAD, "cells_per_gpu": args.n ** 3, "blocks": 8, "stages_per_step": 4,
                       "parallelism": f"replicas{dist.world}",
                       "l2": "inputs larger than L2 (state buffers 4 x 84 MB per GPU)"}}
    if args.impl == "reference":
        if dist.rank != 0:
            dist.close()
            return
        # a bounded sample: at most 60 steps (about 25 s on 16 host threads)
        ksteps = max(1, min(args.steps, 60))
        v, th, sec = cpu_oracle(args.n, ksteps, min(args.warmup, 3))
        line = dict(base)
        line.update({"impl": "reference", "value": v, "ms_per_step": sec / ksteps * 1e3, "dtype": "f64",
                     "n_gpus": dist.world,
                     "cpu_baseline": {"value": v, "unit": UNIT, "cores": th, "kind": "port",
                                      "sample": f"{ksteps} RK4 steps of the full 8-block {args.n}^3 case "
                                                f"({sec:.1f} s; C++ restatement of the reference path, OpenMP)"},
                     "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
        print(json.dumps(line))
        dist.close()
        return

    if args.only:
        leg = {"tgv": tgv, "riemann2d": riemann2d_leg, "accuracy": accuracy_leg, "batched": batched,
               "serve": serve, "resid": resid_leg}[args.only]
        if dist.rank == 0:
            print(json.dumps({"leg": args.only, **leg(args)}))
        dist.close()
        return

    res = product(args, dist)
    line = dict(base)
    line.update({"value": res.pop("value"), "ms_per_step": res.pop("ms_per_step"), "dtype": res.pop("dtype"),
                 "gpu_launches": res.pop("gpu_launches"), "roofline": res.pop("roofline"),
                 "clocks": res.pop("clocks")})
    if "e2e" in res:
        line["e2e"] = res.pop("e2e")
    line["timing"] = res.pop("timing")
    ratios = {}
    if "vortex_fp32_over_fp64" in res:
        ratios["vortex"] = res.pop("vortex_fp32_over_fp64")
    # the GPU legs first, the CPU baseline last: the oracle's OpenMP threads
    # keep spinning for a while after it returns and would slow the host
    # loops of the serving leg
    legs = {}
    if dist.world == 1 and not args.no_serve:
        legs["serving"] = serve(args)
    if dist.world == 1 and not args.no_batch:
        b = batched(args)
        legs["batched"] = b
        ratios["batch"] = b["fp32_over_fp64"]
        t = tgv(args)
        legs["navier_stokes_tgv"] = t
        ratios["tgv"] = t.get("fp32_over_fp64")
        r2 = riemann2d_leg(args)
        legs["riemann2d_256"] = r2
        ratios["riemann2d"] = r2.get("fp32_over_fp64")
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu:
        v, th, sec = cpu_oracle(args.n, 30, 1)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": th, "kind": "port",
                                "sample": "30 RK4 steps (after 1 untimed) of the full 8-block case on all host "
                                          f"threads ({sec:.1f} s; C++ restatement of the reference path)"}
        # the reference itself is serial: the same restatement on one thread
        v1, _, sec1 = cpu_oracle(args.n, 3, 0, threads=1)
        line["cpu_baseline_1thread"] = {"value": sig(v1), "cores": 1, "sample": f"3 RK4 steps ({sec1:.1f} s)"}
    sv = legs.pop("serving", None)
    line.update(legs)
    if sv is not None:
        line["serving"] = sv
        line["p50_s"] = sv["continuous_batching"]["p50_s"]
        line["p99_s"] = sv["continuous_batching"]["p99_s"]
    # the precision forms beside the headline, and the FP32 / FP64 speed
    # ratio of every configuration, last (the end of the line is what a
    # truncated log keeps)
    line.update(res)
    if ratios:
        line["fp32_over_fp64"] = ratios
    if dist.rank == 0:
        print(json.dumps(line))
    dist.close()


if __name__ == "__main__":
    main()
