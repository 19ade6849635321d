"""Benchmark of the CIPHER RHS on B200: cell-updates/s, FP32-mixed vs FP64.

Workload (the 3D grain-growth configuration): uniform periodic 128^3 grid,
2000 seeded Voronoi grains (splitmix64 seed 12345), at most 12 active phases
per cell, chemicalenergy none, interface energy 1, mobility 1, width 4 cells.
The input state is a diffuse-interface Voronoi state (phi profiles of width 4
around every grain boundary, active sets united with the face neighbours'),
built on the host; the inputs are larger than L2 (about 180 MB mixed and
270 MB FP64 of state per RHS), so no L2 flush is needed between launches.

A step is one RHS evaluation over all 2,097,152 cells.  One process per GPU;
ranks run independent replicas (the path has no cross-GPU exchange), so
`value` = cells * steps * ranks / max-over-ranks device time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cipher|reference]

`--impl reference` times the reference's own RHSFunction (compiled from its
sources into oracle/_ref) on all host cores, one process per core on a slab
with a one-cell halo, as `mpiexec -n p` runs it.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s mixed vs FP64 at 1e-6 rel err"
UNIT = "cell-updates/s"
WORKLOAD = dict(dim=3, res=(128, 128, 128), ngrains=2000, cap=12, seed=12345, width=4.0)
WORKLOAD_NAME = "3D grain growth 128^3, 2000 Voronoi grains, P=12, diffuse state (width 4)"
# GB/s used only when MEASURED_PEAKS.json is absent: an earlier STREAM-style
# copy measurement on B200, reported with peak_source "fallback"
HBM_PEAK_FALLBACK = 6650.0


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# --------------------------------------------------------------------------- #
# workload                                                                     #
# --------------------------------------------------------------------------- #

def build_problem():
    import cipher_b200 as cb
    w = WORKLOAD
    return cb.Problem.grain_growth(w["dim"], list(w["res"]), w["ngrains"], w["cap"], w["seed"])


def build_state(problem, mesh):
    import cipher_b200 as cb
    return cb.diffuse_state_aos(problem, mesh, WORKLOAD["width"])


def survey_bytes_per_cell(P: int, D: int, S: int, rb: int) -> int:
    """Compulsory bytes of one cell-update in the state format: the active
    set (P+1 uint16), the P phi slots, D chemical potentials, P*S site
    potentials and T read once; the P phi, D, P*S and T rates written once
    (phi and T in `rb` bytes, chemistry fields in FP64; neighbour values are
    re-reads served on chip)."""
    reads = 2 * (P + 1) + rb * P + 8 * D + 8 * P * S + rb
    writes = rb * P + 8 * D + 8 * P * S + rb
    return reads + writes


def state_exact_bytes(nsum: int, ncells: int, P: int, rb: int) -> int:
    """Bytes of one phase-field RHS launch that the sparse state actually
    holds: each cell's count, its active ids and active phi, and T read once;
    all P phi slots and T of F written once."""
    reads = 2 * ncells + 2 * nsum + rb * nsum + rb * ncells
    writes = ncells * (rb * P + rb)
    return reads + writes


def hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return HBM_PEAK_FALLBACK, "fallback"


def traffic_per_launch(kind: str):
    """DRAM bytes per launch of the RHS kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "rhs_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        e = d[kind]
        return float(e["dram_bytes_per_launch"]) * float(e.get("scale_to_workload", 1.0))
    except Exception:
        return None


# --------------------------------------------------------------------------- #
# clocks (NVML sampled from a thread during each timed region)                #
# --------------------------------------------------------------------------- #

class ClockSampler:
    HW = 0x8          # clocks_event_reasons: hw_slowdown
    HW_THERMAL = 0x40
    SW_THERMAL = 0x20
    SW_POWER = 0x4

    def __init__(self, device: int):
        self.samples = []
        self.reasons = 0
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(device)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None

    def _run(self):
        nv = self.nv
        reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            getattr(nv, "nvmlDeviceGetCurrentClocksThrottleReasons")
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                self.reasons |= reasons(self.h)
            except Exception:
                pass
            time.sleep(0.002)

    def start(self):
        if self.nv is None:
            return
        self._stop.clear()
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()

    def stop(self):
        if self._t is not None:
            self._stop.set()
            self._t.join()
            self._t = None

    def summary(self):
        if self.nv is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml unavailable"], "samples": 0}
        names = []
        r = self.reasons
        for bit, name in ((self.HW, "hw_slowdown"), (self.HW_THERMAL, "hw_thermal_slowdown"),
                          (self.SW_THERMAL, "sw_thermal_slowdown"), (self.SW_POWER, "sw_power_cap")):
            if r & bit:
                names.append(name)
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "reasons": names, "samples": len(self.samples)}


# --------------------------------------------------------------------------- #
# reference on host cores                                                     #
# --------------------------------------------------------------------------- #

def _ref_worker(args):
    lo, hi, Xs, reps, warm = args
    import cipher_b200 as cb
    import oracle
    P = build_problem()
    M = cb.Mesh(P, slab=(lo, hi))
    times = []
    with oracle.RefOracle(P, M) as R:
        for i in range(warm + reps):
            _, sec = R.rhs(Xs, with_time=True)
            if i >= warm:
                times.append(sec)
    return times


def reference_rate(X_aos: np.ndarray, procs: int, reps: int, warm: int):
    """cell-updates/s of the reference RHS on `procs` host processes; each
    step's time is the slowest process's (as an MPI run waits for it)."""
    import cipher_b200 as cb
    P = build_problem()
    nz = P.s.resolution[P.s.dim - 1]
    procs = max(1, min(procs, nz))
    bounds = [(nz * k // procs, nz * (k + 1) // procs) for k in range(procs)]
    jobs = []
    for lo, hi in bounds:
        M = cb.Mesh(P, slab=(lo, hi))
        jobs.append((lo, hi, np.ascontiguousarray(X_aos[M.cell_global()]), reps, warm))
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.map(_ref_worker, jobs)
    per_step = [max(r[k] for r in res) for k in range(reps)]
    ncells = int(np.prod(WORKLOAD["res"]))
    return ncells / statistics.mean(per_step), per_step


def workload_config(ncells: int, pcap: int, mean_n: float, world: int) -> dict:
    """the `config` object of both arms' lines (the same workload, the same keys)"""
    return {"workload": WORKLOAD_NAME, "cells": int(ncells), "max_phases": int(pcap),
            "mean_active_phases": float(mean_n), "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (no flush)"}


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# --------------------------------------------------------------------------- #
# arms                                                                         #
# --------------------------------------------------------------------------- #

def run_reference(args, rank, world):
    if rank != 0:
        return
    import oracle
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "metric": METRIC, "unit": UNIT,
                          "unavailable": "oracle/_ref/libcipher_ref.so was not built (reference sources absent)"}))
        return
    import cipher_b200 as cb
    P = build_problem()
    M = cb.Mesh(P)
    X = build_state(P, M)
    cores = host_cores()
    rate, per_step = reference_rate(X, cores, args.steps, args.warmup)
    ms = 1e3 * statistics.mean(per_step)
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(M.nowned, P.s.pf_size, float(X[:M.nowned, 0].mean()), world),
            "host_parallelism": f"{cores} host processes (slab + halo)",
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": f"each step one RHSFunction over all {int(np.prod(WORKLOAD['res']))} "
                                       f"cells split in {cores} slabs"},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def reduce_max(v: float, dist=None, device: str = "cpu") -> float:
    """the largest of every rank's v (the timing rule: a multi-GPU time is
    the slowest rank's); v itself without a process group.  `device` is
    where the backend reduces: cuda:<rank> for NCCL, cpu for gloo."""
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def time_launches(fn, steps, stream):
    """Run fn() `steps` times on `stream`, one CUDA-event pair per launch."""
    import torch
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for k in range(steps):
        starts[k].record(stream)
        fn()
        ends[k].record(stream)
    t1.record(stream)
    torch.cuda.synchronize()
    per = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    return t0.elapsed_time(t1), per


# --------------------------------------------------------------------------- #
# the other configurations (reported beside the headline)                     #
# --------------------------------------------------------------------------- #

def bytes_per_cell_update(P: int, D: int, S: int, rb: int) -> int:
    return survey_bytes_per_cell(P, D, S, rb)


def run_chemistry(dev: int, steps: int, peak: float):
    """config 2 shape on a uniform grid: 512^2, calphad2sl, 4 components,
    2 matrix grains + 20 precipitates, P = 15; the state is the SetUpProblem
    state advanced by 20 accepted device steps (interfaces start to spread)"""
    import torch
    import cipher_b200 as cb
    from cipher_b200 import workloads as W
    P = W.alloy_2d()
    M = cb.Mesh(P)
    A = P.aos
    X0 = cb.initial_state_aos(P, M)
    c64 = cb.Context(P, M, "fp64", device=dev)
    X = c64.alloc_state()
    c64.from_aos(X0, X)
    c64.chem_init(X)
    ts = cb.TimeStepper(c64, cb.ts_options(P, "2a", dt0=1e-6, dtmin=1e-12, dtmax=1e-2, reltol=1e-3, abstol=1e-3,
                                           max_steps=20))
    ts.solve(X, 0.0, 1.0)
    Xa = c64.to_aos(X)
    Xr = Xa.copy()
    Xr[:, A.pf_offset:A.pf_offset + A.pf_size] = Xr[:, A.pf_offset:A.pf_offset + A.pf_size].astype(np.float32)
    Xr[:, A.tm_offset] = Xr[:, A.tm_offset].astype(np.float32)
    c32 = cb.Context(P, M, "mixed", device=dev)
    out = {"workload": "2D alloy 512^2, calphad2sl 4 components (D=3, S=6), 2 grains + 20 precipitates, P=15, "
                       "uniform grid, state after 20 accepted steps",
           "cells": M.ncells, "mean_active_phases": float(Xa[:, 0].mean())}
    stream = torch.cuda.current_stream()
    F = {}
    for name, ctx, Xin in (("fp64", c64, Xr), ("mixed", c32, Xr)):
        dX, dF = ctx.alloc_state(), ctx.alloc_state()
        ctx.from_aos(Xin, dX)
        for _ in range(3):
            ctx.rhs(0.0, dX, dF)
        torch.cuda.synchronize()
        tot, per = time_launches(lambda: ctx.rhs(0.0, dX, dF), steps, stream)
        ctx.check()
        F[name] = ctx.to_aos(dF)
        rb = 8 if name == "fp64" else 4
        B = bytes_per_cell_update(A.pf_size, A.dp_size, A.sp_size, rb)
        ms = tot / steps
        out[name] = {"value": M.ncells / (ms / 1e3), "unit": UNIT, "ms_per_step": ms,
                     "bytes_per_cell_update": B, "roofline_frac": B * M.ncells / (ms / 1e3) / 1e9 / peak,
                     "kernels": ["k_chem_single", "k_chem_cell", "k_rhs_single", "k_item_list", "k_items",
                                 "k_rhs_general"]}
    errs = {}
    for nm, off, size in (("pf", A.pf_offset, A.pf_size), ("dp", A.dp_offset, A.dp_size),
                          ("ex", A.ex_offset, A.ex_size), ("tm", A.tm_offset, 1)):
        a, b = F["mixed"][:, off:off + size], F["fp64"][:, off:off + size]
        errs[nm] = float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
    out["mixed_rel_err_vs_fp64"] = errs
    out["mixed_speedup_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    return out


def run_config1_steps(dev: int, P, M, steps: int = 200):
    """configuration 1 as specified: the SetUpProblem start of the 128^3
    2000-grain problem (built on the device) stepped for `steps` accepted
    adaptive RK 2a steps from the reference's first step (mintimestep)
    through cipher_ts_solve (stage combinations, error norm, PostStep with
    its face maps, every step), in both precisions; cell-updates/s counts
    every RHS call of the solve and divides by the whole solve's device
    time"""
    import torch
    import cipher_b200 as cb
    out = {"workload": "3D grain growth 128^3, 2000 Voronoi grains, P=12, SetUpProblem start, "
                       f"{steps} accepted RK 2a steps through cipher_ts_solve (PostStep each step)"}
    stream = torch.cuda.current_stream()
    for name in ("fp64", "mixed"):
        ctx = cb.Context(P, M, name, device=dev)
        dX = ctx.alloc_state()
        ctx.init_sharp(dX)
        ts = cb.TimeStepper(ctx, cb.ts_options(P, "2a", max_steps=steps))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st = ts.solve(dX, 0.0, 1.0e30)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        out[name] = {"value": M.ncells * st.rhs_calls / (ms / 1e3), "unit": UNIT, "ms_total": ms,
                     "steps": int(st.steps), "rejected": int(st.rejected), "rhs_calls": int(st.rhs_calls),
                     "t_reached": float(st.t), "ms_per_rhs_call": ms / max(int(st.rhs_calls), 1),
                     "mean_active_phases_end": float(ctx.planes(dX)[0][0, :M.ncells].float().mean().item())}
        del ts, ctx, dX
    out["mixed_speedup_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    return out


def run_chemistry_amr(dev: int, steps: int = 20):
    """configuration 2 as specified: the 512^2 alloy (calphad2sl, 4
    components, 2 grains + 20 precipitates, P = 15) on an adaptive forest,
    levels 5-9 (the 512^2 grid is level 9), its SetUpProblem state coarsened
    4 times by the reference's marks; the RHS timed on the adapted mesh
    (cell-updates per leaf, and per effective 512^2 cell), then a solve with
    an adaptation every 10 accepted steps"""
    import ctypes as C
    import torch
    import cipher_b200 as cb
    from cipher_b200 import _lib as L
    from cipher_b200 import workloads as W
    P = W.alloy_2d()
    eff = int(np.prod([P.s.resolution[d] for d in range(2)]))
    o = cb.ts_options(P, "2a", dt0=1e-6, dtmin=1e-12, dtmax=1e-2, reltol=1e-3, abstol=1e-3)
    lib = L.load()
    stream = torch.cuda.current_stream()
    out = {"workload": "2D alloy, calphad2sl 4 components (D=3, S=6), 2 grains + 20 precipitates, P=15, "
                       "forest levels 5-9 over a 512^2 effective grid (initial coarsening x4, adaptation every "
                       "10 accepted steps)", "effective_cells": eff}
    for prec in ("fp64", "mixed"):
        amr = cb.AMR(P, [1, 1], 5, 9, 4, 10, o, prec, device=dev)
        ctx, X, m, _ = amr.state()
        lay = L.StateLayout()
        L.check(lib.cipher_ctx_layout(ctx, C.byref(lay)), "cipher_ctx_layout")
        F = torch.empty(int(lay.bytes), dtype=torch.uint8, device=f"cuda:{dev}")
        leaves = int(m.ncells)

        def rhs():
            L.check(lib.cipher_rhs(ctx, 0.0, X, C.c_void_p(F.data_ptr()), C.c_void_p(stream.cuda_stream)),
                    "cipher_rhs")
        for _ in range(3):
            rhs()
        torch.cuda.synchronize()
        tot, _ = time_launches(rhs, steps, stream)
        ms = tot / steps
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st = amr.solve(1.0, max_steps=30)
        e1.record(stream)
        torch.cuda.synchronize()
        _, _, m2, nad = amr.state()
        out[prec] = {"leaves": leaves, "rhs_ms": ms, "value": leaves / (ms / 1e3), "unit": UNIT,
                     "effective_value": eff / (ms / 1e3),
                     "solve": {"steps": int(st.steps), "rejected": int(st.rejected), "rhs_calls": int(st.rhs_calls),
                               "ms_total": e0.elapsed_time(e1), "adaptations": int(nad),
                               "leaves_end": int(m2.ncells), "t_reached": float(st.t)}}
        amr.close()
    out["mixed_speedup_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    return out


def _config1_only(dev: int, steps: int):
    import cipher_b200 as cb
    P = build_problem()
    return run_config1_steps(dev, P, cb.Mesh(P, grid_only=True), steps)


def _batched_leg(dev: int, precision: str, specs, t_end: float, n_alone: int):
    """one precision of the batched configuration: every domain attached to
    one batch and stepped together (one graph launch per step), then a
    sample solved one at a time with the single stepper"""
    import cipher_b200 as cb
    from cipher_b200 import workloads as W
    n_domains = len(specs)
    opts = cb.ts_options(W.batch_problem(specs[0]), "2a")
    doms = []
    for sp in specs:
        P = W.batch_problem(sp)
        M = cb.Mesh(P)
        ctx = cb.Context(P, M, precision, device=dev)
        X = ctx.alloc_state()
        ctx.from_aos(cb.initial_state_aos(P, M), X)
        doms.append((P, M, ctx, X))
    b = cb.Batch(opts, precision, device=dev)
    slots = [b.attach(ctx, X, 0.0, t_end) for _, _, ctx, X in doms]
    b.step()                      # builds the tables, tunes the tile shapes, captures the graph
    t0 = time.perf_counter()
    nsteps = 1
    while b.step() > 0:
        nsteps += 1
    b.flush()
    t_batch = time.perf_counter() - t0
    upd, failed = 0, 0
    for (P, M, _, _), sl in zip(doms, slots):
        st, status, _ = b.stats(sl)
        upd += M.ncells * st.rhs_calls
        failed += status != L_BATCH_FINISHED()
    b.close()
    # one at a time: every (n/n_alone)-th domain, solved alone from t = 0
    stride = max(1, n_domains // n_alone)
    t_alone, alone_upd, n_al = 0.0, 0, 0
    for k in range(0, n_domains, stride):
        P = W.batch_problem(specs[k])
        M = cb.Mesh(P)
        ctx = cb.Context(P, M, precision, device=dev)
        X = ctx.alloc_state()
        ctx.from_aos(cb.initial_state_aos(P, M), X)
        ts = cb.TimeStepper(ctx, opts)
        t1 = time.perf_counter()
        st = ts.solve(X, 0.0, t_end)
        t_alone += time.perf_counter() - t1
        alone_upd += M.ncells * st.rhs_calls
        n_al += 1
    return {"batched_steps": nsteps, "failed": failed,
            "batched": {"solves_per_s": n_domains / t_batch, "seconds": t_batch,
                        "cell_updates_per_s": upd / t_batch},
            "one_at_a_time": {"solves_per_s": n_al / t_alone, "seconds_per_solve": t_alone / n_al,
                              "cell_updates_per_s": alone_upd / t_alone, "sample": n_al},
            "speedup_solves_per_s": (n_domains / t_batch) / (n_al / t_alone)}


def run_batched(dev: int, n_domains: int, t_end: float, n_alone: int, precisions=("fp64", "mixed")):
    """config 3: independent 2D grain-growth domains of uneven size stepped
    together to t_end, FP32-mixed and FP64, each against a sample solved one
    at a time in the same precision"""
    import cipher_b200 as cb
    from cipher_b200 import workloads as W
    specs = W.batch_domains(n_domains)
    cells = sum(cb.Mesh(W.batch_problem(sp)).ncells for sp in specs)
    out = {"workload": f"{n_domains} 2D grain-growth domains, side 2^U[5,8] (32..256), 8-128 grains, P=8, "
                       f"SetUpProblem start, RK 2a at rtol=atol=1e-4 to t={t_end}",
           "domains": n_domains, "cells": cells}
    for precision in precisions:
        out[precision] = _batched_leg(dev, precision, specs, t_end, n_alone)
    if "fp64" in out and "mixed" in out:
        out["mixed_vs_fp64_batched_solves_per_s"] = (out["mixed"]["batched"]["solves_per_s"] /
                                                     out["fp64"]["batched"]["solves_per_s"])
    return out


def L_BATCH_FINISHED():
    from cipher_b200 import _lib as L
    return L.BATCH_FINISHED


def _serve_trace(dev: int, precision: str, trace, opts):
    """the trace served with continuous batching in `precision`: wall time,
    per-request latency from arrival, failures, peak HBM, host counters"""
    import cipher_b200 as cb
    from cipher_b200 import workloads as W
    srv = cb.Server(opts, precision, device=dev, hbm_budget=16 << 30, max_active=512)
    # warm the kernels and the tile tuner on one request of each kind
    for kind in ("gg", "alloy"):
        ex = next(t for t in trace if t[1] == kind)
        rid = srv.submit(W.trace_problem(ex[1], ex[2]), ex[4], ex[3])
        while srv.result(rid)[0].state != 2:
            srv.poll()
        srv.release(rid)
    ids, k = [], 0
    t0 = time.perf_counter()
    mono0 = time.monotonic()
    while True:
        now = time.perf_counter() - t0
        while k < len(trace) and trace[k][0] <= now:
            a, kind, args, init, te = trace[k]
            ids.append((srv.submit(W.trace_problem(kind, args), te, init), a))
            k += 1
        queued, active, _ = srv.poll()
        if queued == 0 and active == 0:
            if k == len(trace):
                break
            time.sleep(max(0.0, min(1e-3, trace[k][0] - (time.perf_counter() - t0))))
    wall = time.perf_counter() - t0
    lat, failed = [], 0
    for rid, a in ids:
        r, _ = srv.result(rid)
        failed += r.status != L_BATCH_FINISHED()
        lat.append(r.t_finish - (mono0 + a) if r.t_finish > 0 else float("nan"))
    used, peak_b = srv.usage()
    counters = srv.counters()
    srv.close()
    return wall, lat, failed, peak_b, counters


def run_serving(dev: int, rate: float, duration: float):
    """config 4: Poisson arrivals served with continuous batching (FP64, and
    FP32-mixed) vs the same trace served one request at a time with the
    plain FP64 path (each solved alone, FIFO)"""
    import cipher_b200 as cb
    from cipher_b200 import workloads as W
    trace = W.serving_trace(rate, duration)
    opts = cb.ts_options(W.trace_problem(trace[0][1], trace[0][2]), "2a", dt0=1e-6, dtmin=1e-12, dtmax=1.0,
                         reltol=1e-4, abstol=1e-4)
    pct = lambda v, q: float(np.percentile(np.asarray(v), q))
    served = {}
    failed = 0
    for precision in ("fp64", "mixed"):
        wall, lat, nf, peak_b, counters = _serve_trace(dev, precision, trace, opts)
        failed += nf
        served[precision] = {"solves_per_s": len(trace) / wall, "p50_s": pct(lat, 50), "p99_s": pct(lat, 99),
                             "peak_hbm_bytes": peak_b, "host_counters": counters}
    # the same trace one request at a time: each solved alone, FIFO from its arrival
    solve = []
    for a, kind, args, init, te in trace:
        P = W.trace_problem(kind, args)
        # the same work the server does per request: grid, context, the
        # SetUpProblem state on the device, the solve, the result to host
        t1 = time.perf_counter()
        M = cb.Mesh(P, grid_only=True)
        ctx = cb.Context(P, M, "fp64", device=dev)
        X = ctx.alloc_state()
        ctx.init_sharp(X)
        cb.TimeStepper(ctx, opts).solve(X, 0.0, te)
        ctx.to_aos(X)
        solve.append(time.perf_counter() - t1)
    fin, lat1 = 0.0, []
    for (a, *_), sv in zip(trace, solve):
        start = max(a, fin)
        fin = start + sv
        lat1.append(fin - a)
    return {"workload": f"Poisson({rate}/s) arrivals for {duration} s: 3/4 grain growth 64^2-256^2 to t=5, "
                        f"1/4 binary two-phase calphaddis 64^2-128^2 to t=0.02; RK 2a, rtol=atol=1e-4",
            "requests": len(trace), "failed": failed,
            "served": served["fp64"], "served_mixed": served["mixed"],
            "one_at_a_time": {"solves_per_s": len(trace) / fin, "p50_s": pct(lat1, 50), "p99_s": pct(lat1, 99),
                              "mean_solve_s": float(np.mean(solve)), "precision": "fp64"}}


def run_cipher(args, rank, world, local_rank):
    import torch
    import cipher_b200 as cb
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(local_rank)
    dev = local_rank

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v: float) -> float:
        return reduce_max(v, dist, f"cuda:{dev}")

    t_setup = time.time()
    P = build_problem()
    M = cb.Mesh(P)
    X = build_state(P, M)
    Lay = P.aos
    Pcap = P.s.pf_size
    ncells = M.nowned
    nsum = int(X[:, Lay.as_offset].sum())
    # the mixed path stores phi and T in FP32; both paths get those values
    X32 = X.copy()
    X32[:, Lay.pf_offset:Lay.pf_offset + Pcap] = X32[:, Lay.pf_offset:Lay.pf_offset + Pcap].astype(np.float32)
    X32[:, Lay.tm_offset] = X32[:, Lay.tm_offset].astype(np.float32)
    log(f"[rank {rank}] setup {time.time() - t_setup:.1f}s, mean active phases {nsum / ncells:.2f}")

    c64 = cb.Context(P, M, "fp64", device=dev)
    c32 = cb.Context(P, M, "mixed", device=dev)
    X64d, F64d = c64.alloc_state(), c64.alloc_state()
    X32d, F32d = c32.alloc_state(), c32.alloc_state()
    c64.from_aos(X, X64d)
    c32.from_aos(X32, X32d)
    stream = torch.cuda.current_stream()

    # accuracy of the mixed path against FP64 on the same input values
    Xc, Fc = c64.alloc_state(), c64.alloc_state()
    c64.from_aos(X32, Xc)
    c64.rhs(0.0, Xc, Fc)
    c32.rhs(0.0, X32d, F32d)
    c64.check()
    c32.check()
    Fa, Fb = c64.to_aos(Fc), c32.to_aos(F32d)
    sl = slice(Lay.pf_offset, Lay.pf_offset + Pcap)
    rel_err = float(np.abs(Fb[:, sl] - Fa[:, sl]).max() / np.abs(Fa[:, sl]).max())
    del Xc, Fc, Fa, Fb
    # the FP64 closed form against the FP64 reference-order kernel on the FP64 state
    Fref, Fcf = c64.alloc_state(), c64.alloc_state()
    c64.rhs(0.0, X64d, Fref)
    c64.set_rhs_form("closed")
    c64.rhs(0.0, X64d, Fcf)
    c64.set_rhs_form("reference")
    c64.check()
    Fa, Fb = c64.to_aos(Fref), c64.to_aos(Fcf)
    rel_err_cf = float(np.abs(Fb[:, sl] - Fa[:, sl]).max() / np.abs(Fa[:, sl]).max())
    del Fref, Fcf, Fa, Fb

    for _ in range(args.warmup):
        c64.rhs(0.0, X64d, F64d)
        c32.rhs(0.0, X32d, F32d)
    barrier()

    clk = ClockSampler(dev)
    # FP64 timed region
    barrier()
    clk.start()
    tot64, per64 = time_launches(lambda: c64.rhs(0.0, X64d, F64d), args.steps, stream)
    barrier()
    # mixed timed region (the headline)
    barrier()
    tot32, per32 = time_launches(lambda: c32.rhs(0.0, X32d, F32d), args.steps, stream)
    barrier()
    # FP64 closed form (the mixed kernel's algebra on the FP64 state)
    c64.set_rhs_form("closed")
    for _ in range(args.warmup):
        c64.rhs(0.0, X64d, F64d)
    barrier()
    totcf, percf = time_launches(lambda: c64.rhs(0.0, X64d, F64d), args.steps, stream)
    barrier()
    c64.set_rhs_form("reference")
    clk.stop()
    c64.check()
    c32.check()
    tot64 = max_over_ranks(tot64)
    tot32 = max_over_ranks(tot32)
    totcf = max_over_ranks(totcf)

    # end to end through the host-buffer entry point (reference AoS layout,
    # pinned host memory, copies inside the timed region)
    hx = torch.from_numpy(X).pin_memory()
    hf = torch.empty_like(hx).pin_memory()
    e2e_steps = max(1, min(args.steps, 10))
    c32.rhs_aos_host(0.0, hx, hf)
    barrier()
    clk2 = ClockSampler(dev)
    clk2.start()
    tot_e2e, _ = time_launches(lambda: c32.rhs_aos_host(0.0, hx, hf), e2e_steps, stream)
    clk2.stop()
    barrier()
    tot_e2e = max_over_ranks(tot_e2e)
    aos_bytes = int(X.nbytes)

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return

    value = ncells * args.steps * world / (tot32 / 1e3)
    value64 = ncells * args.steps * world / (tot64 / 1e3)
    peak, peak_src = hbm_peak()
    avg32 = statistics.mean(per32) / 1e3
    avg64 = statistics.mean(per64) / 1e3
    valuecf = ncells * args.steps * world / (totcf / 1e3)
    avgcf = statistics.mean(percf) / 1e3
    b32 = survey_bytes_per_cell(Pcap, 0, 0, 4) * ncells
    b64 = survey_bytes_per_cell(Pcap, 0, 0, 8) * ncells
    e32 = state_exact_bytes(nsum, ncells, Pcap, 4)
    e64 = state_exact_bytes(nsum, ncells, Pcap, 8)
    ach32 = b32 / avg32 / 1e9
    ach64 = b64 / avg64 / 1e9
    tr32 = traffic_per_launch("mixed")
    tr64 = traffic_per_launch("fp64")

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        import oracle
        if oracle.ref_available():
            cores = host_cores()
            rate, per_step = reference_rate(X, cores, 2, 1)
            cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": "reference",
                   "sample": f"2 timed RHSFunction calls (after 1 warm-up) over all {ncells} cells, "
                             f"{cores} processes on z-slabs with a one-cell halo"}
        else:
            rate, sec = None, None
            t0 = time.time()
            oracle.port_rhs(P, M, X)
            rate = ncells / (time.time() - t0)
            cpu = {"value": rate, "unit": UNIT, "cores": 1, "kind": "port",
                   "sample": f"1 RHS over all {ncells} cells, one thread"}

    c = clk.summary()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": tot32 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": workload_config(ncells, Pcap, nsum / ncells, world),
        "fp64": {"value": value64, "unit": UNIT, "ms_per_step": tot64 / args.steps,
                 "roofline_frac": ach64 / peak, "algorithmic_bytes_per_launch": b64,
                 "state_exact_roofline_frac": e64 / avg64 / 1e9 / peak},
        "fp64_closed_form": {"value": valuecf, "unit": UNIT, "ms_per_step": totcf / args.steps,
                             "roofline_frac": b64 / avgcf / 1e9 / peak, "rel_err_vs_reference_order": rel_err_cf,
                             "kernel": "k_rhs_pf_items<3,int,double>"},
        "mixed_speedup_vs_fp64": value / value64,
        "mixed_speedup_vs_fp64_closed_form": value / valuecf,
        "mixed_rel_err_vs_fp64": rel_err,
        "roofline": {"bound": "hbm", "achieved": ach32, "peak": peak, "unit": "GB/s", "frac": ach32 / peak,
                     "traffic": tr32, "peak_source": peak_src, "algorithmic_bytes_per_launch": b32,
                     "bytes_per_cell_update": b32 // ncells, "fp64_format_frac": b64 / avg32 / 1e9 / peak,
                     "state_exact_bytes_per_launch": e32, "state_exact_frac": e32 / avg32 / 1e9 / peak,
                     "kernel": "k_rhs_pf_items<3,int,float>"},
        "cpu_baseline": cpu,
        "e2e": {"value": ncells * e2e_steps * world / (tot_e2e / 1e3), "unit": UNIT,
                "h2d_bytes_per_step": aos_bytes, "d2h_bytes_per_step": aos_bytes,
                "path": "cipher_rhs_aos_host, reference AoS doubles in pinned host memory"},
        "clocks": {"sm_mhz": c["sm_mhz"], "sm_max_mhz": c["sm_max_mhz"], "reasons": c["reasons"],
                   "samples": c["samples"]},
        "gpu_launches": args.steps,
    }
    if not args.no_extra and world == 1:
        for key, fn in (("config1_steps", lambda: run_config1_steps(dev, P, M, 200)),
                        ("chemistry_amr", lambda: run_chemistry_amr(dev, 20)),
                        ("chemistry", lambda: run_chemistry(dev, 20, peak)),
                        ("batched", lambda: run_batched(dev, 256, 50.0, 16)),
                        ("serving", lambda: run_serving(dev, 50.0, args.serving_seconds))):
            t1 = time.time()
            try:
                line[key] = fn()
            except Exception as exc:       # a failed extra leg must not lose the headline line
                line[key] = {"error": f"{type(exc).__name__}: {exc}"}
            log(f"{key}: {time.time() - t1:.1f}s")
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="cipher", choices=["cipher", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the chemistry, batched and serving legs reported beside the headline")
    ap.add_argument("--only", choices=["chemistry", "batched", "serving", "config1_steps", "chemistry_amr"],
                    help="run one of the legs beside the headline alone (for profiling) and print its object")
    ap.add_argument("--batch-domains", type=int, default=256, help="--only batched: number of domains")
    ap.add_argument("--batch-t-end", type=float, default=50.0, help="--only batched: end time of every domain")
    ap.add_argument("--batch-precisions", default="fp64,mixed", help="--only batched: precisions to run")
    ap.add_argument("--serving-seconds", type=float, default=60.0,
                    help="length of the serving leg's arrival trace (Poisson, 50 requests/s)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    import cipher_b200.build as b
    if not os.path.exists(b.LIB):
        b.build()
    if args.only:
        import torch
        torch.cuda.set_device(local_rank)
        peak, _ = hbm_peak()
        fn = {"chemistry": lambda: run_chemistry(local_rank, args.steps, peak),
              "batched": lambda: run_batched(local_rank, args.batch_domains, args.batch_t_end, 16,
                                             tuple(args.batch_precisions.split(","))),
              "serving": lambda: run_serving(local_rank, 50.0, args.serving_seconds),
              "config1_steps": lambda: _config1_only(local_rank, args.steps),
              "chemistry_amr": lambda: run_chemistry_amr(local_rank, args.steps)}[args.only]
        print(json.dumps({args.only: fn()}), flush=True)
    elif args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_cipher(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
