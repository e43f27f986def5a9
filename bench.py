#!/usr/bin/env python
"""Benchmark: seconds per marker-in-cell time step at 129^3 nodes, Stokes to relative residual
1e-8 (plus heat solve, RK4 marker advection and marker->node averaging), on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|mixed]
                    [--workload incl129|sphere33|incl65] [--impl ours|reference]

One step is one reference time step (i3mg.c:80-147) on a synthetic model of the named shape:
129^3 nodes in a 200 km cube, 27 jittered markers per cell (56.6 M markers), 100 seeded
spherical inclusions (radius 2-8 km, density 3250-3450), Arrhenius matrix viscosity clipped to
1e18-1e24 Pa s.  Inputs are resident in HBM when the timed region starts; the model is far
larger than L2, so no flush is needed.  Under torchrun (N > 1) every rank advances its own
model (replicas; the path has no cross-rank exchange), and the reported value is the
aggregate seconds per step: max-over-ranks time / (steps * N).
"""
from __future__ import annotations

import argparse
import copy
import json
import os
import shutil
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from i3elvis_b200 import abi, config, model  # noqa: E402
from i3elvis_b200.prn import write_prn  # noqa: E402

METRIC = "s/time-step at 129^3, Stokes residual 1e-8"

WORKLOADS = {
    "incl129": dict(n=129, mnum=3, multinum=4, seed=7, count=100,
                    desc="129^3 nodes, 200 km cube, 27 markers/cell (56.6M), 100 inclusions, Arrhenius 1e18-1e24"),
    "incl65": dict(n=65, mnum=3, multinum=3, seed=7, count=100,
                   desc="65^3 nodes, 200 km cube, 27 markers/cell, 100 inclusions, Arrhenius 1e18-1e24"),
    "sphere33": dict(n=33, mnum=3, multinum=2, seed=1,
                     desc="33^3 nodes, 100 km cube, 27 markers/cell, sinking sphere 1e23/1e21"),
    "subd257": dict(n=257, mnum=3, multinum=4, seed=11,
                    desc="257x129x257 nodes (y vertical), 1000x500x1000 km, 27 markers/cell (226.5M), 100 km "
                         "lithosphere 1e24, 45-degree slab +50 kg/m3, 10 km weak layer 1e19, Arrhenius mantle "
                         "1e19-1e22, Drucker-Prager 10 MPa + 0.6 P"),
}


def default_sweeps(mn):
    """Relaxation sweeps per level in the proportions of the reference's shipped mode.t3c
    (more sweeps on coarser levels), for multinum = mn."""
    return (8, 16, 16, 32, 32, 32)[:mn] + (0,), (8, 16, 16, 32, 32, 32)[:mn] + (64,)


# Sweeps of the FP32 V-cycle when it preconditions FGMRES: the Krylov iteration removes the slow
# components, so a lighter cycle (a quarter of the reference's sweeps) reaches the tolerance sooner
# in time (incl129, previous-step start: 24 V-cycles in 82 ms against 14 in 104 ms with the full
# sweeps).  On the coarsest level 4 sweeps do as well as 16 (incl129 with the quadratic start:
# 13-14 V-cycles either way, Stokes 36.0 -> 30.8 ms per step); one level-0 sweep per leg, or fewer
# on levels 1-3, costs more V-cycles than it saves.
MIXED_SWEEPS = {4: "2,4,4,8/2,4,4,8,4", 3: "2,4,4/2,4,4,4", 2: "2,4/2,4,4"}


def build_case(name, seed_offset=0, sweeps=None):
    """Seeded model and mode of a named workload.  ``sweeps`` = "d0,d1,../u0,u1,..,uc" replaces
    the relaxation sweeps per level (down leg / up leg, the coarsest level last on the up leg)."""
    w = WORKLOADS[name]
    if name.startswith("sphere"):
        prn, spec = model.sinking_sphere(n=w["n"], mnum=w["mnum"], multinum=w["multinum"], seed=w["seed"] + seed_offset)
        size = 100e3
    elif name.startswith("subd"):
        prn, spec = model.subduction(mnum=w["mnum"], multinum=w["multinum"], seed=w["seed"] + seed_offset)
        size = 1000e3 * (w["n"] - 1) / 256.0
    else:
        prn, spec = model.random_inclusions(n=w["n"], mnum=w["mnum"], multinum=w["multinum"],
                                            seed=w["seed"] + seed_offset, count=w["count"])
        size = 200e3
    mn = w["multinum"]
    down, up = default_sweeps(mn)
    if sweeps:
        d, u = sweeps.split("/")
        down = tuple(int(v) for v in d.split(",")) + (0,)
        up = tuple(int(v) for v in u.split(","))
        if len(down) != mn + 1 or len(up) != mn + 1:
            raise SystemExit(f"--sweeps needs {mn} down and {mn + 1} up counts")
    dx = size / (w["n"] - 1)
    mode = config.Mode(
        infile="in0.prn", multinum=mn, multicyc=1, multinnn=(down, up),
        p0koef=0.71, p1koef=1.0, v0koef=0.7, v1koef=0.7, nubeg=1e18, nuend=1e24,
        files=[config.OutFile("out1.prn", maxxystep=0.5 * dx, maxtmstep_yr=1e9, nubeg=1e18, nuend=1e24,
                              p0koef=0.71, p1koef=1.0, p0koef2=0.71, p1koef2=0.0, multinum=mn, multinum2=mn)])
    return prn, mode


def host_threads():
    """CPU threads this process may use: its affinity set, capped by a cgroup CPU quota."""
    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        n = os.cpu_count() or 1
    try:
        with open("/sys/fs/cgroup/cpu.max") as fh:
            quota, period = fh.read().split()[:2]
        if quota != "max":
            n = max(1, min(n, int(int(quota) / int(period))))
    except (OSError, ValueError):
        pass
    return n


def max_over_ranks(x, world, device):
    """Largest value of x over all ranks (the job's time is the slowest rank's)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def per_step_seconds(ms_max, steps, world):
    """Aggregate seconds per time step of the whole job: world replicas each ran `steps` steps
    in ms_max milliseconds."""
    return ms_max / 1e3 / (steps * world)


def log(msg):
    print(f"[bench {time.strftime('%H:%M:%S')}] {msg}", file=sys.stderr, flush=True)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """SM clock, power and clock-event (throttle) reasons sampled during the timed region: NVML
    read-only queries every 20 ms from a thread, else nvidia-smi every 200 ms.  Nothing is set."""
    PERIOD_S = 0.02
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, dev, nvml=None):
        self.dev = dev          # CUDA device index
        self.nvml = nvml        # an NVML module (pynvml when None)
        self.proc = None
        self.file = None
        self.thread = None
        self.rows = []          # (sm MHz, max sm MHz, W, [4 reason flags])

    def _nvml_index(self):
        """NVML index of the CUDA device (CUDA_VISIBLE_DEVICES may renumber the devices)."""
        try:
            import torch
            return int(torch.cuda._get_nvml_device_index(self.dev))
        except Exception:
            return self.dev

    def _start_nvml(self):
        try:
            nv = self.nvml
            if nv is None:
                import pynvml as nv
            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByIndex(self._nvml_index())
            reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            bits = [getattr(nv, "nvmlClocksEventReason" + k, d) for k, d in
                    (("HwSlowdown", 0x8), ("HwThermalSlowdown", 0x40), ("SwThermalSlowdown", 0x20), ("SwPowerCap", 0x4))]
            smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))

            def sample():
                m = int(reasons(h))
                return (float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)), smax, nv.nvmlDeviceGetPowerUsage(h) / 1000.0,
                        ["Active" if m & b else "Not Active" for b in bits])
            sample()            # a failing query falls back to nvidia-smi here, not in the thread
        except Exception:
            return False
        self._nv, self._stop = nv, threading.Event()

        def run():
            while True:
                try:
                    self.rows.append(sample())
                except Exception:
                    pass
                if self._stop.wait(self.PERIOD_S):
                    break
        self.thread = threading.Thread(target=run, daemon=True)
        self.thread.start()
        return True

    def start(self):
        self.rows = []
        if self._start_nvml() or not shutil.which("nvidia-smi"):
            return
        self.file = tempfile.NamedTemporaryFile("w+", delete=False, suffix=".csv")
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self._nvml_index()), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits", "-lms", "200"],
                                     stdout=self.file, stderr=subprocess.DEVNULL)

    def stop(self):
        source = None
        if self.thread:
            self._stop.set()
            self.thread.join()
            try:
                self._nv.nvmlShutdown()
            except Exception:
                pass
            source = "nvml"
        elif self.proc:
            self.proc.terminate()
            self.proc.wait()
            self.file.flush()
            with open(self.file.name) as fh:
                for line in fh:
                    f = [x.strip() for x in line.split(",")]
                    if len(f) >= 7:
                        try:
                            self.rows.append((float(f[0]), float(f[1]), float(f[2]), f[3:7]))
                        except ValueError:
                            pass
            os.unlink(self.file.name)
            source = "nvidia-smi"
        rows = self.rows
        if not rows:
            return None
        reasons = sorted({self.NAMES[i] for r in rows for i, v in enumerate(r[3]) if v.lower() == "active"})
        return {"sm_mhz": float(np.median([r[0] for r in rows])), "sm_max_mhz": max(r[1] for r in rows),
                "power_w_max": max(r[2] for r in rows), "samples": len(rows), "reasons": reasons, "source": source}


# titerate (heat3mg.c:463-560) repeats its iteration block until heatsum <= HEATMIN, which its
# racy multi-threaded relaxation may never reach; the reference steps stop it after this many
# blocks (the count used is in each step's "heat_blocks")
REF_HEAT_CAP = 20
# V-cycles per reference step: the reference's lexicographic multigrid does not reach relative
# residual 1e-8 on the inclusion models (65^3: 4e-7 after 300 cycles), so every timed step
# stops here and reports the residual it reached; its step time is a lower bound of the
# reference's time to 1e-8 (twice the plain FP64 GPU multigrid's ~20 cycles per step)
REF_MAX_CYCLES = 40


def reference_steps(prn, mode, rtol, reps, threads, dt=0.0, timeout=3000):
    """Whole time steps of the reference's own functions on this workload, wall clock, all
    host threads: its initial-condition passes, then ``reps`` steps of vpiterate set-up,
    V-cycles to ``rtol`` (at most REF_MAX_CYCLES), titerate, movemark and ronurecalc.  Returns
    the per-step JSON records (None without the reference harness)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not O.have_reference():
        return None
    args = ("steps", rtol, REF_MAX_CYCLES, reps, 1, REF_HEAT_CAP) + ((repr(float(dt)),) if dt else ())
    with tempfile.TemporaryDirectory() as d:
        write_prn(os.path.join(d, "in0.prn"), prn)
        config.write_mode(os.path.join(d, "mode.t3c"), mode)
        config.write_file_t3c(os.path.join(d, "file.t3c"), 0)
        rs = O.run_reference_lines(d, *args, threads=threads, timeout=timeout)
        if (not rs or not all(r.get("vmax", 0.0) > 0 for r in rs)) and threads > 8:
            # the reference's racy multi-threaded Gauss-Seidel (move3mg.c:3089-3130) left no finite
            # velocity (seen with 16 and more threads at 129^3): time it again with 8 threads
            rs = O.run_reference_lines(d, *args, threads=8, timeout=timeout)
    return rs


def _ref_sample_text(rs, workload, rtol):
    cyc = [r["ncyc"] for r in rs]
    rel = [r["rel"] for r in rs]
    return (f"{len(rs)} whole reference time steps on the full {workload} model (one process, after the "
            f"reference's initial-condition passes and one untimed step): vpiterate set-up, V-cycles until the "
            f"relative residual <= {rtol:g} or {REF_MAX_CYCLES} cycles (cycles {cyc}, residual reached "
            f"{', '.join(f'{x:.2e}' for x in rel)}), the CFL step, titerate (at most {REF_HEAT_CAP} iteration blocks), "
            f"movemark, ronurecalc; {rs[0]['threads']} OpenMP threads")


def run_reference_arm(args):
    """--impl reference: the reference's CPU implementation of the step on this box's cores.
    Whole steps are timed (at most 4 after one untimed step, so that the arm ends within a few
    minutes); ``steps`` and ``warmup`` in the JSON are the counts actually run."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = host_threads()
    prn, mode = build_case(args.workload, sweeps=args.sweeps)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not O.have_reference():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_harness not built (reference sources absent at build time)"}))
        return 0
    warm, steps = min(args.warmup, 1), max(1, min(args.steps, 4))
    rs = reference_steps(prn, mode, args.rtol, warm + steps, threads)
    timed = rs[warm:]
    v = float(np.mean([r["step_s"] for r in timed]))
    sample = _ref_sample_text(timed, args.workload, args.rtol)
    print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": "s/step", "n_gpus": args.gpus,
                      "steps": len(timed), "warmup": warm, "ms_per_step": v * 1e3, "higher_is_better": False,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                      "config": {"workload": args.workload, "desc": WORKLOADS[args.workload]["desc"],
                                 "stokes_rtol": args.rtol, "max_vcycles_per_step": REF_MAX_CYCLES},
                      "stokes_cycles": [r["ncyc"] for r in timed], "stokes_rel": [r["rel"] for r in timed],
                      "phases_s": {k: float(np.mean([r[k] for r in timed])) for k in
                                   ("assemble_s", "stokes_s", "heat_s", "move_s", "r2n_s")},
                      "cpu_baseline": {"value": v, "unit": "s/step", "cores": timed[-1]["threads"], "kind": "reference",
                                       "sample": sample},
                      "e2e": {"value": v, "unit": "s/step", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--precision", default="mixed", choices=("fp64", "mixed"))
    ap.add_argument("--workload", default="incl129", choices=tuple(WORKLOADS))
    ap.add_argument("--rtol", type=float, default=1e-8)
    ap.add_argument("--sweeps", default=None, help="relaxation sweeps per level, 'down,../up,..'")
    ap.add_argument("--warm", type=int, default=3, choices=(1, 2, 3),
                    help="mixed precision: 1 previous step's solution, 2 linear extrapolation from the last two, "
                         "3 quadratic extrapolation from the last three")
    ap.add_argument("--krylov", type=int, default=8,
                    help="mixed precision: FGMRES restart length around the FP32 V-cycle (0: plain defect correction)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--maxcyc", type=int, default=3000, help="V-cycle cap of each Stokes solve")
    ap.add_argument("--allow-noconv", action="store_true",
                    help="a Stokes solve that reaches --maxcyc before the tolerance continues the step "
                         "(the residual reached is reported)")
    ap.add_argument("--no-fp64-compare", action="store_true",
                    help="mixed precision: skip the plain FP64 multigrid steps timed for comparison")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    import torch.distributed as dist
    from i3elvis_b200 import lib, runtime
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))

    prec = 1 if args.precision == "mixed" else 0
    sweeps = args.sweeps
    if sweeps is None and prec == 1 and args.krylov > 0:
        sweeps = MIXED_SWEEPS.get(WORKLOADS[args.workload]["multinum"])
    prn, mode = build_case(args.workload, seed_offset=rank, sweeps=sweeps)
    prn0 = prn
    krylov = args.krylov if prec == 1 else 0
    warm = args.warm if prec == 1 else 1
    par = abi.make_params(mode, stokes_rtol=args.rtol, stokes_maxcyc=args.maxcyc, heat_rtol=1e-10, precision=prec,
                          krylov=krylov, warm_start=warm)
    nc = args.allow_noconv
    buf = abi.ModelBuffers(prn, pinned=True)
    ctx = lib.Context(buf, par, abi.make_file_params(mode.files[0]))
    f = mode.files[0]
    log("model built and uploaded")
    runtime.prepare(ctx)
    log("prepared")
    cycles = []
    for i in range(args.warmup):
        runtime.time_step(ctx, mode, f, i, nc)
        cycles.append(ctx.stats()["stokes_cycles"])

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    log(f"warm-up done, V-cycles {cycles}")
    clocks = Clocks(local)
    l0 = ctx.stats()["kernel_launches"]
    barrier()
    clocks.start()
    ctx.timer_start()
    logs = []
    for i in range(args.steps):
        logs.append(runtime.time_step(ctx, mode, f, args.warmup + i, nc))
        st = ctx.stats()
        cycles.append(st["stokes_cycles"])
        logs[-1].update({k: st[k] for k in ("stokes_cycles", "stokes_rel", "stokes_rel0", "stokes_start", "ms_stokes",
                                            "ms_heat", "ms_move", "ms_r2n", "heat_cycles")})
    ms = ctx.timer_stop()
    barrier()
    clk = clocks.stop()
    launches = ctx.stats()["kernel_launches"] - l0
    ms_max = max_over_ranks(ms, world, "cuda")
    value = per_step_seconds(ms_max, args.steps, world)

    log(f"timed steps done: {ms_max / args.steps:.1f} ms/step")
    # end to end through the C ABI with host buffers: full state up, step, full state down
    e2e_steps = max(1, min(args.steps, 2))
    n, m = prn.nodenum, prn.marknum
    h2d = n * (8 + 4 * 15) + m * (4 * 12 + 1)
    d2h = h2d + n * 4 * 12
    # host buffers hold the current state, so each upload resumes it; an upload of exactly the
    # library's last solution keeps the extrapolated start, as in the device-resident steps
    ctx.download(abi.SYNC_ALL)
    barrier()
    e2e_cycles = []
    t0 = time.perf_counter()
    for i in range(e2e_steps):
        # nodal fields first; the 2.8 GB of marker copies overlap the Stokes solve (they are
        # first needed by the heat step's marker update)
        ctx.upload(abi.SYNC_NODES | abi.SYNC_MARKERS | abi.SYNC_ASYNC)
        runtime.time_step(ctx, mode, f, 100 + i, nc)
        ctx.download(abi.SYNC_ALL)
        e2e_cycles.append(ctx.stats()["stokes_cycles"])
    barrier()
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    e2e_value = max_over_ranks(e2e_s, world, "cuda") / world

    # the plain FP64 multigrid (the reference's iteration and sweeps) on the same state, for the
    # Stokes + heat speed-up of this configuration
    fp64_mg = None
    if prec == 1 and not args.no_fp64_compare:
        d64, u64 = default_sweeps(WORKLOADS[args.workload]["multinum"])
        m64 = copy.deepcopy(mode)
        m64.multinnn = (d64, u64)
        ctx.set_params(abi.make_params(m64, stokes_rtol=args.rtol, stokes_maxcyc=args.maxcyc, heat_rtol=1e-10, precision=0,
                                       krylov=0))
        runtime.time_step(ctx, m64, f, 200, nc)
        lg64 = []
        for i in range(args.steps):
            lg64.append(runtime.time_step(ctx, m64, f, 201 + i, nc))
            st = ctx.stats()
            lg64[-1].update({k: st[k] for k in ("stokes_cycles", "ms_stokes", "ms_heat", "stokes_rel")})
        ctx.set_params(par)
        s64 = float(np.mean([lg["ms_stokes"] + lg["ms_heat"] for lg in lg64]))
        s32 = float(np.mean([lg["ms_stokes"] + lg["ms_heat"] for lg in logs]))
        fp64_mg = {"ms_stokes": float(np.mean([lg["ms_stokes"] for lg in lg64])),
                   "ms_heat": float(np.mean([lg["ms_heat"] for lg in lg64])),
                   "stokes_cycles": [lg["stokes_cycles"] for lg in lg64],
                   "stokes_rel": [lg["stokes_rel"] for lg in lg64],
                   "sweeps": [list(d64), list(u64)],
                   "speedup_stokes_heat": s64 / s32}
        log(f"plain FP64 multigrid: {s64:.1f} ms Stokes+heat per step, this run {s32:.1f} ms")

    # rooflines of the step's main kernels, each timed live with an empty L2 before every launch
    # (library's cold-cache timer) against each kernel's algorithmic bytes per unit (marker,
    # node) times the units of one launch; the dominant kernel is the one with the most device
    # time per step
    peak, peak_src = peaks()
    traffic_tab = {}
    tf = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tf):
        try:
            with open(tf) as fh:
                traffic_tab = json.load(fh).get(args.workload, {})
        except Exception:
            traffic_tab = {}
    cyc = float(np.mean(cycles[args.warmup:])) if cycles[args.warmup:] else 0.0
    heat_cyc = float(np.mean([lg.get("heat_cycles", 0) for lg in logs])) if logs else 0.0
    sweeps0 = mode.multinnn[0][0] + mode.multinnn[1][0]
    specs = [("stokes_sweep_" + ("f32" if prec else "f64"), 8 if prec else 10, sweeps0 * cyc,
              "one level-0 multicolour sweep, %s (k_relax_vel x6, k_relax_p, boundary rows)" % ("FP32" if prec else "FP64"),
              "68 B/node FP32" if prec else "116 B/node FP64"),
             ("k_move", 5, 1.0, "RK4 marker advection", "45 B/marker + 13 nodal FP32 fields"),
             ("k_r2n_cells", 4, 1.0, "marker -> node sums", "25 B/marker + 48 B/node"),
             ("k_heat_mark_cells", 9, 1.0, "marker temperature update", "42 B/marker"),
             ("heat_sweep", 6, 4.0 * heat_cyc, "one level-0 heat sweep (k_heat_relax x2)", "32 B/node")]
    kernels = []
    for name, kind, per_step, what, unit_bytes in specs:
        kms, kbytes = ctx.time_kernel(kind, 10)
        ach = kbytes / (kms * 1e-3) / 1e9
        tr = traffic_tab.get(name)
        kernels.append({"kernel": name, "what": what, "algorithmic_bytes": unit_bytes, "ms_per_launch": kms,
                        "bytes_per_launch": kbytes, "achieved": ach, "frac": ach / peak, "launches_per_step": per_step,
                        "ms_per_step": kms * per_step, "traffic": tr})
    dom = max(kernels, key=lambda k: k["ms_per_step"])
    log("rooflines: " + ", ".join(f"{k['kernel']} {k['ms_per_launch']:.3f} ms {k['frac']:.2f}" for k in kernels))
    out = {
        "metric": METRIC, "value": value, "unit": "s/step", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if prec == 0 else "f32-in-f64", "data": "synthetic",
        "config": {"workload": args.workload, "desc": WORKLOADS[args.workload]["desc"], "precision": args.precision,
                   "stokes_rtol": args.rtol, "krylov": krylov, "warm_start": warm, "sweeps": [list(mode.multinnn[0]), list(mode.multinnn[1])],
                   "l2": "inputs larger than L2 (no flush)", "parallelism": f"replicas x{world}",
                   "stokes_maxcyc": args.maxcyc, "allow_noconv": bool(nc)},
        "timestep_s": float(np.median([lg["timestep"] for lg in logs])),
        "stokes_cycles": cycles[args.warmup:], "stokes_rel": [lg["stokes_rel"] for lg in logs],
        "stokes_rel0": [lg["stokes_rel0"] for lg in logs], "stokes_start": [lg["stokes_start"] for lg in logs], "phases_ms": {k: float(np.mean([lg[k] for lg in logs])) for k in
                                                           ("ms_stokes", "ms_heat", "ms_move", "ms_r2n")},
        "gpu_launches": int(launches),
        "fp64_multigrid": fp64_mg,
        "e2e": {"value": e2e_value, "unit": "s/step", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "stokes_cycles": e2e_cycles},
        "roofline": {"bound": "hbm", "kernel": dom["kernel"], "achieved": dom["achieved"], "peak": peak,
                     "peak_source": peak_src, "unit": "GB/s", "frac": dom["frac"], "traffic": dom["traffic"],
                     "bytes_per_launch": dom["bytes_per_launch"], "ms_per_launch": dom["ms_per_launch"],
                     "ms_per_step": dom["ms_per_step"], "l2": "flushed before every timed launch"},
        "kernels": kernels,
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            log("cpu baseline: reference steps")
            dts = [lg["timestep"] for lg in logs if lg.get("timestep")]
            rs = reference_steps(prn0, mode, args.rtol, 2, host_threads(), float(np.median(dts)) if dts else 0.0)
            log("cpu baseline done")
        except Exception as e:  # the CPU baseline is reported, never required
            rs = None
            out["cpu_baseline_error"] = str(e)[:300]
        if rs:
            r = rs[-1]
            out["cpu_baseline"] = {"value": r["step_s"], "unit": "s/step", "cores": r["threads"], "kind": "reference",
                                   "sample": _ref_sample_text(rs[1:], args.workload, args.rtol) +
                                   f" (time step fixed to this run's {r['timestep']:.4g} s); {json.dumps(r)}"}
    ctx.close()
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
