"""Learned warm start: data from the library's own solves, training, and the comparison.

    python -m i3elvis_b200.learned [--n 33] [--train 48] [--test 8] [--iters 600] [--out FILE]

1. Data: seeded random-inclusion models (``model.random_inclusions``).  For each seed the
   model is prepared like the reference's initial-condition passes (``in3mg.c:990-1031``) and
   advanced ``--steps`` time steps; before every Stokes solve the network's inputs are
   recorded (log10 eta, rho, the start velocity) and after it the target (converged v, P
   minus the start).  The solves are the library's mixed-precision FGMRES to relative
   residual 1e-8, started the reference's way (the previous step's v, P).
2. Training: Adam on the GPU (``i3g_unet_train_step``) over random mini-batches.
3. Comparison on held-out seeds, every step run twice from identical states: default start
   (step 0: zero velocity and hydrostatic pressure, later steps: the previous step's
   solution) against the learned start (default + network correction, kept by the solver only
   when its residual is lower).  Reported: relative residual of each start, V-cycles and
   Stokes milliseconds to 1e-8.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import sys
import time

import numpy as np

from . import abi, config, lib, model, runtime
from .prn import YEAR
from .warmstart import UNet, guess_info


@dataclasses.dataclass
class Case:
    n: int = 33
    size_km: float = 200.0
    mnum: int = 2
    count: int = 30
    r_km: tuple = (8.0, 24.0)
    contrast: float | None = None

    @property
    def multinum(self):
        return {17: 2, 33: 2, 65: 3, 129: 4}.get(self.n, 2)


MIXED_SWEEPS = {4: ((2, 4, 4, 8, 0), (2, 4, 4, 8, 16)), 3: ((2, 4, 4, 0), (2, 4, 4, 8)), 2: ((2, 4, 0), (2, 4, 8))}


def build(case: Case, seed: int):
    """Seeded inclusion model and its mode (relaxation set and file row as the benchmark's)."""
    prn, spec = model.random_inclusions(n=case.n, size_km=case.size_km, mnum=case.mnum, multinum=case.multinum,
                                        seed=seed, count=case.count, r_km=case.r_km, contrast=case.contrast)
    mn = case.multinum
    dx = case.size_km * 1e3 / (case.n - 1)
    mode = config.Mode(
        infile="in0.prn", multinum=mn, multicyc=1, multinnn=MIXED_SWEEPS[mn],
        p0koef=0.71, p1koef=1.0, v0koef=0.7, v1koef=0.7, nubeg=1e18, nuend=1e24,
        files=[config.OutFile("out1.prn", maxxystep=0.5 * dx, maxtmstep_yr=1e9, nubeg=1e18, nuend=1e24,
                              p0koef=0.71, p1koef=1.0, p0koef2=0.71, p1koef2=0.0, multinum=mn, multinum2=mn)])
    return prn, mode


def solver_params(mode, rtol=1e-8):
    return abi.make_params(mode, stokes_rtol=rtol, stokes_maxcyc=3000, heat_rtol=1e-10, precision=1, krylov=8,
                           warm_start=1)


def _advance(ctx, mode, f, n0, timestep):
    """The rest of the reference time step after the Stokes solve (i3mg.c:112-146)."""
    if timestep:
        ctx.heat(n0, timestep)
        ctx.move_markers(timestep)
    ctx.markers_to_nodes(timestep)
    ctx.add_time(timestep)


def record(net: UNet, case: Case, seeds, steps: int, slot0: int = 0, rtol=1e-8):
    """Run every seed for `steps` time steps, recording one sample per Stokes solve."""
    slot = slot0
    for seed in seeds:
        prn, mode = build(case, seed)
        ctx = lib.Context(abi.ModelBuffers(prn), solver_params(mode, rtol), abi.make_file_params(mode.files[0]))
        runtime.prepare(ctx)
        f = mode.files[0]
        for s in range(steps):
            net.capture_input(ctx, slot)
            dt = ctx.stokes(s, f.maxtmstep_yr * YEAR)
            net.capture_target(ctx, slot)
            slot += 1
            _advance(ctx, mode, f, s, dt)
        ctx.close()
    return list(range(slot0, slot))


def fit_scales(net: UNet, slots):
    """Normalisation from the recorded samples: mean/std of log10 eta and rho, RMS of the
    velocity and pressure targets."""
    le, ro, dv, dp = [], [], [], []
    for s in slots:
        in5, tg4 = net.get_sample(s)
        le.append(in5[0])
        ro.append(in5[1])
        dv.append(tg4[1:].ravel())
        dp.append(tg4[0])
    le, ro, dv, dp = (np.concatenate(a).astype(np.float64) for a in (le, ro, dv, dp))
    sc = (float(le.mean()), float(1.0 / max(le.std(), 1e-3)), float(ro.mean()), float(1.0 / max(ro.std(), 1e-3)),
          float(max(np.sqrt(np.mean(dv ** 2)), 1e-30)), float(max(np.sqrt(np.mean(dp ** 2)), 1e-30)))
    net.set_scales(*sc)
    return sc


def train(net: UNet, slots, iters: int, batch: int = 4, lr: float = 2e-3, seed: int = 0, log_every: int = 0):
    rng = np.random.default_rng(seed)
    hist = []
    for it in range(iters):
        b = rng.choice(slots, size=min(batch, len(slots)), replace=False)
        # cosine decay to a tenth of the initial rate
        lr_t = lr * (0.1 + 0.9 * 0.5 * (1 + np.cos(np.pi * it / max(iters - 1, 1))))
        hist.append(net.train_step(b, float(lr_t)))
        if log_every and it % log_every == 0:
            print(f"[learned] iter {it} loss {hist[-1]:.4e}", file=sys.stderr, flush=True)
    return hist


def compare(net: UNet, case: Case, seeds, steps: int, rtol=1e-8):
    """Per held-out seed and step: default start against learned start from identical states."""
    rows = []
    for seed in seeds:
        prn, mode = build(case, seed)
        f = mode.files[0]
        ctxs = []
        for _ in range(2):
            c = lib.Context(abi.ModelBuffers(prn), solver_params(mode, rtol), abi.make_file_params(f))
            runtime.prepare(c)
            ctxs.append(c)
        for s in range(steps):
            row = {"seed": seed, "step": s}
            dts = []
            for k, c in enumerate(ctxs):
                if k == 1:
                    net.predict(c)
                dt = c.stokes(s, f.maxtmstep_yr * YEAR)
                st = c.stats()
                tag = "default" if k == 0 else "learned"
                row[tag + "_cycles"] = st["stokes_cycles"]
                row[tag + "_ms"] = st["ms_stokes"]
                row[tag + "_rel0"] = st["stokes_rel0"]
                if k == 1:
                    used, rg, rd, al = guess_info(c)
                    row.update(guess_used=used, rel_guess=rg, rel_default=rd, alpha=al)
                dts.append(dt)
            # both contexts continue from the default run's state so that every step compares
            # the two starts on the same model (the converged solutions agree to the tolerance)
            for c in ctxs:
                _advance(c, mode, f, s, dts[0])
            rows.append(row)
        for c in ctxs:
            c.close()
    return rows


def summarize(rows):
    out = {}
    for s in sorted({r["step"] for r in rows}):
        rs = [r for r in rows if r["step"] == s]
        out[f"step{s}"] = {
            "default_cycles": float(np.mean([r["default_cycles"] for r in rs])),
            "learned_cycles": float(np.mean([r["learned_cycles"] for r in rs])),
            "default_ms": float(np.mean([r["default_ms"] for r in rs])),
            "learned_ms": float(np.mean([r["learned_ms"] for r in rs])),
            "rel0_default": float(np.exp(np.mean(np.log([r["rel_default"] for r in rs])))),
            "rel0_learned_guess": float(np.exp(np.mean(np.log([max(r["rel_guess"], 1e-300) for r in rs])))),
            "alpha_median": float(np.median([r["alpha"] for r in rs])),
            "guess_used": int(sum(r["guess_used"] == 1 for r in rs)), "cases": len(rs)}
    return out


def bench(n: int, reps: int = 10, layers=None, convs_only: bool = False):
    """Device times of the network on an n^3 grid: forward pass, training step (unless
    ``convs_only``), and each forward convolution in ``layers`` (default all) with its achieved
    bandwidth (algorithmic bytes / time)."""
    net = UNet(n, n, n, capacity=1, seed=1)
    N = n ** 3
    g = np.linspace(0.0, 1.0, n)
    zz, xx, yy = np.meshgrid(g, g, g, indexing="ij")
    in5 = np.stack([(21 + 2 * np.sin(5 * xx) * np.cos(3 * yy + zz)).ravel(), (3300 + 50 * np.cos(4 * zz + yy)).ravel(),
                    np.zeros(N), np.zeros(N), np.zeros(N)]).astype(np.float32)
    tg4 = np.stack([1e6 * np.sin(2 * xx + yy).ravel()] + [1e-10 * np.cos(k + 3 * yy).ravel() for k in range(3)]).astype(np.float32)
    net.set_scales(21.0, 0.5, 3300.0, 0.02, 1e-10, 1e6)
    net.set_sample(0, in5, tg4)
    ms_train, ms_fwd = net.time(reps) if not convs_only else (None, None)
    convs = []
    for layer in (range(15) if layers is None else layers):
        ms, by = net.time_conv(layer, 3 * reps)
        convs.append({"layer": layer, "ms": ms, "bytes": by, "gbs": by / (ms * 1e-3) / 1e9})
    net.close()
    return {"grid": n, "ms_forward": ms_fwd, "ms_train_step": ms_train, "convs": convs}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--bench", type=int, default=0, help="only time the network on an N^3 grid")
    ap.add_argument("--layers", default=None, help="with --bench: comma list of the convolutions to time")
    ap.add_argument("--reps", type=int, default=10, help="with --bench: timed repetitions")
    ap.add_argument("--convs-only", action="store_true", help="with --bench: skip the forward and training times")
    ap.add_argument("--n", type=int, default=33)
    ap.add_argument("--mnum", type=int, default=2)
    ap.add_argument("--train", type=int, default=48, help="training seeds")
    ap.add_argument("--test", type=int, default=8, help="held-out seeds")
    ap.add_argument("--steps", type=int, default=2, help="time steps per seed")
    ap.add_argument("--iters", type=int, default=600)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    import torch
    torch.cuda.set_device(0)
    if a.bench:
        layers = [int(v) for v in a.layers.split(",")] if a.layers else None
        print(json.dumps(bench(a.bench, a.reps, layers, a.convs_only)))
        return 0
    case = Case(n=a.n, mnum=a.mnum)
    nsamp = a.train * a.steps
    net = UNet(case.n, case.n, case.n, capacity=nsamp, seed=1)
    t0 = time.perf_counter()
    slots = record(net, case, range(1000, 1000 + a.train), a.steps)
    t_rec = time.perf_counter() - t0
    sc = fit_scales(net, slots)
    t0 = time.perf_counter()
    hist = train(net, slots, a.iters, a.batch, a.lr, log_every=max(a.iters // 10, 1))
    t_train = time.perf_counter() - t0
    ms_train, ms_fwd = net.time(5)
    rows = compare(net, case, range(5000, 5000 + a.test), a.steps)
    res = {"grid": case.n, "markers_per_cell": case.mnum ** 3, "inclusions": case.count, "train_seeds": a.train,
           "test_seeds": a.test, "steps_per_seed": a.steps, "samples": nsamp, "iters": a.iters, "batch": a.batch,
           "lr": a.lr, "scales": sc, "loss_first": hist[0], "loss_last": float(np.mean(hist[-20:])),
           "record_s": t_rec, "train_s": t_train, "ms_train_step": ms_train, "ms_forward": ms_fwd,
           "summary": summarize(rows), "rows": rows}
    js = json.dumps(res)
    print(js)
    if a.out:
        with open(a.out, "w") as fh:
            fh.write(js + "\n")
    net.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
