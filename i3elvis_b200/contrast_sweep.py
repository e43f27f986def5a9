"""Viscosity-contrast sweep: mixed precision against FP64 on the 129^3 inclusion model.

    python -m i3elvis_b200.contrast_sweep [--n 129] [--contrasts 1e2,1e4,1e6] [--krylov 12]
                                          [--maxcyc 3000] [--solvers fp64,fp64k,mixed]

For each contrast C the 100 seeded inclusions get viscosity contrasts log-uniform in [1, C]
against the Arrhenius matrix (binned into rock types as ``model.random_inclusions`` does).
From the same prepared state (nodes from markers, hydrostatic pressure, zero velocity) it
solves Stokes, then heat, three ways:

* ``ref``   the FP64 oracle solve: restarted FGMRES(12) on the FP64 residual preconditioned by
            the FP64 V-cycle -- no FP32 arithmetic anywhere -- towards relative residual 1e-11
            (at most 1500 V-cycles; the residual it reaches is reported as ``ref_rel``); every
            error below is measured against its FP64 solution vector;
* ``fp64``  the plain FP64 multigrid (the reference's iteration and sweeps) to 1e-8;
* ``fp64k`` the same FGMRES(12) with the FP64 V-cycle to 1e-8 (FP64 with Krylov acceleration);
* ``mixed`` the mixed-precision solver of the benchmark (FGMRES(12) preconditioned by the FP32
            V-cycle, light sweeps) to 1e-8.

It prints one JSON line per contrast with the V-cycle counts (capped at 3000; ``converged``
says whether 1e-8 was reached), times and the relative L2 errors of the FP64 solution vector's
Vx, Vy, Vz, P (pressure relative to the pinning cell) and of T against ``ref``.  The solves start cold (zero velocity), the hardest
start: in time stepping each solve starts from the previous step's solution.
"""
from __future__ import annotations

import argparse
import copy
import json

import numpy as np

from . import abi, config, lib, model, runtime
from .prn import YEAR


def _sweeps(mn, light):
    if light:
        d = (2, 4, 4, 8, 8, 8)[:mn] + (0,)
        u = (2, 4, 4, 8, 8, 8)[:mn] + (16,)
    else:
        d = (8, 16, 16, 32, 32, 32)[:mn] + (0,)
        u = (8, 16, 16, 32, 32, 32)[:mn] + (64,)
    return d, u


def _state(ctx):
    ctx.download(abi.SYNC_NODES)
    b = ctx.buf
    return {"pr": b.pr.copy(), **{f: b.f32[f].copy() for f in abi.NODE_F32}}


def _restore(ctx, s):
    b = ctx.buf
    b.pr[:] = s["pr"]
    for f in abi.NODE_F32:
        b.f32[f][:] = s[f]
    ctx.upload(abi.SYNC_NODES)


def _cfl(ctx, f):
    """Time step limit maxxystep / max|v| of the current velocities (move3mg.c:2608-2632)."""
    b = ctx.buf
    v = max(float(np.abs(b.f32[k]).max()) for k in ("vx", "vy", "vz"))
    return min(f.maxtmstep_yr * YEAR, f.maxxystep / v) if v > 0 else f.maxtmstep_yr * YEAR


def _rel(a, b):
    d = np.linalg.norm(a.astype(np.float64) - b.astype(np.float64))
    n = np.linalg.norm(b.astype(np.float64))
    return float(d / n) if n > 0 else float(d)


def run(n=129, contrasts=(1e2, 1e4, 1e6), mnum=3, multinum=4, seed=7, krylov=12, maxcyc=3000, solvers=None):
    out = []
    for C in contrasts:
        prn, _ = model.random_inclusions(n=n, mnum=mnum, multinum=multinum, seed=seed, count=100, contrast=C)
        dx = 200e3 / (n - 1)
        f = config.OutFile("o.prn", maxxystep=0.5 * dx, maxtmstep_yr=1e9, nubeg=1e18, nuend=1e24, p0koef=0.71,
                           p1koef=1.0, p0koef2=0.71, p1koef2=0.0, multinum=multinum, multinum2=multinum)
        mode = config.Mode(multinum=multinum, multicyc=1, multinnn=_sweeps(multinum, False), p0koef=0.71, p1koef=1.0,
                           v0koef=0.7, v1koef=0.7, nubeg=1e18, nuend=1e24, files=[f])
        light = copy.deepcopy(mode)
        light.multinnn = _sweeps(multinum, True)
        runs = {
            "ref": (light, dict(stokes_rtol=1e-11, stokes_maxcyc=1500, precision=0, krylov=krylov)),
            "fp64": (mode, dict(stokes_rtol=1e-8, precision=0, krylov=0)),
            "fp64k": (light, dict(stokes_rtol=1e-8, precision=0, krylov=krylov)),
            "mixed": (light, dict(stokes_rtol=1e-8, precision=1, krylov=krylov)),
        }
        if solvers:
            runs = {k: v for k, v in runs.items() if k == "ref" or k in solvers}
        ctx = lib.Context(abi.ModelBuffers(prn, pinned=True), abi.make_params(mode), abi.make_file_params(f))
        runtime.prepare(ctx)
        s0 = _state(ctx)
        res = {}
        for name, (md, solver) in runs.items():
            _restore(ctx, s0)
            ctx.set_params(abi.make_params(md, heat_rtol=1e-10, **{"stokes_maxcyc": maxcyc, **solver}))
            conv = True
            try:
                dt = ctx.stokes(0, f.maxtmstep_yr * YEAR)
            except lib.I3gError as e:
                if "NOCONV" not in str(e):
                    raise
                conv = False              # the solution after the cycle cap is still compared
                ctx.download(abi.SYNC_NODES)
                dt = _cfl(ctx, f)
            st = ctx.stats()
            sol = ctx.get(abi.A_SOL, 0, 4 * prn.nodenum).reshape(-1, 4)
            ctx.heat(0, dt)
            sh = ctx.stats()
            ctx.download(abi.SYNC_NODES)
            b = ctx.buf
            pin = (prn.head["pzinit"] * n + prn.head["pxinit"]) * n + prn.head["pyinit"]
            res[name] = {"vx": sol[:, 1].copy(), "vy": sol[:, 2].copy(), "vz": sol[:, 3].copy(),
                         "pr": sol[:, 0] - sol[pin, 0], "tk": b.f32["tk"].copy(), "cycles": st["stokes_cycles"],
                         "ms_stokes": st["ms_stokes"], "ms_heat": sh["ms_heat"], "rel": st["stokes_rel"], "dt": dt,
                         "converged": conv}
        ctx.close()
        ref = res["ref"]
        line = {"contrast": C, "n": n, "markers": prn.marknum, "ref_cycles": ref["cycles"], "ref_rel": ref["rel"]}
        line["krylov"] = krylov
        for name in ("fp64", "fp64k", "mixed"):
            if name not in res:
                continue
            r = res[name]
            line[name] = {"cycles": r["cycles"], "rel": r["rel"], "converged": r["converged"],
                          "ms_stokes": r["ms_stokes"], "ms_heat": r["ms_heat"],
                          "err": {k: _rel(r[k], ref[k]) for k in ("vx", "vy", "vz", "pr", "tk")},
                          "dt_rel": abs(r["dt"] - ref["dt"]) / ref["dt"]}
        print(json.dumps(line), flush=True)
        out.append(line)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=129)
    ap.add_argument("--contrasts", default="1e2,1e4,1e6")
    ap.add_argument("--krylov", type=int, default=12, help="FGMRES restart length (<= 16)")
    ap.add_argument("--maxcyc", type=int, default=3000, help="V-cycle cap of the 1e-8 solves")
    ap.add_argument("--solvers", default="fp64,fp64k,mixed", help="solvers besides the FP64 reference solve")
    a = ap.parse_args()
    run(n=a.n, contrasts=tuple(float(x) for x in a.contrasts.split(",")), krylov=a.krylov, maxcyc=a.maxcyc,
        solvers=tuple(a.solvers.split(",")))


if __name__ == "__main__":
    main()
