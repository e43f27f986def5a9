"""Convergence of Stokes solver variants on one model from a cold start.

    python -m i3elvis_b200.solver_study [--model subduction] [--dims 129,65,129] [--multinum 3]
                                        [--maxcyc 600]

Builds the model (``model.subduction``: lithosphere, 45-degree slab, weak layer, Arrhenius
mantle, Drucker-Prager yielding; or ``model.random_inclusions`` with ``--model inclusions``),
prepares it (nodes from markers, hydrostatic pressure, zero velocity) and, for each solver
variant, restores that state and solves Stokes towards relative residual 1e-8 with at most
``maxcyc`` V-cycles.  Prints one JSON line per variant: V-cycles, the momentum and continuity
relative residuals reached, and the device time.  The variants cover the relaxation schedule
(light 2,4,4,8 / heavy 8,16,16,32 sweeps per level), the precision of the V-cycle, the FGMRES
restart length, and the relaxation factors.
"""
from __future__ import annotations

import argparse
import json
import time

from . import abi, config, lib, model, runtime
from .prn import YEAR


def _mode(mn, d, u, dx, p0=0.71, p1=1.0, p12=0.0, v0=0.7, v1=0.7):
    f = config.OutFile("o.prn", maxxystep=0.5 * dx, maxtmstep_yr=1e9, nubeg=1e18, nuend=1e24, p0koef=p0, p1koef=p1,
                       p0koef2=p0, p1koef2=p12, multinum=mn, multinum2=mn)
    return config.Mode(infile="in0.prn", multinum=mn, multicyc=1, multinnn=(d, u), p0koef=p0, p1koef=p1, v0koef=v0,
                       v1koef=v1, nubeg=1e18, nuend=1e24, files=[f])


def run(kind="subduction", dims=(129, 65, 129), multinum=3, maxcyc=600, seed=11):
    nx, ny, nz = dims
    if kind == "subduction":
        prn, _ = model.subduction(nx=nx, ny=ny, nz=nz, mnum=2, multinum=multinum)
        dx = 1000e3 / (nx - 1)
    else:
        prn, _ = model.random_inclusions(n=nx, mnum=2, multinum=multinum, seed=seed, count=100)
        dx = 200e3 / (nx - 1)
    mn = multinum
    light = (tuple([2, 4, 4, 8, 8][:mn]) + (0,), tuple([2, 4, 4, 8, 8][:mn]) + (16,))
    heavy = (tuple([8, 16, 16, 32, 32][:mn]) + (0,), tuple([8, 16, 16, 32, 32][:mn]) + (64,))
    variants = [
        ("mixed light k8", light, 1, 8, {}), ("mixed heavy k8", heavy, 1, 8, {}), ("mixed light k16", light, 1, 16, {}),
        ("mixed light k8 p1=0", light, 1, 8, dict(p1=0.0)), ("fp64 heavy", heavy, 0, 0, {}),
        ("fp64 light k8", light, 0, 8, {}), ("mixed light k8 v0=0.5 p0=0.5", light, 1, 8, dict(v0=0.5, p0=0.5)),
    ]
    m0 = _mode(mn, *light, dx)
    ctx = lib.Context(abi.ModelBuffers(prn, pinned=True), abi.make_params(m0), abi.make_file_params(m0.files[0]))
    runtime.prepare(ctx)
    ctx.download(abi.SYNC_ALL)
    s0 = {"pr": ctx.buf.pr.copy(), **{f: ctx.buf.f32[f].copy() for f in abi.NODE_F32}}
    out = []
    for name, (d, u), prec, kry, kw in variants:
        m = _mode(mn, d, u, dx, **kw)
        for k, v in s0.items():
            (ctx.buf.pr if k == "pr" else ctx.buf.f32[k])[:] = v
        ctx.upload(abi.SYNC_NODES)
        ctx.set_params(abi.make_params(m, stokes_rtol=1e-8, stokes_maxcyc=maxcyc, precision=prec, krylov=kry,
                                       warm_start=1))
        ctx.set_file_params(abi.make_file_params(m.files[0]))
        t = time.time()
        try:
            ctx.stokes(0, 1e9 * YEAR)
            conv = True
        except lib.I3gError as e:
            if "NOCONV" not in str(e):
                raise
            conv = False
        st = ctx.stats()
        line = {"variant": name, "converged": conv, "cycles": st["stokes_cycles"], "mom": st["stokes_mom_rel"],
                "cont": st["stokes_cont_rel"], "ms": st["ms_stokes"], "wall_s": round(time.time() - t, 2)}
        print(json.dumps(line), flush=True)
        out.append(line)
    ctx.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--model", default="subduction", choices=("subduction", "inclusions"))
    ap.add_argument("--dims", default="129,65,129", help="nodes x,y,z (y vertical)")
    ap.add_argument("--multinum", type=int, default=3)
    ap.add_argument("--maxcyc", type=int, default=600)
    a = ap.parse_args()
    run(a.model, tuple(int(x) for x in a.dims.split(",")), a.multinum, a.maxcyc)


if __name__ == "__main__":
    main()
