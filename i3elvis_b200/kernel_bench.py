"""Kernel micro-benchmark: one model, one kernel class, a few launches.

    python -m i3elvis_b200.kernel_bench --n 129 --mnum 1 --kind 0 --reps 3

Builds the inclusion model (``model.random_inclusions``) at the given size, prepares it on the
GPU and times ``reps`` launches of one kernel class through ``i3g_time_kernel`` (0 FP64
smoother colour, 7 FP32 smoother colour, 1 residual, 2 restriction, 3 prolongation,
4 marker->node tile pass, 5 RK4 advection, 6 heat smoother colour, 9 marker temperature update);
``--exact 1`` runs the marker kernels in the reference's operation order.  Prints one JSON line.
Used as the small, self-contained command under ``ncu``.
"""
from __future__ import annotations

import argparse
import json

from . import abi, config, lib, model, runtime


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=129)
    ap.add_argument("--mnum", type=int, default=1)
    ap.add_argument("--multinum", type=int, default=4)
    ap.add_argument("--kind", type=int, default=0)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--exact", type=int, default=0, help="marker kernels in the reference's operation order (1)")
    a = ap.parse_args()
    prn, spec = model.random_inclusions(n=a.n, mnum=a.mnum, multinum=a.multinum)
    mode = config.Mode(multinum=a.multinum, multinnn=((8,) * a.multinum + (0,), (8,) * a.multinum + (64,)),
                       nubeg=1e18, nuend=1e24, files=[config.OutFile("o.prn", maxxystep=1e3, multinum=a.multinum)])
    ctx = lib.Context(abi.ModelBuffers(prn), abi.make_params(mode, marker_exact=a.exact), abi.make_file_params(mode.files[0]))
    runtime.prepare(ctx)
    ctx.call("i3g_stokes_setup")
    if a.kind == 6:
        ctx.heat(0, 1e13)
    ms, by = ctx.time_kernel(a.kind, a.reps)
    print(json.dumps({"kind": a.kind, "exact": a.exact, "n": a.n, "markers": prn.marknum, "ms_per_launch": ms,
                      "bytes_per_launch": by, "GBps": by / ms / 1e6}))


if __name__ == "__main__":
    main()
