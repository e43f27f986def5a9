"""Host time loop over the C ABI, mirroring the reference's ``i3mg.c`` main loop.

``run(workdir)`` reads ``file.t3c`` / ``mode.t3c`` and the input ``.prn`` like ``loadconf`` +
``loader`` (``load3mg.c:2-892``), then for each output file applies its parameter row
(``i3mg.c:64-77``) and runs ``cyc0max`` time steps of Stokes -> heat -> markers -> marker
to node (``i3mg.c:80-147``) on the GPU, and writes the ``.prn`` (``saver``) and ``file.t3c``.
The same loop is available in C as ``host/i3g``.
"""
from __future__ import annotations

import os
import time

import numpy as np

from . import abi, config, lib
from .prn import YEAR, read_prn, write_prn


def hydrostatic_pressure(buf: abi.ModelBuffers) -> None:
    """Initial pressure column integration of ``in3mg.c:1010-1021``."""
    h = buf.prn.head
    nx, ny, nz = int(h["xnumx"]), int(h["ynumy"]), int(h["znumz"])
    g = float(h["gykoef"])
    if g <= 0:
        return
    gy = buf.gy.astype(np.float64)
    ro = buf.f32["ro"].reshape(nz, nx, ny)
    pr = buf.pr.reshape(nz, nx, ny)
    # mean density of the 4 nodes around each vertical cell edge, FP32 sum as in C
    rs = ((ro[1:, 1:, 1:-1] + ro[1:, :-1, 1:-1]) + ro[:-1, 1:, 1:-1]) + ro[:-1, :-1, 1:-1]
    inc = (gy[2:] - gy[:-2])[None, None, :] / 2.0 * g * (rs.astype(np.float64) / 4.0)
    pr[1:, 1:, 1] = float(h["pinit"])
    pr[1:, 1:, 2:] = float(h["pinit"]) + np.cumsum(inc, axis=2)


def prepare(ctx: lib.Context) -> None:
    """Node fields from markers, hydrostatic pressure, node fields again (``in3mg.c:990-1031``),
    on the device (``i3g_prepare``); the host buffers receive the result."""
    ctx.prepare()
    ctx.download(abi.SYNC_ALL)


def time_step(ctx: lib.Context, mode: config.Mode, f: config.OutFile, n0: int, allow_noconv: bool = False) -> dict:
    """One reference time step (``i3mg.c:80-147``); returns the step size and phase times.
    ``allow_noconv``: a Stokes solve that stops at its cycle cap does not end the step."""
    timestep = f.maxtmstep_yr * YEAR
    t = {}
    if mode.movemod:
        t0 = time.perf_counter()
        timestep = ctx.stokes(n0, timestep, allow_noconv)
        t["stokes_s"] = time.perf_counter() - t0
    if mode.tempmod and timestep:
        t0 = time.perf_counter()
        ctx.heat(n0, timestep)
        t["heat_s"] = time.perf_counter() - t0
    if mode.markmod and timestep:
        t0 = time.perf_counter()
        ctx.move_markers(timestep)
        t["move_s"] = time.perf_counter() - t0
    if mode.gridmod:
        t0 = time.perf_counter()
        ctx.markers_to_nodes(timestep)
        t["r2n_s"] = time.perf_counter() - t0
    ctx.add_time(timestep)
    t["timestep"] = timestep
    return t


def run(workdir: str, max_files: int | None = None, **solver) -> list:
    """The ``i3mg`` program over the GPU library, run inside ``workdir``."""
    with open(os.path.join(workdir, "file.t3c")) as fh:
        fln3 = config.c_atoi(fh.read().split()[0]) - 1
    mode = config.read_mode(os.path.join(workdir, "mode.t3c"))
    infile = mode.infile
    if 0 <= fln3 < len(mode.files):
        infile = mode.files[fln3].name
    else:
        fln3 = -1
    prn = read_prn(os.path.join(workdir, infile))
    buf = abi.ModelBuffers(prn)
    ctx = lib.Context(buf, abi.make_params(mode, **solver))
    if mode.cyc1max < 0:
        # reset v, P, strain rates and stresses, then nodes from markers (i3mg.c:40-52)
        buf.pr[:] = 0.0
        for f in ("vx", "vy", "vz") + abi.STRESS_F32:
            buf.f32[f][:] = 0.0
        ctx.upload(abi.SYNC_NODES | abi.SYNC_STRESS)
        ctx.markers_to_nodes(0.0)
    log = []
    first = fln3 + 1
    last = min(first + mode.filesjob, len(mode.files))
    if max_files is not None:
        last = min(last, first + max_files)
    for f0 in range(first, last):
        f = mode.files[f0]
        ctx.set_file_params(abi.make_file_params(f))
        for n0 in range(f.cyc0max):
            log.append(time_step(ctx, mode, f, n0))
        ctx.download(abi.SYNC_ALL)
        out = buf.to_prn()
        out.head["cycle"] = f.cyc0max - 1
        write_prn(os.path.join(workdir, f.name), out)
        config.write_file_t3c(os.path.join(workdir, "file.t3c"), f0 + 1)
    ctx.close()
    return log
