"""CUDA Stokes multigrid against the CPU oracle (bit for bit) and the reference (converged)."""
import numpy as np
import pytest

import cases
import oracle as O
from conftest import ALL_CASES, golden
from i3elvis_b200 import abi, lib

pytestmark = pytest.mark.gpu


def pair(name, **solver):
    p, mode, fx = golden(name)
    par = abi.make_params(mode, **solver)
    fp = abi.make_file_params(mode.files[0])
    g = lib.Context(abi.ModelBuffers(p), par, fp)
    o = O.Oracle(abi.ModelBuffers(p), par, fp)
    return p, mode, fx, g, o


def bc_rows(p, mode, level):
    """Boolean mask [4*N_l] of boundary rows on one level."""
    sizes = cases.level_sizes(p, mode.multinum)
    off = int(np.sum(sizes[:level])) * 4
    rows = p.bond["row"]
    rows = rows[(rows >= off) & (rows < off + 4 * sizes[level])] - off
    m = np.zeros(4 * sizes[level], bool)
    m[rows] = True
    return m


@pytest.mark.parametrize("name", ALL_CASES)
def test_setup_bit_exact(name):
    p, mode, fx, g, o = pair(name)
    g.call("i3g_stokes_setup")
    o.call("orc_stokes_setup")
    for l, n in enumerate(cases.level_sizes(p, mode.multinum)):
        assert np.array_equal(g.get(abi.A_NU, l, n, np.float32), o.get(abi.A_NU, l, n, np.float32)), l
        assert np.array_equal(g.get(abi.A_ETA, l, 4 * n), o.get(abi.A_ETA, l, 4 * n)), l
    n0 = cases.level_sizes(p, mode.multinum)[0]
    assert np.array_equal(g.get(abi.A_RHS, 0, 4 * n0), o.get(abi.A_RHS, 0, 4 * n0))
    assert np.array_equal(g.get(abi.A_SOL, 0, 4 * n0), o.get(abi.A_SOL, 0, 4 * n0))


@pytest.mark.parametrize("name", ALL_CASES)
def test_residual_smooth_transfer_bit_exact(name):
    p, mode, fx, g, o = pair(name)
    g.call("i3g_stokes_setup")
    o.call("orc_stokes_setup")
    rng = np.random.default_rng(11)
    sizes = cases.level_sizes(p, mode.multinum)
    for l, n in enumerate(sizes):
        x = rng.standard_normal(4 * n) * 1e-9
        x[0::4] *= 1e9
        g.set(abi.A_SOL, l, x); o.set(abi.A_SOL, l, x)
        if l > 0:
            f = rng.standard_normal(4 * n) * 1e4
            f[bc_rows(p, mode, l)] = 0.0
            g.set(abi.A_RHS, l, f); o.set(abi.A_RHS, l, f)
        g.call("i3g_stokes_residual", l); o.call("orc_stokes_residual", l)
        assert np.array_equal(g.get(abi.A_RES, l, 4 * n), o.get(abi.A_RES, l, 4 * n)), ("residual", l)
        g.call("i3g_stokes_smooth", l, 3); o.call("orc_stokes_smooth", l, 3)
        assert np.array_equal(g.get(abi.A_SOL, l, 4 * n), o.get(abi.A_SOL, l, 4 * n)), ("smooth", l)
        assert np.array_equal(g.get(abi.A_RES, l, 4 * n), o.get(abi.A_RES, l, 4 * n)), ("smooth res", l)
    for l in range(1, len(sizes)):
        g.call("i3g_stokes_restrict", l); o.call("orc_stokes_restrict", l)
        assert np.array_equal(g.get(abi.A_RHS, l, 4 * sizes[l]), o.get(abi.A_RHS, l, 4 * sizes[l])), ("restrict", l)
        xc = rng.standard_normal(4 * sizes[l])
        g.set(abi.A_SOL, l, xc); o.set(abi.A_SOL, l, xc)
        g.call("i3g_stokes_prolong", l); o.call("orc_stokes_prolong", l)
        assert np.array_equal(g.get(abi.A_SOL, l - 1, 4 * sizes[l - 1]), o.get(abi.A_SOL, l - 1, 4 * sizes[l - 1])), ("prolong", l)


@pytest.mark.parametrize("tail", ["12000", "2000", "0", "0-separate", "0-level0", "coop", "cluster"])
@pytest.mark.parametrize("name", ALL_CASES)
def test_vcycles_bit_exact(name, tail, monkeypatch):
    """V-cycles equal the oracle's bit for bit, with the small levels in the one-block tail
    kernel (default), with one kernel per phase on every level (I3G_TAIL_NODES=0), the same
    with separate boundary, residual and transfer launches (I3G_FUSE=0) and with in-kernel
    boundary rows on level 0 too (I3G_FUSE=3), with every coarse
    level in the cooperative grid-wide kernel (I3G_COOP_NODES), and with the tail on a 16-CTA
    thread-block cluster (I3G_TAIL_CLUSTER)."""
    if tail in ("0-separate", "0-level0"):
        monkeypatch.setenv("I3G_TAIL_NODES", "0")
        monkeypatch.setenv("I3G_FUSE", "0" if tail == "0-separate" else "3")
    elif tail == "coop":
        monkeypatch.setenv("I3G_COOP_NODES", "1000000")
    elif tail == "cluster":
        monkeypatch.setenv("I3G_TAIL_NODES", "12000")
        monkeypatch.setenv("I3G_TAIL_CLUSTER", "16")
    else:
        monkeypatch.setenv("I3G_TAIL_NODES", tail)
    p, mode, fx, g, o = pair(name)
    g.call("i3g_stokes_setup")
    o.call("orc_stokes_setup")
    g.call("i3g_stokes_vcycles", 3)
    o.call("orc_stokes_vcycles_mc", 3)
    for l, n in enumerate(cases.level_sizes(p, mode.multinum)):
        assert np.array_equal(g.get(abi.A_SOL, l, 4 * n), o.get(abi.A_SOL, l, 4 * n)), l
    gm, gc = g.relres()
    om, oc = o.relres()
    assert np.isclose(gm, om, rtol=1e-12) and np.isclose(gc, oc, rtol=1e-12)


def _compare_to_reference(p, sol, ref, tol):
    got = sol.reshape(-1, 4)
    ref = ref.reshape(-1, 4)
    x, y, z = p.shape
    kk, ii, jj = np.meshgrid(np.arange(z), np.arange(x), np.arange(y), indexing="ij")
    has_p = ((ii > 0) & (jj > 0) & (kk > 0)).reshape(-1)
    pin = (p.head["pzinit"] * x + p.head["pxinit"]) * y + p.head["pyinit"]
    errs = [np.linalg.norm(got[:, k] - ref[:, k]) / np.linalg.norm(ref[:, k]) for k in (1, 2, 3)]
    gp = (got[:, 0] - got[pin, 0])[has_p]
    rp = (ref[:, 0] - ref[pin, 0])[has_p]
    errs.append(np.linalg.norm(gp - rp) / np.linalg.norm(rp))
    assert max(errs) < tol, errs
    return errs


@pytest.mark.parametrize("precision,krylov", [(0, 0), (0, 8), (1, 0), (1, 8)])
@pytest.mark.parametrize("name", ALL_CASES)
def test_solve_matches_reference(name, precision, krylov):
    """Converged velocity and pressure equal the reference's converged FP64 solution to
    relative L2 1e-8 (FP64 multigrid, plain and as the FGMRES preconditioner; FP32 multigrid
    inside FP64 defect correction, plain and FGMRES-accelerated).  Cases: sinking spheres (13^3, 17^3, the 33^3 CPU-runnable benchmark
    configuration, whose own bar is 1e-6), Arrhenius inclusions, Drucker-Prager yielding and a
    non-uniform grid."""
    p, mode, fx = golden(name)
    par = abi.make_params(mode, stokes_rtol=1e-11, stokes_maxcyc=3000, precision=precision, krylov=krylov)
    g = lib.Context(abi.ModelBuffers(p), par, abi.make_file_params(mode.files[0]))
    dt = g.stokes(0, 1e30)
    st = g.stats()
    assert st["stokes_rel"] <= 1e-11
    n0 = cases.level_sizes(p, mode.multinum)[0]
    _compare_to_reference(p, g.get(abi.A_SOL, 0, 4 * n0), fx["solve_sol"], 1e-8)
    assert 0 < dt < 1e30


@pytest.mark.parametrize("warm", [2, 3])
def test_extrapolated_warm_start_reaches_same_solution(warm):
    """warm_start 2 and 3 (linear / quadratic extrapolation from the last two / three solutions)
    change only the start of the iteration: after four time steps the state equals the one of
    warm_start 1 to the solver tolerance, with no more V-cycles, and the start kinds follow the
    history (previous solution, then linear, then quadratic)."""
    from i3elvis_b200 import runtime
    sols, cyc, starts = [], [], []
    for w in (1, warm):
        p, mode, fx = golden("sphere17")
        par = abi.make_params(mode, stokes_rtol=1e-10, stokes_maxcyc=3000, precision=1, krylov=8, warm_start=w)
        g = lib.Context(abi.ModelBuffers(p), par, abi.make_file_params(mode.files[0]))
        f = mode.files[0]
        c, st = [], []
        for n0 in range(4):
            runtime.time_step(g, mode, f, n0)
            c.append(g.stats()["stokes_cycles"])
            st.append(g.stats()["stokes_start"])
        n0 = cases.level_sizes(p, mode.multinum)[0]
        sols.append(g.get(abi.A_SOL, 0, 4 * n0))
        cyc.append(c)
        starts.append(st)
        g.close()
    a, b = sols[0].reshape(-1, 4), sols[1].reshape(-1, 4)
    for k in (1, 2, 3):
        assert np.linalg.norm(a[:, k] - b[:, k]) <= 1e-6 * np.linalg.norm(a[:, k]), (k, cyc)
    assert cyc[1][3] <= cyc[0][3] + 2, cyc
    assert starts[0] == [0, 0, 0, 0], starts
    assert starts[1] == ([0, 0, 1, 1] if warm == 2 else [0, 0, 1, 3]), starts


def test_weak_layer_cells_converge_with_face_pressure_scale(monkeypatch):
    """Visco-plastic subduction model at 65 x 33 x 65 (weak layer of 1e19 Pa s inside a 1e24
    lithosphere): the FP32 preconditioner with the face rows' pressure scale for enclosed weak
    cells reaches relative residual 1e-8; with the cell viscosity as the scale (the reference's
    nd) the continuity residual of those cells stalls."""
    from i3elvis_b200 import config, model, runtime
    from i3elvis_b200.prn import YEAR
    prn, _ = model.subduction(nx=65, ny=33, nz=65, mnum=2, multinum=3, seed=11)
    dx = 1000e3 / 64
    mode = config.Mode(infile="in0.prn", multinum=3, multicyc=1, multinnn=((2, 4, 4, 0), (2, 4, 4, 4)),
                       p0koef=0.71, p1koef=1.0, v0koef=0.7, v1koef=0.7, nubeg=1e18, nuend=1e24,
                       files=[config.OutFile("out1.prn", maxxystep=0.5 * dx, maxtmstep_yr=1e9, nubeg=1e18,
                                             nuend=1e24, p0koef=0.71, p1koef=1.0, p0koef2=0.71, p1koef2=0.0,
                                             multinum=3, multinum2=3)])
    res = {}
    for scale in ("10", "0"):
        monkeypatch.setenv("I3G_ND_SCHUR", scale)
        par = abi.make_params(mode, stokes_rtol=1e-8, stokes_maxcyc=200, precision=1, krylov=8, warm_start=1)
        g = lib.Context(abi.ModelBuffers(prn), par, abi.make_file_params(mode.files[0]))
        runtime.prepare(g)
        try:
            g.stokes(0, 1e9 * YEAR)
            ok = True
        except lib.I3gError as e:
            assert abi.E_CODES.get(e.code) == "NOCONV", e
            ok = False
        res[scale] = (ok, g.stats())
        g.close()
    ok, st = res["10"]
    assert ok and st["stokes_rel"] <= 1e-8 and st["stokes_cycles"] < 200, st
    ok0, st0 = res["0"]
    assert not ok0 and st0["stokes_cont_rel"] > 1e-5, st0
