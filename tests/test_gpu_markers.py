"""CUDA marker kernels (RK4 advection, marker -> node), heat and post-Stokes stresses against the
oracle and the reference, on every reference-generated marker case."""
import numpy as np
import pytest

import cases
import oracle as O
from i3elvis_b200 import abi, lib, runtime
from test_oracle_markers import MARKER_CASES, check_markers_vs_reference, marker_setup

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("exact", [1, 0])
@pytest.mark.parametrize("name", MARKER_CASES)
def test_move_markers_matches_reference(name, exact):
    """Marker x, y, z, strain and type after the reference's RK4 step are bit-exact; the
    viscosity from viscalc (Newtonian, Arrhenius, Drucker-Prager) within 2e-7.  Both
    arithmetic variants: the reference's operation order (exact = 1) and the fast one, whose
    FP64 interpolations differ in the last bits and whose FP32 positions are still expected to
    round to the same values."""
    p, mode, fx, buf = marker_setup(name)
    dt = float(fx["fld_dt"][0])
    g = lib.Context(buf, abi.make_params(mode, marker_exact=exact), abi.make_file_params(mode.files[0]))
    g.move_markers(dt)
    g.download(abi.SYNC_MARKERS)
    check_markers_vs_reference(fx, buf, name)
    if name == "dp17":
        assert int((buf.f32["marke"] > 0).sum()) == fx["meta"]["csr_sha256"]["yielding_markers"] > 0


@pytest.mark.parametrize("exact", [1, 0])
@pytest.mark.parametrize("name", MARKER_CASES)
def test_markers_to_nodes_matches_oracle_and_reference(name, exact):
    p, mode, fx, buf = marker_setup(name)
    dt = float(fx["fld_dt"][0])
    g = lib.Context(buf, abi.make_params(mode, marker_exact=exact), abi.make_file_params(mode.files[0]))
    g.move_markers(dt)
    g.markers_to_nodes(dt)
    g.download(abi.SYNC_ALL)
    p2, mode2, fx2, buf2 = marker_setup(name)
    o = O.Oracle(buf2, abi.make_params(mode2), abi.make_file_params(mode2.files[0]))
    o.call("orc_move_markers", dt)
    o.call("orc_markers_to_nodes", dt)
    o.download(abi.SYNC_ALL)
    ref = dict(zip(O.NODE_NAMES, fx["r2n"]))
    for f in ("ro", "nu", "nxx", "nxy", "nxz", "nyz", "tk", "cp", "kt", "et", "ht", "rr"):
        # FP64 sums in a different order than the oracle: equal up to the final FP32 rounding
        np.testing.assert_allclose(buf.f32[f], buf2.f32[f], rtol=3e-7, atol=0, err_msg=f"{name} {f}")
        np.testing.assert_allclose(buf.f32[f], ref[f], rtol=2e-6, atol=0, err_msg=f"{name} {f}")
    # downloads return markers in the original order
    np.testing.assert_array_equal(buf.f32["markx"], buf2.f32["markx"])


@pytest.mark.parametrize("name", MARKER_CASES)
def test_prepare_matches_reference(name):
    """Node fields after the initial marker -> node passes (in3mg.c:990-1031)."""
    from i3elvis_b200 import prn as P
    p, mode = cases.build(name)
    fx = dict(np.load(cases.os.path.join(cases.HERE, f"{name}.npz")))
    buf = abi.ModelBuffers(p)
    g = lib.Context(buf, abi.make_params(mode), abi.make_file_params(mode.files[0]))
    runtime.prepare(g)
    ref = dict(zip(P.NODE_FIELDS, fx["nodes"]))
    for f in ("ro", "nu", "nxx", "nxy", "nxz", "nyz", "tk", "cp", "kt"):
        np.testing.assert_allclose(buf.f32[f], ref[f], rtol=2e-6, atol=0, err_msg=f"{name} {f}")
    np.testing.assert_allclose(buf.pr, ref["pr"].astype(np.float64), rtol=1e-6, atol=1e-3)
    np.testing.assert_allclose(buf.f32["markv"], fx["markv"], rtol=2e-7)


@pytest.mark.parametrize("exact", [1, 0])
@pytest.mark.parametrize("name", MARKER_CASES)
def test_heat_matches_reference_and_oracle(name, exact):
    """titerate on the GPU: converged FP64 temperature equals the reference's heat rows solved
    to 1e-13; marker temperatures match the oracle's restatement and the reference's run."""
    p, mode, fx, buf = marker_setup(name)
    dt = float(fx["fld_dt"][0])
    g = lib.Context(buf, abi.make_params(mode, heat_rtol=1e-13, marker_exact=exact), abi.make_file_params(mode.files[0]))
    assert g.heat(0, dt) == dt
    T = g.get(abi.A_TK, 0, p.nodenum)
    ref = fx["heat_sol"]
    assert np.linalg.norm(T - ref) / np.linalg.norm(ref) < 1e-12
    g.download(abi.SYNC_ALL)
    p2, mode2, fx2, buf2 = marker_setup(name)
    o = O.Oracle(buf2, abi.make_params(mode2, heat_rtol=1e-13), abi.make_file_params(mode2.files[0]))
    o.call("orc_heat", (O.C.c_double * 1)(dt))
    o.download(abi.SYNC_ALL)
    np.testing.assert_allclose(buf.f32["tk"], buf2.f32["tk"], rtol=2e-7, atol=0)
    np.testing.assert_allclose(buf.f32["markk"], buf2.f32["markk"], rtol=1e-6, atol=1e-4)
    stride = fx["meta"].get("stride", 1)
    mk_ref = fx["heat_mk"] if "heat_mk" in fx else fx["heat_mk_sub"]
    np.testing.assert_allclose(buf.f32["markk"][::stride], mk_ref, rtol=1e-5, atol=1e-3)
    st = g.stats()
    assert st["heat_rel"] <= 1e-13 and st["heat_substeps"] >= 1


@pytest.mark.parametrize("name", MARKER_CASES)
def test_stresses_match_reference(name):
    """Strain rates and stresses from the reference's final velocities (sxxcalc..syzcalc with
    ynval = 0, recomputed by vpiterate after its iterations) equal the reference's exx..syz."""
    p, mode, fx, buf = marker_setup(name)
    g = lib.Context(buf, abi.make_params(mode), abi.make_file_params(mode.files[0]))
    for f in O.FIELD_NAMES[3:]:
        buf.f32[f][:] = 0.0
    g.call("i3g_stokes_stresses")
    g.download(abi.SYNC_STRESS)
    for i, f in enumerate(O.FIELD_NAMES[3:]):
        ref = fx["fld"][3 + i]
        got = buf.f32[f]
        scale = float(np.abs(ref).max()) or 1.0
        nbad = int(np.count_nonzero(got != ref))
        err = float(np.abs(got.astype(np.float64) - ref).max()) / scale
        print(name, f, "differing entries", nbad, "max |diff| / max |ref|", err)
        assert err <= 1e-6, (name, f, nbad, err)


def test_async_marker_upload_gives_the_same_step():
    """An upload whose marker copies overlap the Stokes solve (I3G_SYNC_ASYNC) leaves the time
    step bit-identical to a synchronous upload of the same host state."""
    out = []
    for mask in (abi.SYNC_NODES | abi.SYNC_MARKERS, abi.SYNC_NODES | abi.SYNC_MARKERS | abi.SYNC_ASYNC):
        p, mode, fx, buf = marker_setup("sphere13")
        g = lib.Context(buf, abi.make_params(mode, stokes_rtol=1e-10), abi.make_file_params(mode.files[0]))
        runtime.time_step(g, mode, mode.files[0], 0)   # device state moves away from the host's
        g.upload(mask)
        runtime.time_step(g, mode, mode.files[0], 1)
        g.download(abi.SYNC_ALL)
        out.append({f: buf.f32[f].copy() for f in ("markx", "marky", "markk", "markv", "tk", "vx", "nu")})
        g.close()
    for f in out[0]:
        np.testing.assert_array_equal(out[0][f], out[1][f], err_msg=f)


def test_round_trip_upload_keeps_the_extrapolated_start():
    """A host loop that downloads the state after every step and uploads it again (the
    reference's own loop around the library) keeps the extrapolated start of a device-resident
    run: the history survives an upload of exactly the last solution.  Changing one velocity
    before an upload drops it, and that step starts from the uploaded state."""
    runs = []
    for mode_ in ("resident", "round trip", "edited"):
        p, mode, fx, buf = marker_setup("sphere13")
        g = lib.Context(buf, abi.make_params(mode, stokes_rtol=1e-10, precision=1, krylov=8, warm_start=2),
                        abi.make_file_params(mode.files[0]))
        starts, cycles = [], []
        for step in range(4):
            if mode_ != "resident" and step > 0:
                g.download(abi.SYNC_ALL)
                if mode_ == "edited" and step == 3:
                    buf.f32["vx"][p.nodenum // 2] *= 1.0 + 1e-3
                g.upload(abi.SYNC_ALL)
            runtime.time_step(g, mode, mode.files[0], step)
            st = g.stats()
            starts.append(st["stokes_start"])
            cycles.append(st["stokes_cycles"])
        g.download(abi.SYNC_ALL)
        runs.append((starts, cycles, {f: buf.f32[f].copy() for f in ("markx", "markk", "tk", "vx", "nu")}, buf.pr.copy()))
        g.close()
    (s0, c0, f0, p0), (s1, c1, f1, p1), (s2, c2, f2, p2) = runs
    assert s0 == [0, 0, 1, 1], s0
    assert s1 == s0, s1
    assert s2 == [0, 0, 1, 0], s2
    # the same starts; the uploaded markers are re-sorted from the host's order, which may change
    # the order of the FP64 node sums within a cell (last bits), and with them a cycle count by one
    assert all(abs(a - b) <= 1 for a, b in zip(c0, c1)), (c0, c1)
    for f in f0:
        np.testing.assert_allclose(f1[f], f0[f], rtol=1e-6, atol=0, err_msg=f)
    np.testing.assert_allclose(p1, p0, rtol=1e-9, atol=1e-3)
