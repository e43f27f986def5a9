"""CUDA marker kernels (RK4 advection, marker -> node) against the oracle and the reference."""
import numpy as np
import pytest

import oracle as O
from conftest import golden
from i3elvis_b200 import abi, lib, runtime
from test_oracle_markers import marker_setup

pytestmark = pytest.mark.gpu


def test_move_markers_matches_reference():
    p, mode, fx, buf = marker_setup()
    dt = float(fx["fld_dt"][0])
    g = lib.Context(buf, abi.make_params(mode), abi.make_file_params(mode.files[0]))
    g.move_markers(dt)
    g.download(abi.SYNC_MARKERS)
    ref = dict(zip(O.MARK_NAMES, fx["mk"]))
    for f, bf in (("x", "markx"), ("y", "marky"), ("z", "markz")):
        np.testing.assert_array_equal(buf.f32[bf], ref[f], err_msg=f)
    np.testing.assert_allclose(buf.f32["markv"], ref["v"], rtol=2e-7)
    np.testing.assert_array_equal(buf.f32["marke"], ref["e"])
    np.testing.assert_array_equal(buf.markt, fx["mk_t"])


def test_markers_to_nodes_matches_oracle_and_reference():
    p, mode, fx, buf = marker_setup()
    dt = float(fx["fld_dt"][0])
    g = lib.Context(buf, abi.make_params(mode), abi.make_file_params(mode.files[0]))
    g.move_markers(dt)
    g.markers_to_nodes(dt)
    g.download(abi.SYNC_ALL)
    p2, mode2, fx2, buf2 = marker_setup()
    o = O.Oracle(buf2, abi.make_params(mode2), abi.make_file_params(mode2.files[0]))
    o.call("orc_move_markers", dt)
    o.call("orc_markers_to_nodes", dt)
    o.download(abi.SYNC_ALL)
    ref = dict(zip(O.NODE_NAMES, fx["r2n"]))
    for f in ("ro", "nu", "nxx", "nxy", "nxz", "nyz", "tk", "cp", "kt", "et", "ht", "rr"):
        # FP64 sums in a different order than the oracle: equal up to the final FP32 rounding
        np.testing.assert_allclose(buf.f32[f], buf2.f32[f], rtol=3e-7, atol=0, err_msg=f)
        np.testing.assert_allclose(buf.f32[f], ref[f], rtol=2e-6, atol=0, err_msg=f)
    # downloads return markers in the original order
    np.testing.assert_array_equal(buf.f32["markx"], buf2.f32["markx"])


def test_prepare_matches_reference():
    """Node fields after the initial marker -> node passes (in3mg.c:990-1031)."""
    import cases
    from i3elvis_b200 import prn as P
    p, mode = cases.build("sphere13")
    fx = dict(np.load(cases.os.path.join(cases.HERE, "sphere13.npz")))
    buf = abi.ModelBuffers(p)
    g = lib.Context(buf, abi.make_params(mode), abi.make_file_params(mode.files[0]))
    runtime.prepare(g)
    ref = dict(zip(P.NODE_FIELDS, fx["nodes"]))
    for f in ("ro", "nu", "nxx", "nxy", "nxz", "nyz", "tk", "cp", "kt"):
        np.testing.assert_allclose(buf.f32[f], ref[f], rtol=2e-6, atol=0, err_msg=f)
    np.testing.assert_allclose(buf.pr, ref["pr"].astype(np.float64), rtol=1e-6, atol=1e-3)
    np.testing.assert_allclose(buf.f32["markv"], fx["markv"], rtol=2e-7)


def test_heat_matches_reference_and_oracle():
    """titerate on the GPU: converged FP64 temperature equals the reference's heat rows solved
    to 1e-13; marker temperatures match the oracle's restatement and the reference's run."""
    p, mode, fx, buf = marker_setup()
    dt = float(fx["fld_dt"][0])
    g = lib.Context(buf, abi.make_params(mode, heat_rtol=1e-13), abi.make_file_params(mode.files[0]))
    assert g.heat(0, dt) == dt
    T = g.get(abi.A_TK, 0, p.nodenum)
    ref = fx["heat_sol"]
    assert np.linalg.norm(T - ref) / np.linalg.norm(ref) < 1e-12
    g.download(abi.SYNC_ALL)
    p2, mode2, fx2, buf2 = marker_setup()
    o = O.Oracle(buf2, abi.make_params(mode2, heat_rtol=1e-13), abi.make_file_params(mode2.files[0]))
    o.call("orc_heat", (O.C.c_double * 1)(dt))
    o.download(abi.SYNC_ALL)
    np.testing.assert_allclose(buf.f32["tk"], buf2.f32["tk"], rtol=2e-7, atol=0)
    np.testing.assert_allclose(buf.f32["markk"], buf2.f32["markk"], rtol=1e-6, atol=1e-4)
    np.testing.assert_allclose(buf.f32["markk"], fx["heat_mk"], rtol=1e-5, atol=1e-3)
    st = g.stats()
    assert st["heat_rel"] <= 1e-13 and st["heat_substeps"] == 1
