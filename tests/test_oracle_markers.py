"""The CPU oracle's marker operations against the reference (movemark + ronurecalc)."""
import hashlib

import numpy as np
import pytest

import cases
import oracle as O
from conftest import golden
from i3elvis_b200 import abi

MARKER_CASES = list(cases.MARKER_CASES)
SMALL_MARKER_CASES = [c for c in MARKER_CASES if not cases.CASES[c].get("big")]


def marker_setup(name="sphere13"):
    """Buffers holding the reference's post-Stokes fields (v, P, strain rates, stresses)."""
    p, mode, fx = golden(name)
    if "fld" not in fx:
        pytest.skip("no marker fixture for this case")
    buf = abi.ModelBuffers(p)
    buf.pr[:] = fx["fld_pr"]
    for i, f in enumerate(O.FIELD_NAMES):
        buf.f32[f][:] = fx["fld"][i]
    return p, mode, fx, buf


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def check_markers_vs_reference(fx, buf, name):
    """Marker positions, strain and type bit-exact, viscosity within 2e-7, against the
    reference's movemark (full arrays, or digests plus every stride-th marker for big cases)."""
    got = {"x": buf.f32["markx"], "y": buf.f32["marky"], "z": buf.f32["markz"], "e": buf.f32["marke"],
           "v": buf.f32["markv"], "t": buf.markt}
    if "mk" in fx:
        ref = dict(zip(O.MARK_NAMES, fx["mk"]))
        ref["t"] = fx["mk_t"]
        stride = 1
    else:
        stride = fx["meta"]["stride"]
        ref = dict(zip(O.MARK_NAMES, fx["mk_sub"]))
        ref["t"] = fx["mk_t_sub"]
        dig = fx["meta"]["csr_sha256"]["mk"]
    for f in ("x", "y", "z", "e", "t"):
        sub = got[f][::stride]
        nbad = int(np.count_nonzero(sub != ref[f]))
        assert nbad == 0, (name, f, nbad, "of", sub.size)
        if stride > 1:
            assert _sha(got[f]) == dig[f], (name, f, "digest of all markers differs")
    np.testing.assert_allclose(got["v"][::stride], ref["v"], rtol=2e-7, err_msg=name)


@pytest.mark.parametrize("name", MARKER_CASES)
def test_oracle_move_markers_matches_reference(name):
    p, mode, fx, buf = marker_setup(name)
    dt = float(fx["fld_dt"][0])
    o = O.Oracle(buf, abi.make_params(mode), abi.make_file_params(mode.files[0]))
    o.call("orc_move_markers", dt)
    o.download(abi.SYNC_MARKERS)
    check_markers_vs_reference(fx, buf, name)


@pytest.mark.parametrize("name", SMALL_MARKER_CASES)
def test_oracle_markers_to_nodes_matches_reference(name):
    p, mode, fx, buf = marker_setup(name)
    dt = float(fx["fld_dt"][0])
    o = O.Oracle(buf, abi.make_params(mode), abi.make_file_params(mode.files[0]))
    o.call("orc_move_markers", dt)
    o.call("orc_markers_to_nodes", dt)
    o.download(abi.SYNC_NODES)
    ref = dict(zip(O.NODE_NAMES, fx["r2n"]))
    # the reference sums most node fields in FP32 (in marker order); the oracle in FP64
    for f in ("ro", "nu", "nxx", "nxy", "nxz", "nyz", "tk", "cp", "kt", "et", "ht", "rr"):
        np.testing.assert_allclose(buf.f32[f], ref[f], rtol=2e-6, atol=0, err_msg=f"{name} {f}")


@pytest.mark.parametrize("name", SMALL_MARKER_CASES)
def test_oracle_heat_matches_reference(name):
    """titerate: converged FP64 temperature equals the reference's tightly solved heat rows;
    marker temperatures (subgrid diffusion) equal the reference's titerate to its tolerance."""
    p, mode, fx, buf = marker_setup(name)
    dt = float(fx["fld_dt"][0])
    o = O.Oracle(buf, abi.make_params(mode, heat_rtol=1e-13), abi.make_file_params(mode.files[0]))
    t = (O.C.c_double * 1)(dt)
    o.call("orc_heat", t)
    T = o.get(abi.A_TK, 0, p.nodenum)
    ref = fx["heat_sol"]
    assert np.linalg.norm(T - ref) / np.linalg.norm(ref) < 1e-12
    o.download(abi.SYNC_ALL)
    # the reference stops on HEATMIN = 1e-3 K evaluated on FP32 temperatures
    np.testing.assert_allclose(buf.f32["tk"], fx["heat_tk"], rtol=1e-5, atol=1e-3)
    np.testing.assert_allclose(buf.f32["markk"], fx["heat_mk"], rtol=1e-5, atol=1e-3)
