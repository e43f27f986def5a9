"""The CPU oracle against the reference's own outputs (golden fixtures)."""
import hashlib

import numpy as np

import pytest

import cases
import oracle as O
from conftest import golden
from i3elvis_b200 import abi


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _oracle(p, mode):
    return O.Oracle(abi.ModelBuffers(p), abi.make_params(mode), abi.make_file_params(mode.files[0]))


def test_assembled_rows_bit_exact(golden_case):
    """Rows of every level equal the reference's row store bit for bit (gausmat2 layout)."""
    name, p, mode, fx = golden_case
    o = _oracle(p, mode)
    o.call("orc_stokes_setup")
    sizes = cases.level_sizes(p, mode.multinum)
    for l, n in enumerate(sizes):
        cnt, cols, vals = o.csr(l, 4 * n)
        d = fx["meta"]["csr_sha256"][f"L{l}"]
        assert _sha(cnt) == d["counts"] and _sha(cols) == d["cols"] and _sha(vals) == d["vals"], f"level {l}"
    assert _sha(o.get(abi.A_RHS, 0, 4 * sizes[0])) == fx["meta"]["csr_sha256"]["rhs0"]


def test_assembled_rows_bit_exact_33():
    """The same on the 33^3 sinking sphere of the benchmark's CPU-runnable configuration."""
    test_assembled_rows_bit_exact(("sphere33",) + golden("sphere33"))


def test_vcycles_bit_exact(golden_case):
    """Five V-cycles in the reference's lexicographic order reproduce the reference's
    iterate on every level bit for bit."""
    name, p, mode, fx = golden_case
    o = _oracle(p, mode)
    o.call("orc_stokes_setup")
    o.call("orc_stokes_vcycles", 5)
    sizes = cases.level_sizes(p, mode.multinum)
    off = 0
    for l, n in enumerate(sizes):
        got = o.get(abi.A_SOL, l, 4 * n)
        if "vcyc_sol" in fx:
            assert np.array_equal(got, fx["vcyc_sol"][off:off + 4 * n]), f"level {l}"
        else:
            assert _sha(got) == fx["meta"]["csr_sha256"][f"vcyc_L{l}"], f"level {l}"
        off += 4 * n
    mom, cont = o.relres()
    assert np.isclose(mom, fx["vcyc_hist"][-2], rtol=1e-12) and np.isclose(cont, fx["vcyc_hist"][-1], rtol=1e-12)


def test_vcycles_bit_exact_33():
    test_vcycles_bit_exact(("sphere33",) + golden("sphere33"))


def test_multicolour_converges_to_reference_solution(golden_case):
    """The multicolour ordering (the CUDA library's) converges to the reference's solution of
    the same discrete system: relative L2 <= 1e-8 for velocity and pressure."""
    name, p, mode, fx = golden_case
    o = _oracle(p, mode)
    o.call("orc_stokes_setup")
    for _ in range(400):
        o.call("orc_stokes_vcycles_mc", 5)
        mom, cont = o.relres()
        if mom < 1e-12 and cont < 1e-12:
            break
    n0 = cases.level_sizes(p, mode.multinum)[0]
    got = o.get(abi.A_SOL, 0, 4 * n0).reshape(-1, 4)
    ref = fx["solve_sol"].reshape(-1, 4)
    pin = (p.head["pzinit"] * p.shape[0] + p.head["pxinit"]) * p.shape[1] + p.head["pyinit"]
    for k in range(1, 4):
        err = np.linalg.norm(got[:, k] - ref[:, k]) / np.linalg.norm(ref[:, k])
        assert err < 1e-8, (k, err)
    x, y, z = p.shape
    kk, ii, jj = np.meshgrid(np.arange(z), np.arange(x), np.arange(y), indexing="ij")
    has_p = ((ii > 0) & (jj > 0) & (kk > 0)).reshape(-1)
    gp = (got[:, 0] - got[pin, 0])[has_p]
    rp = (ref[:, 0] - ref[pin, 0])[has_p]
    assert np.linalg.norm(gp - rp) / np.linalg.norm(rp) < 1e-8
