"""The allocation-free stopping test against the context's own (i3g_stokes_relres).

i3g_stokes_relres_noalloc is for host codes that cannot allocate device memory once they
are running (their pool allocator owns the GPU, or an allocation would synchronise work they
have queued).  It reads a level-0 system from caller-owned device buffers and keeps its
partial sums in a static device array.  Its two numbers must equal those of
i3g_stokes_relres on the same solution up to summation order (rtol 1e-12), on two
consecutive calls that reuse the array.
"""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import golden

RTOL = 1e-12


def _fn():
    from i3elvis_b200 import lib
    L = C.CDLL(lib.LIBPATH)
    f = L.i3g_stokes_relres_noalloc
    P4 = C.c_void_p * 4
    f.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p, P4, P4, P4, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    L.i3g_last_error.argtypes = [C.c_void_p]
    L.i3g_last_error.restype = C.c_char_p
    return L, f, P4


def _mean_spacing(p):
    h = p.head
    nx, ny, nz = p.shape
    return (float(h["xsize"]) / (nx - 1) + float(h["ysize"]) / (ny - 1) + float(h["zsize"]) / (nz - 1)) / 3.0


def _bc_bits(p, n0):
    """Byte per node with bit v set when row v of the node is a boundary row (level 0)."""
    rows = p.bond["row"].astype(np.int64)
    rows = rows[rows < 4 * n0]
    bits = np.zeros(n0, np.uint8)
    np.bitwise_or.at(bits, rows // 4, (1 << (rows % 4)).astype(np.uint8))
    return bits


def test_rejects_grid_beyond_static_scratch():
    """The size check comes before any CUDA call, so this runs without a GPU."""
    from i3elvis_b200 import lib
    if not os.path.exists(lib.LIBPATH):
        pytest.skip("libi3g.so not built")
    L, f, P4 = _fn()
    z = P4(1, 1, 1, 1)
    rc = f(257, 17, 257, 1.0, 1, z, z, z, 1, None)
    assert rc == -1
    assert b"65536" in L.i3g_last_error(None)


@pytest.mark.gpu
def test_noalloc_relres_matches_context():
    import torch
    from i3elvis_b200 import abi, lib
    p, mode, _ = golden("sphere17")
    g = lib.Context(abi.ModelBuffers(p), abi.make_params(mode), abi.make_file_params(mode.files[0]))
    g.call("i3g_stokes_setup")
    L, f, P4 = _fn()
    nx, ny, nz = p.shape
    n0 = nx * ny * nz
    h = _mean_spacing(p)
    dev = torch.device("cuda", 0)
    bc = torch.from_numpy(_bc_bits(p, n0)).to(dev)
    out = torch.full((2,), -1.0, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    for ncyc in (1, 2):                       # two calls in a row on different iterates
        g.call("i3g_stokes_vcycles", ncyc)
        want = g.relres()
        g.call("i3g_stokes_residual", 0)
        comp = {}
        for name, which in (("res", abi.A_RES), ("rhs", abi.A_RHS), ("sol", abi.A_SOL)):
            a = g.get(which, 0, 4 * n0).reshape(n0, 4)
            comp[name] = [torch.from_numpy(np.ascontiguousarray(a[:, v])).to(dev) for v in range(4)]
        torch.cuda.synchronize(dev)
        ptr = {k: P4(*[t.data_ptr() for t in v]) for k, v in comp.items()}
        rc = f(nx, ny, nz, h, bc.data_ptr(), ptr["res"], ptr["rhs"], ptr["sol"], out.data_ptr(), stream.cuda_stream)
        assert rc == 0, L.i3g_last_error(None)
        stream.synchronize()
        got = out.cpu().numpy()
        assert want[0] > 0 and want[1] > 0
        np.testing.assert_allclose(got, np.array(want), rtol=RTOL)
