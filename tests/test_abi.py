"""The C-ABI libraries load and export every entry point include/i3g.h declares (no GPU needed)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "i3g.h")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(i3g_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_time_step_calls():
    names = declared()
    for n in ("i3g_create", "i3g_stokes", "i3g_heat", "i3g_move_markers", "i3g_markers_to_nodes",
              "i3g_download", "i3g_upload", "i3g_destroy"):
        assert n in names


def test_libi3g_exports_every_declared_symbol():
    from i3elvis_b200 import lib
    if not os.path.exists(lib.LIBPATH):
        from i3elvis_b200 import build
        build.build()
    L = ctypes.CDLL(lib.LIBPATH)
    missing = [n for n in declared() if not hasattr(L, n)]
    assert not missing, missing


def test_create_without_gpu_fails_cleanly():
    """Without a visible GPU the library reports an error instead of falling back."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    from i3elvis_b200 import abi, config, lib, model
    p, _ = model.sinking_sphere(n=9, mnum=1, multinum=1, seed=2)
    with pytest.raises(lib.I3gError):
        lib.Context(abi.ModelBuffers(p), abi.make_params(config.Mode(multinum=1, multinnn=((8, 0), (8, 16)))))
