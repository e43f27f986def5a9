"""ctypes binding of ``libi3g.so`` (the C ABI in ``include/i3g.h``).

There is no CPU fallback: if the CUDA library is missing or no GPU is visible, the
constructor raises.  Every call goes through the extern "C" entry points.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libi3g.so")


class I3gError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"i3g error {abi.E_CODES.get(code, code)}: {msg}")
        self.code = code


_lib = None


def load():
    """Load ``libi3g.so``; raise if it is absent (build it with ``python -m i3elvis_b200.build``)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBPATH):
        raise I3gError(-2, f"{LIBPATH} not built; run python -m i3elvis_b200.build")
    L = C.CDLL(LIBPATH)
    P = C.c_void_p
    L.i3g_create.argtypes = [C.POINTER(abi.Model), C.POINTER(abi.Params), C.POINTER(P)]
    L.i3g_destroy.argtypes = [P]
    L.i3g_last_error.argtypes = [P]
    L.i3g_last_error.restype = C.c_char_p
    L.i3g_set_file_params.argtypes = [P, C.POINTER(abi.FileParams)]
    L.i3g_set_params.argtypes = [P, C.POINTER(abi.Params)]
    L.i3g_stokes.argtypes = [P, C.c_int, C.POINTER(C.c_double)]
    L.i3g_heat.argtypes = [P, C.c_int, C.POINTER(C.c_double)]
    L.i3g_move_markers.argtypes = [P, C.c_double]
    L.i3g_markers_to_nodes.argtypes = [P, C.c_double]
    L.i3g_add_time.argtypes = [P, C.c_double]
    L.i3g_download.argtypes = [P, C.POINTER(abi.Model), C.c_uint]
    L.i3g_upload.argtypes = [P, C.POINTER(abi.Model), C.c_uint]
    L.i3g_get_stats.argtypes = [P, C.POINTER(abi.Stats)]
    L.i3g_get_array.argtypes = [P, C.c_int, C.c_int, C.c_void_p, C.c_int64]
    L.i3g_set_array.argtypes = [P, C.c_int, C.c_int, C.c_void_p, C.c_int64]
    L.i3g_stokes_setup.argtypes = [P]
    L.i3g_stokes_stresses.argtypes = [P]
    L.i3g_write_vtr.argtypes = [P, C.c_char_p]
    L.i3g_init_markers.argtypes = [P, C.POINTER(abi.Init)]
    L.i3g_prepare.argtypes = [P]
    for name in ("i3g_stokes_residual", "i3g_stokes_restrict", "i3g_stokes_prolong", "i3g_stokes_vcycles"):
        getattr(L, name).argtypes = [P, C.c_int]
    L.i3g_stokes_smooth.argtypes = [P, C.c_int, C.c_int]
    L.i3g_stokes_relres.argtypes = [P, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.i3g_timer.argtypes = [P, C.c_int, C.POINTER(C.c_double)]
    L.i3g_time_kernel.argtypes = [P, C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    _lib = L
    return L


class Context:
    """One model resident on the current GPU (owns an ``i3g_ctx``)."""

    def __init__(self, buffers: abi.ModelBuffers, params: abi.Params, fparams: abi.FileParams = None):
        L = load()
        self.buf = buffers
        self.params = params
        self.h = C.c_void_p()
        rc = L.i3g_create(C.byref(buffers.model), C.byref(params), C.byref(self.h))
        if rc != 0:
            raise I3gError(rc, L.i3g_last_error(None).decode())
        if fparams is not None:
            self.set_file_params(fparams)

    def _check(self, rc):
        if rc != 0:
            raise I3gError(rc, load().i3g_last_error(self.h).decode())
        return rc

    def call(self, name, *args):
        return self._check(getattr(load(), name)(self.h, *args))

    def close(self):
        if getattr(self, "h", None):
            load().i3g_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_file_params(self, fp: abi.FileParams):
        self.call("i3g_set_file_params", C.byref(fp))

    def set_params(self, p: abi.Params):
        self.call("i3g_set_params", C.byref(p))

    # the four time-step calls of the host loop (i3mg.c:98-137)
    def stokes(self, n0: int, timestep: float, allow_noconv: bool = False) -> float:
        """``i3g_stokes``; with ``allow_noconv`` an iteration cap reached before the tolerance is
        not an error (the solution reached, its stresses and the CFL step are kept, as the
        library writes them before returning I3G_E_NOCONV)."""
        t = C.c_double(timestep)
        rc = load().i3g_stokes(self.h, n0, C.byref(t))
        if not (allow_noconv and rc == -5):
            self._check(rc)
        return t.value

    def heat(self, n0: int, timestep: float) -> float:
        t = C.c_double(timestep)
        self.call("i3g_heat", n0, C.byref(t))
        return t.value

    def move_markers(self, timestep: float):
        self.call("i3g_move_markers", timestep)

    def markers_to_nodes(self, timestep: float):
        self.call("i3g_markers_to_nodes", timestep)

    def add_time(self, timestep: float):
        self.call("i3g_add_time", timestep)

    def download(self, mask=abi.SYNC_ALL):
        self.call("i3g_download", C.byref(self.buf.model), mask)

    def upload(self, mask=abi.SYNC_ALL):
        self.call("i3g_upload", C.byref(self.buf.model), mask)

    def stats(self) -> dict:
        s = abi.Stats()
        self.call("i3g_get_stats", C.byref(s))
        return s.as_dict()

    def get(self, which, level, count, dtype=np.float64):
        out = np.zeros(count, dtype)
        self.call("i3g_get_array", which, level, out.ctypes.data, out.nbytes)
        return out

    def set(self, which, level, arr):
        arr = np.ascontiguousarray(arr)
        self.call("i3g_set_array", which, level, arr.ctypes.data, arr.nbytes)

    def relres(self):
        a, b = C.c_double(), C.c_double()
        self.call("i3g_stokes_relres", C.byref(a), C.byref(b))
        return a.value, b.value

    def init_markers(self, init: abi.Init, bodies=()):
        """Replace the markers by in3mg's initial markers (``i3g_init_markers``)."""
        arr = (abi.Body * max(len(bodies), 1))(*bodies)
        init.nbodies = len(bodies)
        init.bodies = C.cast(arr, C.POINTER(abi.Body))
        self.call("i3g_init_markers", C.byref(init))

    def prepare(self):
        """Initial-condition passes on the device (``i3g_prepare``, in3mg.c:990-1031)."""
        self.call("i3g_prepare")

    def write_vtr(self, path: str):
        """ParaView rectilinear-grid file of the nodal fields (``i3g_write_vtr``)."""
        self.call("i3g_write_vtr", os.fsencode(path))

    def timer_start(self):
        self.call("i3g_timer", 0, None)

    def timer_stop(self) -> float:
        ms = C.c_double()
        self.call("i3g_timer", 1, C.byref(ms))
        return ms.value

    def time_kernel(self, kind: int, reps: int):
        ms, by = C.c_double(), C.c_double()
        self.call("i3g_time_kernel", kind, reps, C.byref(ms), C.byref(by))
        return ms.value, by.value
