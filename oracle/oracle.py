"""TEST INFRASTRUCTURE: ctypes binding of the CPU oracle (``liborc.so``) and of the
reference harness binary (``_ref/ref_harness``).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use
this module, always as the checker and never as the thing measured or shipped.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess

import numpy as np

from i3elvis_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liborc.so")
REF = os.path.join(HERE, "_ref", "ref_harness")


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        P = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(abi.Model), C.POINTER(abi.Params), C.POINTER(P)]
        L.orc_destroy.argtypes = [P]
        L.orc_last_error.argtypes = [P]
        L.orc_last_error.restype = C.c_char_p
        L.orc_set_file_params.argtypes = [P, C.POINTER(abi.FileParams)]
        for name in ("orc_stokes_setup",):
            getattr(L, name).argtypes = [P]
        for name in ("orc_stokes_vcycles",):
            getattr(L, name).argtypes = [P, C.c_int]
        for name in ("orc_stokes_smooth", "orc_stokes_smooth_ref"):
            getattr(L, name).argtypes = [P, C.c_int, C.c_int]
        for name in ("orc_stokes_residual", "orc_stokes_restrict", "orc_stokes_prolong"):
            getattr(L, name).argtypes = [P, C.c_int]
        L.orc_stokes_vcycles_mc.argtypes = [P, C.c_int]
        L.orc_get_csr.argtypes = [P, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_stokes_relres.argtypes = [P, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_get_array.argtypes = [P, C.c_int, C.c_int, C.c_void_p, C.c_int64]
        L.orc_set_array.argtypes = [P, C.c_int, C.c_int, C.c_void_p, C.c_int64]
        L.orc_stokes.argtypes = [P, C.c_int, C.POINTER(C.c_double)]
        L.orc_get_stats.argtypes = [P, C.POINTER(abi.Stats)]
        L.orc_download.argtypes = [P, C.POINTER(abi.Model), C.c_uint]
        L.orc_upload.argtypes = [P, C.POINTER(abi.Model), C.c_uint]
        for name in ("orc_heat",):
            if hasattr(L, name):
                getattr(L, name).argtypes = [P, C.POINTER(C.c_double)]
        for name in ("orc_move_markers", "orc_markers_to_nodes"):
            if hasattr(L, name):
                getattr(L, name).argtypes = [P, C.c_double]
        _lib = L
    return _lib


class OracleError(RuntimeError):
    pass


class Oracle:
    """CPU restatement of the reference time step on one model (single-threaded)."""

    def __init__(self, buffers: abi.ModelBuffers, params: abi.Params, fparams: abi.FileParams = None):
        self.buf = buffers
        self.params = params
        self.h = C.c_void_p()
        self._check(lib().orc_create(C.byref(buffers.model), C.byref(params), C.byref(self.h)))
        if fparams is not None:
            self._check(lib().orc_set_file_params(self.h, C.byref(fparams)))

    def _check(self, rc):
        if rc != 0:
            msg = lib().orc_last_error(self.h).decode() if self.h else ""
            raise OracleError(f"oracle error {abi.E_CODES.get(rc, rc)}: {msg}")
        return rc

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = C.c_void_p()

    __del__ = close

    def call(self, name, *args):
        return self._check(getattr(lib(), name)(self.h, *args))

    def get(self, which, level, count, dtype=np.float64):
        out = np.zeros(count, dtype)
        self.call("orc_get_array", which, level, out.ctypes.data, out.nbytes)
        return out

    def set(self, which, level, arr):
        arr = np.ascontiguousarray(arr)
        self.call("orc_set_array", which, level, arr.ctypes.data, arr.nbytes)

    def csr(self, level, nrows):
        """Assembled rows of one level: (counts, cols, vals)."""
        cnt = np.zeros(nrows, np.int64)
        lib().orc_get_csr(self.h, level, cnt.ctypes.data, None, None)
        nnz = int(cnt.sum())
        cols = np.zeros(nnz, np.int64)
        vals = np.zeros(nnz, np.float64)
        lib().orc_get_csr(self.h, level, None, cols.ctypes.data, vals.ctypes.data)
        return cnt, cols, vals

    def relres(self):
        a, b = C.c_double(), C.c_double()
        self.call("orc_stokes_relres", C.byref(a), C.byref(b))
        return a.value, b.value

    def stats(self):
        s = abi.Stats()
        lib().orc_get_stats(self.h, C.byref(s))
        return s.as_dict()

    def download(self, mask=abi.SYNC_ALL):
        self.call("orc_download", C.byref(self.buf.model), mask)


# ---- reference harness ------------------------------------------------------------------
def have_reference():
    return os.path.exists(REF)


def run_reference(workdir, *args, threads=1, timeout=3600):
    """Run the reference harness in ``workdir`` (which holds mode.t3c, file.t3c and the
    input .prn).  Returns the parsed JSON line it prints last, or None."""
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    r = subprocess.run([REF, *map(str, args)], cwd=workdir, env=env, stdin=subprocess.DEVNULL,
                       capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise OracleError(f"reference harness failed ({r.returncode}): {r.stderr[-2000:]}")
    for line in reversed(r.stdout.splitlines()):
        i = line.find("{\"")
        if i >= 0:
            try:
                return json.loads(_c_numbers(line[i:]))
            except json.JSONDecodeError:
                continue
    return None


def run_reference_lines(workdir, *args, threads=1, timeout=3600):
    """Like ``run_reference`` but returns every JSON line the harness printed, in order."""
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    try:
        r = subprocess.run([REF, *map(str, args)], cwd=workdir, env=env, stdin=subprocess.DEVNULL,
                           capture_output=True, text=True, timeout=timeout)
    except subprocess.TimeoutExpired as e:
        err = e.stderr.decode(errors="replace") if isinstance(e.stderr, bytes) else (e.stderr or "")
        raise OracleError(f"reference harness timed out after {timeout} s; last progress: {err[-400:]}")
    if r.returncode != 0:
        raise OracleError(f"reference harness failed ({r.returncode}): {r.stderr[-2000:]}")
    out = []
    for line in r.stdout.splitlines():
        i = line.find("{\"")
        if i >= 0:
            try:
                out.append(json.loads(_c_numbers(line[i:])))
            except json.JSONDecodeError:
                continue
    return out


def _c_numbers(line):
    """printf's nan / inf tokens as the JSON parser's NaN / Infinity."""
    import re
    line = re.sub(r"(?<![A-Za-z])-?nan(?![A-Za-z])", "NaN", line)
    return re.sub(r"(?<![A-Za-z])(-?)inf(?![A-Za-z])", r"\1Infinity", line)


def read_csr(path):
    with open(path, "rb") as fh:
        nrows, nnz = np.frombuffer(fh.read(16), np.int64)
        num = np.frombuffer(fh.read(8 * nrows), np.int64)
        col = np.frombuffer(fh.read(8 * nnz), np.int64)
        val = np.frombuffer(fh.read(8 * nnz), np.float64)
        rhs = np.frombuffer(fh.read(8 * nrows), np.float64)
        nn = nrows // 4
        nd = np.frombuffer(fh.read(4 * nn), np.float32)
        nu = np.frombuffer(fh.read(4 * nn), np.float32)
    indptr = np.concatenate([[0], np.cumsum(num)])
    return dict(indptr=indptr, col=col, val=val, rhs=rhs, nd=nd, nu=nu)


def read_sol(path):
    with open(path, "rb") as fh:
        n = int(np.frombuffer(fh.read(8), np.int64)[0])
        sol = np.frombuffer(fh.read(8 * n), np.float64).copy()
        h = int(np.frombuffer(fh.read(8), np.int64)[0])
        hist = np.frombuffer(fh.read(8 * h), np.float64).copy()
    return sol, hist


FIELD_NAMES = ("vx", "vy", "vz", "exx", "eyy", "ezz", "exy", "exz", "eyz", "sxx", "syy", "szz", "sxy", "sxz", "syz")
MARK_NAMES = ("x", "y", "z", "k", "w", "d", "v", "e", "ex", "ft", "rr", "rn")
NODE_NAMES = ("ro", "nu", "nxx", "nxy", "nxz", "nyz", "tk", "cp", "et", "kt", "ht", "rr", "vx", "vy", "vz")


def read_fields(path):
    with open(path, "rb") as fh:
        n = int(np.frombuffer(fh.read(8), np.int64)[0])
        out = {"pr": np.frombuffer(fh.read(8 * n), np.float64).copy()}
        for f in FIELD_NAMES:
            out[f] = np.frombuffer(fh.read(4 * n), np.float32).copy()
        out["timestep"] = float(np.frombuffer(fh.read(8), np.float64)[0])
    return out


def read_marks(path):
    with open(path, "rb") as fh:
        n = int(np.frombuffer(fh.read(8), np.int64)[0])
        out = {f: np.frombuffer(fh.read(4 * n), np.float32).copy() for f in MARK_NAMES}
        out["t"] = np.frombuffer(fh.read(n), np.int8).copy()
    return out


def read_nodes(path):
    with open(path, "rb") as fh:
        n = int(np.frombuffer(fh.read(8), np.int64)[0])
        return {f: np.frombuffer(fh.read(4 * n), np.float32).copy() for f in NODE_NAMES}
