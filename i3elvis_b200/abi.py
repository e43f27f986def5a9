"""ctypes mirror of ``include/i3g.h`` and helpers that fill it from a ``.prn`` image.

The C structs hold plain pointers into numpy arrays; ``ModelBuffers`` owns those arrays
(contiguous copies of the ``Prn`` fields plus the stress/strain-rate fields the Stokes step
writes), so that a download writes straight back into numpy.
"""
from __future__ import annotations

import ctypes as C
import numpy as np

from .config import Mode, OutFile
from .prn import Prn, ROCK_FIELDS, YEAR

MAXLEV = 12
c_f32p = C.POINTER(C.c_float)
c_f64p = C.POINTER(C.c_double)
c_i64p = C.POINTER(C.c_int64)
c_i8p = C.POINTER(C.c_int8)

E_CODES = {0: "OK", -1: "ARG", -2: "CUDA", -3: "NOMEM", -4: "UNSUPPORTED", -5: "NOCONV",
           -6: "NAN", -7: "PRESSURE", -8: "BC"}
SYNC_NODES, SYNC_STRESS, SYNC_MARKERS, SYNC_ALL = 1, 2, 4, 7
SYNC_ASYNC = 8   # upload: marker copies overlap the following calls (include/i3g.h)
A_SOL, A_RHS, A_RES, A_NU, A_ETA, A_TK = range(6)

NODE_F32 = ("vx", "vy", "vz", "ro", "nu", "nxx", "nxy", "nxz", "nyz", "tk", "cp", "et", "kt", "ht", "rr")
STRESS_F32 = ("exx", "eyy", "ezz", "exy", "exz", "eyz", "sxx", "syy", "szz", "sxy", "sxz", "syz")
MARK_F32 = ("markx", "marky", "markz", "markk", "markw", "markd", "markv", "marke", "markex",
            "markft", "markrr", "markrn")
_MARK_SRC = dict(zip(MARK_F32, ("x", "y", "z", "k", "w", "d", "v", "e", "ex", "ft", "rr", "rn")))


class Model(C.Structure):
    _fields_ = [
        ("xnumx", C.c_int64), ("ynumy", C.c_int64), ("znumz", C.c_int64),
        ("mnumx", C.c_int64), ("mnumy", C.c_int64), ("mnumz", C.c_int64),
        ("xsize", C.c_double), ("ysize", C.c_double), ("zsize", C.c_double),
        ("pxinit", C.c_int64), ("pyinit", C.c_int64), ("pzinit", C.c_int64),
        ("pinit", C.c_double), ("gxkoef", C.c_double), ("gykoef", C.c_double), ("gzkoef", C.c_double),
        ("timesum", C.c_double),
        ("gx", c_f32p), ("gy", c_f32p), ("gz", c_f32p),
        ("pr", c_f64p),
    ] + [(f, c_f32p) for f in NODE_F32] + [(f, c_f32p) for f in STRESS_F32] + [
        ("bondnum", C.c_int64), ("bond_row", c_i64p), ("bond_c", c_f32p), ("bond_k", c_f32p),
        ("bond_partner1", c_i64p),
        ("marknum", C.c_int64),
    ] + [(f, c_f32p) for f in MARK_F32] + [
        ("markt", c_i8p),
        ("rocknum", C.c_int32),
        ("rock", c_f64p * 24),
    ]


class Body(C.Structure):
    """``i3g_body``: a rock body of init.t3c (in3mg.c:548-797), coordinates relative to the box."""
    _fields_ = [("rock", C.c_int32), ("shape", C.c_int32), ("x", C.c_double * 8), ("y", C.c_double * 8),
                ("z", C.c_double * 8), ("ex", C.c_double), ("e", C.c_double)]


class Init(C.Structure):
    """``i3g_init``: initial markers of in3mg.c:131-797 (jitter, background rock, bodies, T)."""
    _fields_ = [("nonstab", C.c_int32), ("xnonstab", C.c_double), ("ynonstab", C.c_double),
                ("znonstab", C.c_double), ("seed", C.c_uint64), ("background", C.c_int32),
                ("t_top", C.c_double), ("t_bottom", C.c_double), ("nbodies", C.c_int32),
                ("bodies", C.POINTER(Body))]


def box_body(rock, lo, hi, ex=0.0, e=0.0):
    """An axis-aligned box body from relative corners lo = (x, y, z), hi (shape 0)."""
    b = Body(rock=rock, shape=0, ex=ex, e=e)
    for n in range(8):
        b.x[n] = hi[0] if n & 2 else lo[0]
        b.y[n] = hi[1] if n & 1 else lo[1]
        b.z[n] = hi[2] if n & 4 else lo[2]
    return b


def sphere_body(rock, centre, scale, r0=0.0, r1=1.0, cylinder=False, ex=0.0, e=0.0):
    """Ellipsoid shell (or cylinder along y) body: centre and axis scales relative to the box,
    scaled radius between r0 and r1 (shapes 1 and 2)."""
    b = Body(rock=rock, shape=2 if cylinder else 1, ex=ex, e=e)
    b.x[0], b.y[0], b.z[0] = centre
    b.x[7], b.y[7], b.z[7] = scale
    b.x[2], b.x[5] = r0, r1
    return b


class Params(C.Structure):
    _fields_ = [
        ("printmod", C.c_int32), ("movemod", C.c_int32), ("tempmod", C.c_int32), ("markmod", C.c_int32),
        ("gridmod", C.c_int32), ("outgrid", C.c_int32), ("densimod", C.c_int32),
        ("stp100", C.c_double), ("eroslev", C.c_double), ("sedilev", C.c_double), ("waterlev", C.c_double),
        ("DIVVMIN", C.c_double), ("STOKSMIN", C.c_double), ("DIVVMAX", C.c_double), ("STOKSMAX", C.c_double),
        ("multimax", C.c_int32), ("multicyc", C.c_int32), ("multinnn", (C.c_int32 * MAXLEV) * 2),
        ("p0koef", C.c_double), ("p1koef", C.c_double), ("p2koef", C.c_double), ("v0koef", C.c_double),
        ("v1koef", C.c_double), ("nubeg", C.c_double), ("nuend", C.c_double), ("nukoef", C.c_double),
        ("viscmod", C.c_int32),
        ("HEATMIN", C.c_double), ("multicyct", C.c_int32), ("multittt0", C.c_int32),
        ("t0koef", C.c_double), ("heatdif", C.c_double), ("frictyn", C.c_int32), ("adiabyn", C.c_int32),
        ("zdeep", C.c_double), ("vdeep", C.c_double), ("tdeep", C.c_double), ("nudeep", C.c_double),
        ("healrate", C.c_double), ("teclmin", C.c_double), ("teclmax", C.c_double),
        ("timebeg", C.c_double), ("timeend", C.c_double), ("tempend", C.c_double),
        ("stokes_rtol", C.c_double), ("stokes_maxcyc", C.c_int32), ("heat_rtol", C.c_double),
        ("heat_maxcyc", C.c_int32), ("precision", C.c_int32), ("warm_start", C.c_int32),
        ("krylov", C.c_int32), ("marker_exact", C.c_int32),
    ]


class FileParams(C.Structure):
    _fields_ = [
        ("cyc0max", C.c_int32), ("maxxystep", C.c_double), ("maxtkstep", C.c_double),
        ("maxtmstep", C.c_double), ("nubeg", C.c_double), ("nuend", C.c_double),
        ("p0koef", C.c_double), ("p1koef", C.c_double), ("p2koef", C.c_double),
        ("p0koef2", C.c_double), ("p1koef2", C.c_double), ("p2koef2", C.c_double),
        ("multinum", C.c_int32), ("multstp", C.c_int32), ("multinum2", C.c_int32),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("stokes_cycles", C.c_int32), ("stokes_outer", C.c_int32),
        ("stokes_rel0", C.c_double), ("stokes_rel", C.c_double),
        ("stokes_mom_rel", C.c_double), ("stokes_cont_rel", C.c_double),
        ("heat_cycles", C.c_int32), ("heat_substeps", C.c_int32), ("heat_rel", C.c_double),
        ("ms_stokes", C.c_double), ("ms_heat", C.c_double), ("ms_move", C.c_double), ("ms_r2n", C.c_double),
        ("kernel_launches", C.c_int64), ("stokes_start", C.c_int32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def _ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


def _pinned_like(a, keep):
    """Page-locked copy of ``a`` (through torch) so host<->device copies run at full speed;
    the owning tensor is appended to ``keep``."""
    import torch
    t = torch.empty(a.shape, dtype=getattr(torch, str(a.dtype)), pin_memory=True)
    keep.append(t)
    out = t.numpy()
    out[...] = a
    return out


class ModelBuffers:
    """Numpy storage behind one ``Model`` struct (page-locked when ``pinned``)."""

    def __init__(self, prn: Prn, pinned: bool = False):
        self.prn = prn
        n = prn.nodenum
        self.gx = np.ascontiguousarray(prn.gx, np.float32)
        self.gy = np.ascontiguousarray(prn.gy, np.float32)
        self.gz = np.ascontiguousarray(prn.gz, np.float32)
        self.pr = np.ascontiguousarray(prn.nodes["pr"], np.float64)
        self.f32 = {f: np.ascontiguousarray(prn.nodes[f], np.float32).copy() for f in NODE_F32}
        for f in STRESS_F32:
            self.f32[f] = np.zeros(n, np.float32)
        for f in MARK_F32:
            self.f32[f] = np.ascontiguousarray(prn.marks[_MARK_SRC[f]], np.float32).copy()
        self.markt = np.ascontiguousarray(prn.marks["t"], np.int8).copy()
        self._pinned = []
        if pinned:
            self.pr = _pinned_like(self.pr, self._pinned)
            self.f32 = {k: _pinned_like(v, self._pinned) for k, v in self.f32.items()}
            self.markt = _pinned_like(self.markt, self._pinned)
        b = prn.bond
        self.bond_row = np.ascontiguousarray(b["row"], np.int64)
        self.bond_c = np.ascontiguousarray(b["c"], np.float32)
        self.bond_k = np.ascontiguousarray(b["k"], np.float32)
        self.bond_p1 = np.ascontiguousarray(b["partner1"], np.int64)
        self.rocks = [np.ascontiguousarray(prn.rocks[f], np.float64) for f in ROCK_FIELDS]
        h = prn.head
        m = Model()
        for k in ("xnumx", "ynumy", "znumz", "mnumx", "mnumy", "mnumz", "pxinit", "pyinit", "pzinit"):
            setattr(m, k, int(h[k]))
        for k in ("xsize", "ysize", "zsize", "pinit", "gxkoef", "gykoef", "gzkoef"):
            setattr(m, k, float(h[k]))
        m.timesum = float(h["timesum_yr"]) * YEAR
        m.gx, m.gy, m.gz = _ptr(self.gx, C.c_float), _ptr(self.gy, C.c_float), _ptr(self.gz, C.c_float)
        m.pr = _ptr(self.pr, C.c_double)
        for f, a in self.f32.items():
            setattr(m, f, _ptr(a, C.c_float))
        m.bondnum = len(self.bond_row)
        m.bond_row = _ptr(self.bond_row, C.c_int64)
        m.bond_c = _ptr(self.bond_c, C.c_float)
        m.bond_k = _ptr(self.bond_k, C.c_float)
        m.bond_partner1 = _ptr(self.bond_p1, C.c_int64)
        m.marknum = prn.marknum
        m.markt = _ptr(self.markt, C.c_int8)
        m.rocknum = int(h["rocknum"])
        for i, a in enumerate(self.rocks):
            m.rock[i] = _ptr(a, C.c_double)
        self.model = m

    def to_prn(self) -> Prn:
        """A ``Prn`` holding the current buffer contents (for ``write_prn``)."""
        p = self.prn.copy()
        p.nodes["pr"] = self.pr.astype(np.float32)
        for f in NODE_F32:
            p.nodes[f] = self.f32[f].copy()
        for f in MARK_F32:
            p.marks[_MARK_SRC[f]] = self.f32[f].copy()
        p.marks["t"] = self.markt.copy()
        p.head["timesum_yr"] = self.model.timesum / YEAR
        return p


def make_params(mode: Mode, **solver) -> Params:
    p = Params()
    for k in ("printmod", "movemod", "tempmod", "markmod", "gridmod", "outgrid", "densimod"):
        setattr(p, k, int(getattr(mode, k)))
    for k in ("stp100", "eroslev", "sedilev", "waterlev", "DIVVMIN", "STOKSMIN", "DIVVMAX", "STOKSMAX",
              "p0koef", "p1koef", "p2koef", "v0koef", "v1koef", "nubeg", "nuend", "nukoef", "HEATMIN",
              "t0koef", "heatdif"):
        setattr(p, k, float(getattr(mode, k)))
    p.multimax = mode.multinum
    p.multicyc = mode.multicyc
    for i in range(2):
        for l, v in enumerate(mode.multinnn[i]):
            p.multinnn[i][l] = int(v)
    p.viscmod = mode.viscmod
    p.multicyct = mode.multicyct
    p.multittt0 = int(mode.multittt[0][0])
    p.frictyn, p.adiabyn = int(mode.frictyn), int(mode.adiabyn)
    for k in ("zdeep", "vdeep", "tdeep", "nudeep", "healrate", "teclmin", "teclmax"):
        setattr(p, k, mode.water_param(k))
    p.timebeg, p.timeend, p.tempend = mode.timebeg_yr * YEAR, mode.timeend_yr * YEAR, 0.0
    p.stokes_rtol = solver.get("stokes_rtol", 1e-8)
    p.stokes_maxcyc = solver.get("stokes_maxcyc", 2000)
    p.heat_rtol = solver.get("heat_rtol", 1e-10)
    p.heat_maxcyc = solver.get("heat_maxcyc", 2000)
    p.precision = solver.get("precision", 0)
    p.warm_start = solver.get("warm_start", 1)
    p.krylov = solver.get("krylov", 0)
    p.marker_exact = solver.get("marker_exact", 0)
    return p


def make_file_params(f: OutFile) -> FileParams:
    fp = FileParams()
    fp.cyc0max = f.cyc0max
    fp.maxxystep, fp.maxtkstep, fp.maxtmstep = f.maxxystep, f.maxtkstep, f.maxtmstep_yr * YEAR
    fp.nubeg, fp.nuend = f.nubeg, f.nuend
    fp.p0koef, fp.p1koef, fp.p2koef = f.p0koef, f.p1koef, f.p2koef
    fp.p0koef2, fp.p1koef2, fp.p2koef2 = f.p0koef2, f.p1koef2, f.p2koef2
    fp.multinum, fp.multstp, fp.multinum2 = f.multinum, f.multstp, f.multinum2
    return fp
