"""Binary ``.prn`` restart files, byte-compatible with the reference.

The layout follows ``loader`` / ``saver`` in ``load3mg.c:704-1063``:

* four size bytes (int, long, float, double),
* grid and run scalars (``load3mg.c:739-761``),
* 24 rock-property tables of ``rocknum`` doubles (``load3mg.c:766-789``),
* 16 FP32 nodal fields per node, interleaved (``load3mg.c:793-811``),
* FP32 grid-line coordinates ``gx, gy, gz`` (``load3mg.c:814-825``),
* ``bondnum`` boundary records ``(long row, long id, float c, float k, long partner+1)``
  (``load3mg.c:828-838``),
* ``marknum`` 49-byte marker records: 12 FP32 fields and one ``char`` type
  (``load3mg.c:845-859``).

Everything is native little-endian with ``sizeof(long) == 8`` as on the reference's
Linux build.  The reader keeps nodal fields and marker fields as separate numpy arrays
(structure of arrays), which is the layout the device kernels use.
"""
from __future__ import annotations

import dataclasses
import numpy as np

NODE_FIELDS = ("pr", "vx", "vy", "vz", "ro", "nu", "nxx", "nxy", "nxz", "nyz",
               "tk", "cp", "et", "kt", "ht", "rr")
MARK_FIELDS = ("x", "y", "z", "k", "w", "d", "v", "e", "ex", "ft", "rr", "rn")
ROCK_FIELDS = ("n0", "n1", "s0", "s1", "nu", "dh", "dv", "ss", "mm", "ll", "a0", "a1",
               "b0", "b1", "e0", "e1", "ro", "bb", "aa", "cp", "kt", "kf", "kp", "ht")

_HEAD = np.dtype([
    ("xnumx", "<i8"), ("ynumy", "<i8"), ("znumz", "<i8"),
    ("mnumx", "<i8"), ("mnumy", "<i8"), ("mnumz", "<i8"),
    ("xsize", "<f8"), ("ysize", "<f8"), ("zsize", "<f8"),
    ("pxinit", "<i8"), ("pyinit", "<i8"), ("pzinit", "<i8"),
    ("pinit", "<f8"), ("gxkoef", "<f8"), ("gykoef", "<f8"), ("gzkoef", "<f8"),
    ("rocknum", "<i4"), ("bondnum", "<i8"), ("marknum", "<i8"), ("cycle", "<i4"),
    ("timesum_yr", "<f8"), ("gridcur", "<f8"), ("gridtot", "<f8"),
])
_NODE = np.dtype([(f, "<f4") for f in NODE_FIELDS])
_BOND = np.dtype([("row", "<i8"), ("id", "<i8"), ("c", "<f4"), ("k", "<f4"), ("partner1", "<i8")])
_MARK = np.dtype([(f, "<f4") for f in MARK_FIELDS] + [("t", "i1")])
assert _MARK.itemsize == 49 and _BOND.itemsize == 32 and _HEAD.itemsize == 176

YEAR = 3.15576e7  # seconds per year used throughout the reference (load3mg.c:44)


@dataclasses.dataclass
class Prn:
    """In-memory image of one ``.prn`` file (structure of arrays)."""
    head: dict
    rocks: dict            # name -> float64[rocknum]
    nodes: dict            # name -> float32[nodenum]
    gx: np.ndarray         # float32[xnumx]
    gy: np.ndarray
    gz: np.ndarray
    bond: np.ndarray       # structured _BOND records
    marks: dict            # name -> float32[marknum]; "t" -> int8[marknum]

    @property
    def shape(self):
        h = self.head
        return int(h["xnumx"]), int(h["ynumy"]), int(h["znumz"])

    @property
    def nodenum(self):
        x, y, z = self.shape
        return x * y * z

    @property
    def marknum(self):
        return int(self.head["marknum"])

    def copy(self) -> "Prn":
        return Prn(dict(self.head), {k: v.copy() for k, v in self.rocks.items()},
                   {k: v.copy() for k, v in self.nodes.items()}, self.gx.copy(), self.gy.copy(),
                   self.gz.copy(), self.bond.copy(), {k: v.copy() for k, v in self.marks.items()})


class PrnFormatError(ValueError):
    pass


def read_prn(path) -> Prn:
    raw = np.fromfile(path, dtype=np.uint8)
    if raw.size < 4 + _HEAD.itemsize:
        raise PrnFormatError(f"{path}: file too short for a .prn header ({raw.size} bytes)")
    sizes = tuple(int(b) for b in raw[:4])
    if sizes != (4, 8, 4, 8):
        raise PrnFormatError(f"{path}: type sizes {sizes} differ from (int 4, long 8, float 4, double 8)")
    off = 4
    head_rec = np.frombuffer(raw, dtype=_HEAD, count=1, offset=off)[0]
    head = {name: head_rec[name].item() for name in _HEAD.names}
    off += _HEAD.itemsize
    nx, ny, nz = head["xnumx"], head["ynumy"], head["znumz"]
    rn, bn, mn = head["rocknum"], head["bondnum"], head["marknum"]
    if min(nx, ny, nz) < 5 or rn < 0 or bn < 0 or mn < 0:
        raise PrnFormatError(f"{path}: implausible header {head}")
    nodenum = nx * ny * nz
    need = (off + 24 * rn * 8 + nodenum * _NODE.itemsize + (nx + ny + nz) * 4
            + bn * _BOND.itemsize + mn * _MARK.itemsize)
    if raw.size < need:
        raise PrnFormatError(f"{path}: truncated ({raw.size} bytes, header implies {need})")
    rocks = {}
    for name in ROCK_FIELDS:
        rocks[name] = np.frombuffer(raw, "<f8", rn, off).copy()
        off += rn * 8
    nrec = np.frombuffer(raw, _NODE, nodenum, off)
    off += nodenum * _NODE.itemsize
    nodes = {f: np.ascontiguousarray(nrec[f]) for f in NODE_FIELDS}
    gx = np.frombuffer(raw, "<f4", nx, off).copy(); off += nx * 4
    gy = np.frombuffer(raw, "<f4", ny, off).copy(); off += ny * 4
    gz = np.frombuffer(raw, "<f4", nz, off).copy(); off += nz * 4
    bond = np.frombuffer(raw, _BOND, bn, off).copy(); off += bn * _BOND.itemsize
    mrec = np.frombuffer(raw, _MARK, mn, off)
    marks = {f: np.ascontiguousarray(mrec[f]) for f in MARK_FIELDS}
    marks["t"] = np.ascontiguousarray(mrec["t"])
    return Prn(head, rocks, nodes, gx, gy, gz, bond, marks)


def write_prn(path, prn: Prn) -> None:
    """Write ``prn`` in the exact byte layout of ``saver`` (``load3mg.c:898-1063``).  Node and
    marker records are assembled and written in chunks of 2^20 records."""
    h = dict(prn.head)
    h["bondnum"] = int(prn.bond.shape[0])
    h["marknum"] = int(prn.marks["x"].shape[0])
    head_rec = np.zeros(1, _HEAD)
    for name in _HEAD.names:
        head_rec[name] = h[name]
    nodenum = prn.nodenum
    bond = np.ascontiguousarray(prn.bond, dtype=_BOND)
    chunk = 1 << 20
    with open(path, "wb") as fh:
        fh.write(bytes([4, 8, 4, 8]))
        fh.write(head_rec.tobytes())
        for name in ROCK_FIELDS:
            fh.write(np.asarray(prn.rocks[name], "<f8").tobytes())
        for a in range(0, nodenum, chunk):
            e = min(nodenum, a + chunk)
            nrec = np.empty(e - a, _NODE)
            for f in NODE_FIELDS:
                nrec[f] = prn.nodes[f][a:e]
            fh.write(nrec.tobytes())
        fh.write(np.asarray(prn.gx, "<f4").tobytes())
        fh.write(np.asarray(prn.gy, "<f4").tobytes())
        fh.write(np.asarray(prn.gz, "<f4").tobytes())
        fh.write(bond.tobytes())
        for a in range(0, h["marknum"], chunk):
            e = min(h["marknum"], a + chunk)
            mrec = np.empty(e - a, _MARK)
            for f in MARK_FIELDS:
                mrec[f] = prn.marks[f][a:e]
            mrec["t"] = prn.marks["t"][a:e]
            fh.write(mrec.tobytes())


def empty_bond(n: int) -> np.ndarray:
    return np.zeros(n, _BOND)
