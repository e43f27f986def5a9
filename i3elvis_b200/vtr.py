"""Reader of the ParaView rectilinear-grid files written by ``i3g_write_vtr``.

The files are VTK XML ``RectilinearGrid`` documents with raw appended data, as the reference's
``saver_paraview`` writes them (i3vis_output_paraview.c:700-792): each array in the appended
section is a 4-byte byte count followed by the values, at the offset its ``DataArray`` names.
Point data are in VTK order (x fastest); ``to_model_order`` returns the model's order (node =
z*nx*ny + x*ny + y).
"""
from __future__ import annotations

import re

import numpy as np

_TYPES = {"Float32": np.float32, "Float64": np.float64, "Int32": np.int32, "Int64": np.int64}


def read_vtr(path: str) -> dict:
    """{'extent': (nx, ny, nz), 'xcoor'|'ycoor'|'zcoor'|<field>: array in the file's order}."""
    raw = open(path, "rb").read()
    mark = raw.index(b"<AppendedData")
    start = raw.index(b"_", mark) + 1
    head = raw[:mark].decode()
    ext = [int(v) for v in re.search(r'WholeExtent="([^"]+)"', head).group(1).split()]
    out = {"extent": (ext[1] + 1, ext[3] + 1, ext[5] + 1)}
    for m in re.finditer(r'<DataArray Name="([^"]+)" type="([^"]+)"[^>]*offset="(\d+)"', head):
        name, typ, off = m.group(1), _TYPES[m.group(2)], int(m.group(3))
        n = int(np.frombuffer(raw, np.int32, 1, start + off)[0])
        out[name] = np.frombuffer(raw, typ, n // np.dtype(typ).itemsize, start + off + 4).copy()
    return out


def to_model_order(a: np.ndarray, extent) -> np.ndarray:
    """VTK point order (x fastest) -> the model's node order (y fastest)."""
    nx, ny, nz = extent
    return np.ascontiguousarray(a.reshape(nz, ny, nx).transpose(0, 2, 1)).reshape(-1)
