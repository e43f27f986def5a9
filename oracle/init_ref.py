"""TEST INFRASTRUCTURE: numpy restatement of the initial markers of the reference's generator,
used only by tests to check ``i3g_init_markers``.

* placement (in3mg.c:131-175): cells in (z, x, y) order, inside a cell markers in (z, x, y)
  order, first marker at spacing/2 from the cell corner, the next ones by repeated addition of
  the marker spacing d = (size / (n - 1)) / markers per cell;
* jitter (in3mg.c:177-186): marker += (float)(r mod (2n+1) - n) / (float)n * (float)amplitude
  in FP32, amplitude = fraction * d (in3mg.c:87-89), with the library's counter-based r
  (SplitMix64 of seed and 3 * marker + axis, upper 31 bits) in place of rand();
* bodies (in3mg.c:548-797): boxes bounded by bilinear faces through their corners, ellipsoid
  shells and cylinders along y, in order, on relative coordinates (FP64);
* temperature linear in y between t_top and t_bottom.
"""
from __future__ import annotations

import numpy as np

M64 = (1 << 64) - 1


def splitmix64(seed: int, k: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + (k.astype(np.uint64) + np.uint64(1)) * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def _face(w, u, v, corners):
    A = np.array([[1.0, u[n], v[n], u[n] * v[n]] for n in corners])
    return np.linalg.solve(A, np.array([w[n] for n in corners]))


def markers(shape, size, mnum, nonstab, frac, seed, background, bodies, t_top, t_bottom):
    """Marker arrays x, y, z (FP32), t (int8), ex, e, k (FP32) for a grid of ``shape`` nodes."""
    nx, ny, nz = shape
    mx, my, mz = mnum
    st = [size[a] / (shape[a] - 1) for a in range(3)]
    d = [st[0] / mx, st[1] / my, st[2] / mz]
    # positions by repeated addition, per axis: coordinate of cell c, sub-position m
    def axis(ncell, stp, dd, msub):
        out = np.empty((ncell, msub))
        for c in range(ncell):
            v = c * stp + dd / 2.0
            for m in range(msub):
                out[c, m] = v
                v += dd
        return out
    X, Y, Z = axis(nx - 1, st[0], d[0], mx), axis(ny - 1, st[1], d[1], my), axis(nz - 1, st[2], d[2], mz)
    shp = (nz - 1, nx - 1, ny - 1, mz, mx, my)
    z = np.broadcast_to(Z[:, None, None, :, None, None], shp).reshape(-1).astype(np.float32)
    x = np.broadcast_to(X[None, :, None, None, :, None], shp).reshape(-1).astype(np.float32)
    y = np.broadcast_to(Y[None, None, :, None, None, :], shp).reshape(-1).astype(np.float32)
    n = x.size
    if nonstab:
        idx = np.arange(n, dtype=np.uint64)
        span = 2 * nonstab + 1
        for a, arr in enumerate((x, y, z)):
            r = (splitmix64(seed, np.uint64(3) * idx + np.uint64(a)) >> np.uint64(33)).astype(np.int64)
            amp = np.float32(frac[a] * size[a] / (shape[a] - 1) / mnum[a])
            off = ((r % span - nonstab).astype(np.float32) / np.float32(nonstab)) * amp
            arr += off
    t = np.full(n, background, np.int8)
    ex = np.zeros(n, np.float32)
    e = np.zeros(n, np.float32)
    rx, ry, rz = (x.astype(np.float64) / size[0], y.astype(np.float64) / size[1], z.astype(np.float64) / size[2])
    for b in bodies:
        if b["shape"] == 0:
            bx, by, bz = b["x"], b["y"], b["z"]
            k = [_face(bx, by, bz, (0, 1, 4, 5)), _face(bx, by, bz, (2, 3, 6, 7)),
                 _face(by, bx, bz, (0, 2, 4, 6)), _face(by, bx, bz, (1, 3, 5, 7)),
                 _face(bz, by, bx, (0, 1, 2, 3)), _face(bz, by, bx, (4, 5, 6, 7))]
            f = lambda q, u, v: q[0] + q[1] * u + q[2] * v + q[3] * u * v
            inside = ((rx >= f(k[0], ry, rz)) & (rx <= f(k[1], ry, rz)) & (ry >= f(k[2], rx, rz)) &
                      (ry <= f(k[3], rx, rz)) & (rz >= f(k[4], ry, rx)) & (rz <= f(k[5], ry, rx)))
        else:
            ux = (rx - b["x"][0]) / b["x"][7]
            uy = (ry - b["y"][0]) / b["y"][7]
            uz = (rz - b["z"][0]) / b["z"][7]
            r = np.sqrt(ux * ux + uy * uy + uz * uz) if b["shape"] == 1 else np.sqrt(ux * ux + uz * uz)
            inside = (r >= b["x"][2]) & (r <= b["x"][5])
            if b["shape"] == 2:
                inside &= np.abs(uy) <= 1.0
        t[inside] = b["rock"]
        ex[inside] = np.float32(b["ex"])
        e[inside] = np.float32(b["e"])
    k = (t_top + (t_bottom - t_top) * y.astype(np.float64) / size[1]).astype(np.float32)
    return dict(x=x, y=y, z=z, t=t, ex=ex, e=e, k=k)
