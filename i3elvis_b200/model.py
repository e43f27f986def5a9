"""Synthetic model builder: grid, seeded markers, rock types and boundary conditions.

This writes the same kind of restart image that the reference's initial-condition
generator produces (``in3mg.c:25-1055``), for the synthetic workloads used by the tests
and the benchmark:

* grid lines ``gx, gy, gz`` uniform as in ``in3mg.c:96-101`` (stored as FP32 like the
  ``.prn`` writer does),
* markers on a regular sub-grid per cell, cell-major order, jittered by
  ``(r % (2n+1) - n)/n * frac * spacing`` as in ``in3mg.c:131-187`` (``r`` from a seeded
  generator instead of unseeded ``rand()``),
* boundary-condition boxes expanded onto every multigrid level with the index mapping of
  ``in3mg.c:313-408``,
* the multigrid level geometry of ``gridcheck`` (``load3mg.c:1162-1283``).

Nodal fields are left at zero; ``prepare`` in the runtime fills them from the markers the
way ``in3mg.c:990-1031`` does (marker->node average, hydrostatic pressure, average again).
The vertical axis is the reference's ``y`` (gravity ``GYKOEF`` > 0 points to larger y).
"""
from __future__ import annotations

import dataclasses
import numpy as np

from .prn import Prn, ROCK_FIELDS, empty_bond


def level_dims(n0: int, multinum: int):
    """``mgx[n]=((mgx[n-1]-5)/2)+5`` (``load3mg.c:1228``)."""
    dims = [n0]
    for _ in range(multinum):
        dims.append((dims[-1] - 5) // 2 + 5)
    return dims


def level_coords(g: np.ndarray, multinum: int):
    """Per-level grid coordinates keeping 3 outer nodes per side (``load3mg.c:1235-1282``)."""
    g = np.asarray(g, np.float64)
    n = g.size
    out = []
    for lev, m in enumerate(level_dims(n, multinum)):
        s = 1 << lev
        c = np.empty(m)
        c[0:3] = g[0:3]
        c[m - 3:] = g[n - 3:]
        for i in range(3, m - 3):
            c[i] = g[(i - 2) * s + 2]
        out.append(c)
    return out


@dataclasses.dataclass
class BcBox:
    """One boundary-condition box: ``var`` is P, Vx, Vy, Vz or T; the row is
    ``x_i = c + k * x_(i+shift)`` over the inclusive node box (``in3mg.c:266-300``)."""
    var: str
    x0: int
    x1: int
    y0: int
    y1: int
    z0: int
    z1: int
    c: float = 0.0
    k: float = 0.0
    shift: tuple = (0, 0, 0)


_VAR_INDEX = {"P": 0, "Vx": 1, "Vy": 2, "Vz": 3, "T": 4}


def free_slip_boxes(nx, ny, nz, t_top, t_bottom):
    """Free-slip box with fixed top/bottom temperature and insulating sides.

    Same box list as the reference specimen's boundary block (``init.t3c:132-168``) with
    the internal box removed, free slip (``k=1``) on the bottom too and no flow through
    the bottom wall."""
    x, y, z = nx - 1, ny - 1, nz - 1
    B = BcBox
    boxes = []
    for yy, s in ((1, None), (y, None)):
        boxes += [B("P", 1, x, yy, yy, 1, 1, 0, 1, (0, 0, 1)),
                  B("P", 1, 1, yy, yy, 2, z - 1, 0, 1, (1, 0, 0)),
                  B("P", 1, x, yy, yy, z, z, 0, 1, (0, 0, -1)),
                  B("P", x, x, yy, yy, 2, z - 1, 0, 1, (-1, 0, 0))]
        if yy == 1:
            boxes += [B("Vx", 1, x - 1, 0, 0, 0, z - 1, 0, 1, (0, 1, 0)),
                      B("Vy", 0, x - 1, 0, 0, 0, z - 1, 0, 0),
                      B("Vz", 0, x - 1, 0, 0, 1, z - 1, 0, 1, (0, 1, 0)),
                      B("T", 0, x, 0, 0, 0, z, t_top, 0)]
        else:
            boxes += [B("Vx", 1, x - 1, y - 1, y - 1, 0, z - 1, 0, 1, (0, -1, 0)),
                      B("Vy", 0, x - 1, y, y, 0, z - 1, 0, 0),
                      B("Vz", 0, x - 1, y - 1, y - 1, 1, z - 1, 0, 1, (0, -1, 0)),
                      B("T", 0, x, y, y, 0, z, t_bottom, 0)]
    boxes += [B("P", 1, 1, 2, y - 1, 1, 1, 0, 1, (1, 0, 1)),
              B("P", 1, 1, 2, y - 1, z, z, 0, 1, (1, 0, -1)),
              B("Vx", 0, 0, 0, y - 1, 0, z - 1, 0, 0),
              B("Vy", 0, 0, 1, y - 1, 0, z - 1, 0, 1, (1, 0, 0)),
              B("Vz", 0, 0, 0, y - 1, 1, z - 1, 0, 1, (1, 0, 0)),
              B("T", 0, 0, 1, y - 1, 0, z, 0, 1, (1, 0, 0))]
    boxes += [B("P", x, x, 2, y - 1, 1, 1, 0, 1, (-1, 0, 1)),
              B("P", x, x, 2, y - 1, z, z, 0, 1, (-1, 0, -1)),
              B("Vx", x, x, 0, y - 1, 0, z - 1, 0, 0),
              B("Vy", x - 1, x - 1, 1, y - 1, 0, z - 1, 0, 1, (-1, 0, 0)),
              B("Vz", x - 1, x - 1, 0, y - 1, 1, z - 1, 0, 1, (-1, 0, 0)),
              B("T", x, x, 1, y - 1, 0, z, 0, 1, (-1, 0, 0))]
    boxes += [B("Vx", 1, x - 1, 0, y - 1, 0, 0, 0, 1, (0, 0, 1)),
              B("Vy", 0, x - 1, 1, y - 1, 0, 0, 0, 1, (0, 0, 1)),
              B("Vz", 0, x - 1, 0, y - 1, 0, 0, 0, 0),
              B("T", 1, x - 1, 1, y - 1, 0, 0, 0, 1, (0, 0, 1))]
    boxes += [B("Vx", 1, x - 1, 0, y - 1, z - 1, z - 1, 0, 1, (0, 0, -1)),
              B("Vy", 0, x - 1, 1, y - 1, z - 1, z - 1, 0, 1, (0, 0, -1)),
              B("Vz", 0, x - 1, 0, y - 1, z, z, 0, 0),
              B("T", 1, x - 1, 1, y - 1, z, z, 0, 1, (0, 0, -1))]
    return boxes


def _lim(m, n, mg, s):
    """Fine box limit -> level limit (``in3mg.c:319-336``); C division truncates toward 0."""
    if m < 3:
        return m
    if m > n - 4:
        return mg - (n - m)
    return int((m - 2) / s) + 2


def expand_bc(boxes, shape, multinum):
    """Expand BC boxes onto all multigrid levels (``in3mg.c:313-408``).

    Returns the ``.prn`` boundary records sorted by row: ``row`` indexes ``bondm``
    (``4*node + var`` for P/Vx/Vy/Vz, ``8*nodenum + node`` for T, node numbers counting
    all levels), ``partner1`` is the partner row + 1 (0 = none)."""
    nx, ny, nz = shape
    dx, dy, dz = (level_dims(n, multinum) for n in shape)
    nodenum = nx * ny * nz
    mgp = [0]
    for l in range(multinum):
        mgp.append(mgp[-1] + dx[l] * dy[l] * dz[l])
    bondm = {}
    vals = {}
    bid = 0
    for b in boxes:
        var = _VAR_INDEX[b.var]
        has_shift = any(b.shift)
        for l in range(multinum + 1):
            s = 1 << l
            x0, x1 = _lim(b.x0, nx, dx[l], s), _lim(b.x1, nx, dx[l], s)
            y0, y1 = _lim(b.y0, ny, dy[l], s), _lim(b.y1, ny, dy[l], s)
            z0, z1 = _lim(b.z0, nz, dz[l], s), _lim(b.z1, nz, dz[l], s)
            mgy, mgxy = dy[l], dx[l] * dy[l]
            for k3 in range(z0, z1 + 1):
                for k1 in range(x0, x1 + 1):
                    for k2 in range(y0, y1 + 1):
                        m4 = mgp[l] + k3 * mgxy + k1 * mgy + k2
                        m6 = m4 + b.shift[2] * mgxy + b.shift[0] * mgy + b.shift[1]
                        bid += 1
                        if var < 4:
                            row = m4 * 4 + var
                            partner1 = m6 * 4 + var + 1 if has_shift else 0
                        else:
                            row = 8 * nodenum + m4
                            partner1 = m6 + 1 if has_shift else 0
                        bondm[row] = bid
                        vals[bid] = (b.c, b.k if has_shift else 0.0, partner1)
    rows = sorted(bondm)
    bond = empty_bond(len(rows))
    for i, r in enumerate(rows):
        c, k, p1 = vals[bondm[r]]
        bond[i] = (r, bondm[r], c, k, p1)
    return bond


@dataclasses.dataclass
class Rock:
    """One rock type (columns of the reference's rock table, ``in3mg.c:201-234``)."""
    n0: float = 1e18
    n1: float = 1e26
    s0: float = 0.0
    s1: float = 5e29
    nu: float = 1e21
    dh: float = 0.0
    dv: float = 0.0
    ss: float = 0.0
    mm: float = 1.0
    ll: float = 0.0
    a0: float = 0.0
    a1: float = 0.0
    b0: float = 0.0
    b1: float = 0.0
    e0: float = 0.0
    e1: float = 1.0
    ro: float = 3300.0
    bb: float = 0.0
    aa: float = 0.0
    cp: float = 1000.0
    kt: float = 3.0
    kf: float = 0.0
    kp: float = 0.0
    ht: float = 0.0


@dataclasses.dataclass
class ModelSpec:
    shape: tuple
    size: tuple              # xsize, ysize, zsize in metres
    mnum: tuple = (3, 3, 3)  # markers per cell along x, y, z
    jitter: float = 0.5      # fraction of the marker spacing (in3mg ``xnonstab``)
    nonstab: int = 100
    gravity: tuple = (0.0, 10.0, 0.0)
    pinit_cell: tuple = (2, 1, 2)
    pinit: float = 1e5
    t_top: float = 273.0
    t_bottom: float = 1573.0
    multinum: int = 2
    stretch: float = 0.0     # 0: uniform grid lines; a in (0, 1): spacing (1 - a cos(2 pi s)) * size/(n-1)
    spheres: tuple = ()      # (rock, (x, y, z) centre in metres, radius in metres) of the bodies, in order


def _grid(n, size, stretch=0.0):
    """Grid lines from 0 to size: uniform as in in3mg.c:96-101, or (stretch = a > 0) the smooth
    non-uniform map x(s) = size * (s - a sin(2 pi s) / (2 pi)), s = i/(n-1), whose spacing grows
    from (1 - a) h at the walls to (1 + a) h in the middle -- the reference keeps arbitrary grid
    lines in the .prn file (load3mg.c:739-751) and every formula uses them."""
    if stretch:
        s = np.arange(n, dtype=np.float64) / (n - 1)
        g = size * (s - stretch * np.sin(2 * np.pi * s) / (2 * np.pi))
        g[0], g[-1] = 0.0, size
        return g.astype(np.float32)
    step = size / (n - 1)
    g = np.zeros(n)
    for i in range(1, n):
        g[i] = g[i - 1] + step
    g[-1] = size
    return g.astype(np.float32)


def build_markers(spec: ModelSpec, seed: int):
    """Markers on a regular sub-grid per cell in cell-major order (cell (z, x, y), inside a
    cell (z, x, y)) as in in3mg.c:141-175, jittered as in in3mg.c:177-186."""
    nx, ny, nz = spec.shape
    xs, ys, zs = spec.size
    mx, my, mz = spec.mnum
    stp = (xs / (nx - 1), ys / (ny - 1), zs / (nz - 1))
    d = (stp[0] / mx, stp[1] / my, stp[2] / mz)
    shape = (nz - 1, nx - 1, ny - 1, mz, mx, my)
    cz = (np.arange(nz - 1) * stp[2])[:, None, None, None, None, None]
    cx = (np.arange(nx - 1) * stp[0])[None, :, None, None, None, None]
    cy = (np.arange(ny - 1) * stp[1])[None, None, :, None, None, None]
    sz = (d[2] / 2.0 + np.arange(mz) * d[2])[None, None, None, :, None, None]
    sx = (d[0] / 2.0 + np.arange(mx) * d[0])[None, None, None, None, :, None]
    sy = (d[1] / 2.0 + np.arange(my) * d[1])[None, None, None, None, None, :]
    x = np.broadcast_to((cx + sx).astype(np.float32), shape).reshape(-1).copy()
    y = np.broadcast_to((cy + sy).astype(np.float32), shape).reshape(-1).copy()
    z = np.broadcast_to((cz + sz).astype(np.float32), shape).reshape(-1).copy()
    if spec.nonstab:
        n = spec.nonstab
        rng = np.random.default_rng(seed)
        for arr, dd in ((x, d[0]), (y, d[1]), (z, d[2])):
            r = rng.integers(0, 2 * n + 1, size=arr.size, dtype=np.int32)
            jit = ((r - n).astype(np.float32) / np.float32(n)) * np.float32(spec.jitter * dd)
            arr += jit
    return x, y, z


def markers_in_box(spec: ModelSpec, lo, hi):
    """Indices of the markers of all cells overlapping the box [lo, hi] (cell-major order)."""
    nx, ny, nz = spec.shape
    mpc = int(np.prod(spec.mnum))
    stp = [s / (n - 1) for s, n in zip(spec.size, spec.shape)]
    rng_ = []
    for a in range(3):
        n1 = spec.shape[a] - 1
        c0 = max(0, int(np.floor(lo[a] / stp[a])) - 1)
        c1 = min(n1 - 1, int(np.floor(hi[a] / stp[a])) + 1)
        rng_.append(np.arange(c0, c1 + 1))
    cx, cy, cz = rng_
    cells = (cz[:, None, None] * ((nx - 1) * (ny - 1)) + cx[None, :, None] * (ny - 1) + cy[None, None, :]).reshape(-1)
    return (cells[:, None] * mpc + np.arange(mpc)[None, :]).reshape(-1)


def make_prn(spec: ModelSpec, rocks: dict, types: np.ndarray, marks_xyz, seed: int = 0) -> Prn:
    nx, ny, nz = spec.shape
    x, y, z = marks_xyz
    nmark = x.size
    gx, gy, gz = (_grid(n, s, spec.stretch) for n, s in zip(spec.shape, spec.size))
    rocknum = max(rocks) + 1
    rtab = {f: np.zeros(rocknum) for f in ROCK_FIELDS}
    for t, r in rocks.items():
        for f in ROCK_FIELDS:
            rtab[f][t] = getattr(r, f)
    nodenum = nx * ny * nz
    nodes = {f: np.zeros(nodenum, np.float32) for f in
             ("pr", "vx", "vy", "vz", "ro", "nu", "nxx", "nxy", "nxz", "nyz", "tk", "cp", "et",
              "kt", "ht", "rr")}
    # linear temperature between the top and bottom walls, on nodes and markers
    ty = spec.t_top + (spec.t_bottom - spec.t_top) * gy.astype(np.float64) / spec.size[1]
    nodes["tk"][:] = np.broadcast_to(ty[None, None, :], (nz, nx, ny)).reshape(-1)
    mk = spec.t_top + (spec.t_bottom - spec.t_top) * y.astype(np.float64) / spec.size[1]
    marks = {f: np.zeros(nmark, np.float32) for f in
             ("x", "y", "z", "k", "w", "d", "v", "e", "ex", "ft", "rr", "rn")}
    marks["x"], marks["y"], marks["z"] = x, y, z
    marks["k"] = mk.astype(np.float32)
    marks["t"] = types.astype(np.int8)
    bond = expand_bc(free_slip_boxes(nx, ny, nz, spec.t_top, spec.t_bottom), spec.shape, spec.multinum)
    head = dict(xnumx=nx, ynumy=ny, znumz=nz, mnumx=spec.mnum[0], mnumy=spec.mnum[1],
                mnumz=spec.mnum[2], xsize=float(spec.size[0]), ysize=float(spec.size[1]),
                zsize=float(spec.size[2]), pxinit=spec.pinit_cell[0], pyinit=spec.pinit_cell[1],
                pzinit=spec.pinit_cell[2], pinit=spec.pinit, gxkoef=spec.gravity[0],
                gykoef=spec.gravity[1], gzkoef=spec.gravity[2], rocknum=rocknum,
                bondnum=len(bond), marknum=nmark, cycle=0, timesum_yr=0.0, gridcur=0.0, gridtot=0.0)
    return Prn(head, rtab, nodes, gx, gy, gz, bond, marks)


def write_init_t3c(path, spec: ModelSpec, rocks: dict, background: int, bodies, boxes, out_name="init0.prn") -> None:
    """Write the model as the reference's ``init.t3c`` (read by ``in3mg.c:64-956``), so that the
    reference's own initial-condition program builds the same first ``.prn`` as ``make_prn``:

    * grid parameters and marker jitter (``in3mg.c:69-91``; ``spec.nonstab`` = 0 places the
      markers on the regular sub-grid, the reference's jitter draws ``rand()``),
    * no data file to reload, the output file ``out_name`` (binary),
    * the rock table, one row of the 24 columns of ``ROCK_FIELDS`` per type (``in3mg.c:201-236``),
    * the boundary-condition boxes ``boxes`` (``BcBox``; ``in3mg.c:242-300``) with absolute node
      indices,
    * the rock bodies: first a box of rock ``background`` around the whole model (a marker in no
      body keeps type 0 in the reference), then ``bodies`` in order (``abi.Body`` records as
      ``i3g_init_markers`` takes them: shape 0 box ``n``, 1 ellipsoid ``sn``, 2 cylinder ``cn``;
      ``in3mg.c:548-797``),
    * one temperature box of type 0 over the model, ``spec.t_top`` at y = 0 and
      ``spec.t_bottom`` at y = ysize (``in3mg.c:801-955``).
    """
    nx, ny, nz = spec.shape
    f = repr
    L = ["/grid_PARAMETERS_DESCRIPTIONS"]
    L += [str(nx), str(ny), str(nz)] + [str(m) for m in spec.mnum]
    L += [f(float(v)) for v in spec.size] + [str(v) for v in spec.pinit_cell]
    L += [f(float(spec.pinit))] + [f(float(g)) for g in spec.gravity] + ["0.0"]
    L += [f"{int(spec.nonstab)} {f(float(spec.jitter))} {f(float(spec.jitter))} {f(float(spec.jitter))}", ""]
    L += ["/MARKERS_TYPES_FILE_NAME_Y(Name)_N(0)", "0", "/DATA_OUTPUT_FILE_NAME____TYPE", f"{out_name} b", ""]
    L += ["/ROCKS_DESCRIPTIONS"]
    for t in sorted(rocks):
        L.append(f"{t} " + " ".join(f(float(getattr(rocks[t], c))) for c in ROCK_FIELDS))
    L += ["~", "/BONDARY_CONDITIONS_DESCRIPTIONS"]
    for b in boxes:
        row = f"{b.var} {b.x0} {b.x1} {b.y0} {b.y1} {b.z0} {b.z1} {f(float(b.c))} {f(float(b.k))}"
        if b.k:
            row += " {} {} {}".format(*b.shift)
        L.append(row + " 0 0")
    L += ["~", "/ROCKS_BOXES_DESCRIPTION"]

    def body_row(tok, ex, e, xs, ys, zs):
        pts = " ".join(f"{f(float(xs[n]))} {f(float(ys[n]))} {f(float(zs[n]))}" for n in range(8))
        return f"{tok} {f(float(ex))} {f(float(e))} {pts}"
    lo, hi = -0.1, 1.1
    L.append(body_row(str(background), 0.0, 0.0, [hi if n & 2 else lo for n in range(8)],
                      [hi if n & 1 else lo for n in range(8)], [hi if n & 4 else lo for n in range(8)]))
    for b in bodies:
        tok = {0: "", 1: "s", 2: "c"}[b.shape] + str(b.rock)
        L.append(body_row(tok, b.ex, b.e, list(b.x), list(b.y), list(b.z)))
    L += ["~", "/TEMPERATURE_BOXES_TYPE_x0_x2_y0_y1_y2_y3_z0_x5_x7_y4_y5_y6_y7_z7_T0..T7"]
    tt, tb = f(float(spec.t_top)), f(float(spec.t_bottom))
    L.append("0 0 1 0 1 0 1 0 0 1 0 1 0 1 1 " + " ".join([tt, tb] * 4))
    L += ["~", ""]
    with open(path, "w") as fh:
        fh.write("\n".join(L))


# ---------------------------------------------------------------------------------------
# Named workloads
# ---------------------------------------------------------------------------------------
MATRIX, SPHERE = 2, 3
INCLUSION_TYPES = (3, 4, 5, 6, 9, 10, 11, 12, 13, 14, 15, 19)


def sinking_sphere(n=33, size_km=100.0, mnum=3, multinum=2, seed=1, radius_km=20.0, stretch=0.0,
                   sphere_rho=3400.0, centre_frac=(0.5, 0.5, 0.5), plastic=None, nonstab=100):
    """Plain sinking sphere: eta 1e23 / rho 3400 sphere in eta 1e21 / rho 3300 matrix,
    g = 10 along the vertical, free slip, linear T 273 -> 1573 K, k = 3, cp = 1000.

    ``stretch`` makes the grid lines non-uniform (see ``_grid``); ``plastic = (a, b)`` gives the
    matrix Drucker-Prager yielding sigma_y = a + b P (rock columns a0 = a1 = a, b0 = b1 = b,
    viscalc's brittle branch, mark3mg.c:1148-1198); ``nonstab = 0`` leaves the markers on the
    regular sub-grid."""
    L = size_km * 1e3
    spec = ModelSpec(shape=(n, n, n), size=(L, L, L), mnum=(mnum,) * 3, multinum=multinum, stretch=stretch,
                     nonstab=nonstab)
    xyz = build_markers(spec, seed)
    x, y, z = (a.astype(np.float64) for a in xyz)
    c = [f * L for f in centre_frac]
    r = np.sqrt((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2)
    types = np.where(r <= radius_km * 1e3, SPHERE, MATRIX)
    mat = Rock(nu=1e21, ro=3300.0)
    if plastic:
        a, b = plastic
        mat = dataclasses.replace(mat, a0=a, a1=a, b0=b, b1=b, e0=0.0, e1=1.0)
    rocks = {MATRIX: mat, SPHERE: Rock(nu=1e23, ro=sphere_rho)}
    return make_prn(spec, rocks, types, xyz, seed), spec


def random_inclusions(n=129, size_km=200.0, mnum=3, multinum=4, seed=7, count=100,
                      r_km=(2.0, 8.0), rho=(3250.0, 3450.0), contrast=None,
                      arrhenius=True, activation=5e5, eta_ref=1e21, t_ref=923.0, nonstab=100):
    """Random spherical inclusions in an Arrhenius matrix.

    Inclusion centres, radii and densities are seeded; densities (and, when ``contrast``
    is given, log-uniform viscosity contrasts up to ``contrast``) are binned into at most
    12 rock types because the reference keeps rock properties per type.  ``nonstab = 0`` leaves
    the markers on the regular sub-grid."""
    L = size_km * 1e3
    spec = ModelSpec(shape=(n, n, n), size=(L, L, L), mnum=(mnum,) * 3, multinum=multinum, nonstab=nonstab)
    rng = np.random.default_rng(seed)
    cen = rng.uniform(0.1 * L, 0.9 * L, size=(count, 3))
    rad = rng.uniform(r_km[0] * 1e3, r_km[1] * 1e3, size=count)
    dens = rng.uniform(rho[0], rho[1], size=count)
    logc = rng.uniform(0.0, np.log10(contrast), size=count) if contrast else np.zeros(count)
    nbin = len(INCLUSION_TYPES)
    # joint bins: density quantile x contrast quantile, at most 12 types
    if contrast:
        nd, nc = 4, 3
    else:
        nd, nc = nbin, 1
    dbin = np.minimum(((dens - rho[0]) / (rho[1] - rho[0]) * nd).astype(int), nd - 1)
    cbin = np.minimum((logc / max(np.log10(contrast), 1e-30) * nc).astype(int), nc - 1) if contrast else np.zeros(count, int)
    tbin = dbin * nc + cbin
    A = eta_ref / np.exp(activation / (8.314 * t_ref)) if arrhenius else eta_ref
    mat = Rock(nu=A, dh=activation if arrhenius else 0.0, mm=1.0, n0=1e18, n1=1e24, ro=3300.0)
    rocks = {MATRIX: mat}
    for b in range(nd * nc):
        sel = tbin == b
        d_mean = dens[sel].mean() if sel.any() else rho[0] + (b // nc + 0.5) * (rho[1] - rho[0]) / nd
        c_mean = 10 ** logc[sel].mean() if (sel.any() and contrast) else (
            10 ** ((b % nc + 0.5) * np.log10(contrast) / nc) if contrast else 1.0)
        rocks[INCLUSION_TYPES[b]] = dataclasses.replace(mat, nu=A * c_mean, ro=float(d_mean))
    xyz = build_markers(spec, seed)
    x, y, z = xyz
    types = np.full(x.size, MATRIX, np.int8)
    for i in range(count):
        r = rad[i]
        idx = markers_in_box(spec, cen[i] - r, cen[i] + r)
        d2 = ((x[idx] - cen[i, 0]) ** 2 + (y[idx] - cen[i, 1]) ** 2 + (z[idx] - cen[i, 2]) ** 2)
        types[idx[d2 <= r * r]] = INCLUSION_TYPES[tbin[i]]
    spec = dataclasses.replace(spec, spheres=tuple((INCLUSION_TYPES[tbin[i]], tuple(float(v) for v in cen[i]),
                                                    float(rad[i])) for i in range(count)))
    return make_prn(spec, rocks, types, xyz, seed), spec


LITHO, SLAB, WEAK = 3, 4, 5


def subduction(nx=257, ny=129, nz=257, size_km=(1000.0, 500.0, 1000.0), mnum=3, multinum=4, seed=11,
               litho_km=100.0, weak_km=10.0, dip_deg=45.0, trench_frac=0.35, slab_depth_km=300.0,
               cohesion=1e7, friction=0.6, mantle_eta=(1e19, 1e22), activation=3e5):
    """Visco-plastic subduction-like model (x and z horizontal, y vertical and downward).

    * lithosphere: the top ``litho_km``, eta 1e24, rho 3300, Drucker-Prager yielding
      sigma_y = cohesion + friction * P (viscalc's brittle branch, mark3mg.c:1148-1198);
    * slab: a lithosphere-thick plate dipping at ``dip_deg`` from the trench at
      x = ``trench_frac`` * xsize down to ``slab_depth_km``, rho 3350 (+50), eta 1e24, yielding;
    * weak layer: ``weak_km`` on top of the slab and along the trench, eta 1e19;
    * mantle: Arrhenius eta = A exp(E / RT) (viscalc branch B, mark3mg.c:1281-1299) with E =
      ``activation``, A set so that the mantle's temperatures span ``mantle_eta`` (clamps
      n0 / n1 = ``mantle_eta``), rho 3300;
    * free slip on all walls, T linear from 273 K at the top to 1573 K at the bottom.
    The slab extends over the whole z range (a plate boundary along z)."""
    Lx, Ly, Lz = (s * 1e3 for s in size_km)
    spec = ModelSpec(shape=(nx, ny, nz), size=(Lx, Ly, Lz), mnum=(mnum,) * 3, multinum=multinum)
    xyz = build_markers(spec, seed)
    x, y = (a.astype(np.float64) for a in xyz[:2])
    # Arrhenius prefactor: eta(T_bottom) = mantle_eta[0] at the bottom temperature
    A = mantle_eta[0] / np.exp(activation / (8.314 * spec.t_bottom))
    mantle = Rock(nu=A, dh=activation, mm=1.0, n0=mantle_eta[0], n1=mantle_eta[1], ro=3300.0)
    plastic = dict(a0=cohesion, a1=cohesion, b0=friction, b1=friction, e0=0.0, e1=1.0)
    rocks = {MATRIX: mantle,
             LITHO: Rock(nu=1e24, n0=1e18, n1=1e24, ro=3300.0, **plastic),
             SLAB: Rock(nu=1e24, n0=1e18, n1=1e24, ro=3350.0, **plastic),
             WEAK: Rock(nu=1e19, n0=1e18, n1=1e24, ro=3300.0)}
    H, W = litho_km * 1e3, weak_km * 1e3
    xt = trench_frac * Lx
    t = np.tan(np.radians(dip_deg))
    c = np.cos(np.radians(dip_deg))
    # distance below the slab's upper surface y_s(x) = (x - xt) * tan(dip), measured normal to it
    dn = (y - (x - xt) * t) * c
    in_slab_x = x >= xt
    types = np.full(x.size, MATRIX, np.int8)
    types[y <= H] = LITHO
    slab = in_slab_x & (dn >= 0) & (dn <= H) & (y <= slab_depth_km * 1e3)
    types[slab & (y > H)] = SLAB
    weak = in_slab_x & (dn < 0) & (dn >= -W) & (y <= slab_depth_km * 1e3)
    types[weak] = WEAK
    return make_prn(spec, rocks, types, xyz, seed), spec
