"""The reference's initial-condition program against this package's model builder, on CPU.

``model.write_init_t3c`` writes a model as the reference's ``init.t3c``; the reference's own
``in3mg`` (compiled from its sources into oracle/_ref by oracle/build_ref.sh) turns it into the
first ``.prn`` of a run.  These tests check that

* the benchmark models' builder (``model.sinking_sphere`` -> ``make_prn`` with ``expand_bc``),
  followed by the reference's initial passes (the harness's ``prepare``, in3mg.c:990-1031),
  gives that very file: header, rock table, grid lines, every boundary record, every nodal and
  marker field, byte for byte;
* the marker restatement that the GPU's ``i3g_init_markers`` is tested against
  (oracle/init_ref.py) places markers and assigns bodies (bilinear boxes, ellipsoid shells,
  cylinders) and their ``markex``/``marke`` exactly as ``in3mg`` does;
* a ``.prn`` written by ``in3mg`` reads and writes back byte for byte through this package's
  Python and C readers.

The reference jitters markers with ``rand()``; the models here use the regular sub-grid
(``nonstab = 0``), where placement is deterministic.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
IN3MG = os.path.join(ROOT, "oracle", "_ref", "in3mg")
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")

pytestmark = pytest.mark.skipif(not (os.path.exists(IN3MG) and os.path.exists(HARNESS)),
                                reason="reference programs not built (oracle/build_ref.sh)")


def _in3mg(d, spec, rocks, background, bodies, boxes, mode):
    from i3elvis_b200 import config, model as M, prn as P
    M.write_init_t3c(os.path.join(d, "init.t3c"), spec, rocks, background, bodies, boxes)
    config.write_mode(os.path.join(d, "mode.t3c"), mode)
    config.write_file_t3c(os.path.join(d, "file.t3c"), 0)
    r = subprocess.run([IN3MG], cwd=d, capture_output=True, text=True, timeout=3600, stdin=subprocess.DEVNULL,
                       env=dict(os.environ, OMP_NUM_THREADS="1"))
    assert r.returncode == 0 and "OK!" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]
    return os.path.join(d, "init0.prn"), P.read_prn(os.path.join(d, "init0.prn"))


def _rocks_of(p, types):
    from i3elvis_b200 import model as M, prn as P
    return {t: M.Rock(**{f: float(p.rocks[f][t]) for f in P.ROCK_FIELDS}) for t in types}


@pytest.mark.parametrize("case", ["sphere17", "dp17"])
def test_model_builder_gives_the_reference_first_prn(tmp_path, case):
    """The 17^3 sinking sphere (4 multigrid levels), and the one of the Drucker-Prager fixture
    (yielding matrix, dense sphere): builder + the reference's initial passes == the reference's
    initial-condition program, byte for byte."""
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import cases
    import oracle as O
    from i3elvis_b200 import abi, config, model as M, prn as P
    _, mode = cases.build(case)
    c = cases.CASES[case]
    n, L, R = 17, 100e3, 20e3
    ours, spec = M.sinking_sphere(n=n, mnum=2, multinum=mode.multinum, seed=c["seed"], radius_km=R / 1e3,
                                  plastic=c.get("plastic"), sphere_rho=c.get("sphere_rho", 3400.0),
                                  centre_frac=c.get("centre", (0.5, 0.5, 0.5)), nonstab=0)
    centre = c.get("centre", (0.5, 0.5, 0.5))
    bodies = [abi.sphere_body(M.SPHERE, centre, (R / L,) * 3, 0.0, 1.0)]
    boxes = M.free_slip_boxes(n, n, n, spec.t_top, spec.t_bottom)
    a = tmp_path / "in3mg"
    a.mkdir()
    ref_path, ref = _in3mg(str(a), spec, _rocks_of(ours, (M.MATRIX, M.SPHERE)), M.MATRIX, bodies, boxes, mode)
    assert np.count_nonzero(ref.marks["t"] == M.SPHERE) > 1000
    b = tmp_path / "ours"
    b.mkdir()
    P.write_prn(str(b / "in0.prn"), ours)
    mode.infile = "in0.prn"
    config.write_mode(str(b / "mode.t3c"), mode)
    config.write_file_t3c(str(b / "file.t3c"), 0)
    O.run_reference(str(b), "prepare", "prep.prn")
    prep = P.read_prn(str(b / "prep.prn"))
    # field by field first, for a readable failure
    assert ref.head == prep.head
    for f in P.ROCK_FIELDS:
        assert np.array_equal(ref.rocks[f], prep.rocks[f]), f
    for g in ("gx", "gy", "gz"):
        assert np.array_equal(getattr(ref, g), getattr(prep, g)), g
    assert len(ref.bond) == len(prep.bond) == len(ours.bond)
    for f in ref.bond.dtype.names:
        assert np.array_equal(ref.bond[f], ours.bond[f]), f
    for f in P.NODE_FIELDS:
        assert np.array_equal(ref.nodes[f], prep.nodes[f]), f
    for f in P.MARK_FIELDS + ("t",):
        assert np.array_equal(ref.marks[f], prep.marks[f]), f
    if c.get("plastic"):
        # the Drucker-Prager columns (a0, a1, b0, b1) came through init.t3c into the compared table
        a, bb = c["plastic"]
        assert ref.rocks["a0"][M.MATRIX] == ref.rocks["a1"][M.MATRIX] == a
        assert ref.rocks["b0"][M.MATRIX] == ref.rocks["b1"][M.MATRIX] == bb
    with open(ref_path, "rb") as fa, open(str(b / "prep.prn"), "rb") as fb:
        assert fa.read() == fb.read()


def _full_case():
    """The benchmark's own configuration (129^3 nodes, 27 markers per cell = 56.6 M markers, 100
    inclusions, four coarse levels), without jitter: minutes of CPU time and about 12 GB of memory,
    so only with I3G_IN3MG_FULL=1."""
    sys.path.insert(0, ROOT)
    import bench
    w = bench.WORKLOADS["incl129"]
    return pytest.param(w["n"], w["mnum"], w["multinum"], w["seed"], w["count"], (2.0, 8.0), id="incl129",
                        marks=pytest.mark.skipif(not os.environ.get("I3G_IN3MG_FULL"),
                                                 reason="full-size check: set I3G_IN3MG_FULL=1"))


@pytest.mark.parametrize("n,mnum,multinum,seed,count,r_km", [(17, 2, 2, 5, 8, (15.0, 35.0)),
                                                             (33, 2, 3, 7, 100, (2.0, 8.0)), _full_case()])
def test_inclusion_builder_gives_the_reference_first_prn(tmp_path, n, mnum, multinum, seed, count, r_km):
    """The benchmark's model family (``model.random_inclusions``: Arrhenius matrix, seeded
    spherical inclusions binned into 12 rock types, 200 km cube), at 17^3 with 8 inclusions, at
    33^3 with the benchmark's 100 inclusions of 2-8 km and (opt-in) at the benchmark's full size:
    builder + the reference's initial passes == the reference's initial-condition program, byte
    for byte."""
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import cases
    import oracle as O
    from i3elvis_b200 import abi, config, model as M, prn as P
    _, mode = cases.build("incl17")
    mode.multinum = multinum
    mode.multinnn = (tuple([8] * multinum + [0]), tuple([8] * multinum + [32]))
    mode.files[0].multinum = mode.files[0].multinum2 = multinum
    ours, spec = M.random_inclusions(n=n, size_km=200.0, mnum=mnum, multinum=multinum, seed=seed, count=count,
                                     r_km=r_km, nonstab=0)
    L = spec.size[0]
    assert len(spec.spheres) == count
    bodies = [abi.sphere_body(t, tuple(c / L for c in cen), (r / L,) * 3) for t, cen, r in spec.spheres]
    types = [int(t) for t in np.nonzero(ours.rocks["ro"])[0]]
    a = tmp_path / "in3mg"
    a.mkdir()
    ref_path, ref = _in3mg(str(a), spec, _rocks_of(ours, types), M.MATRIX, bodies,
                           M.free_slip_boxes(n, n, n, spec.t_top, spec.t_bottom), mode)
    assert np.count_nonzero(ref.marks["t"] != M.MATRIX) > 1000
    b = tmp_path / "ours"
    b.mkdir()
    P.write_prn(str(b / "in0.prn"), ours)
    mode.infile = "in0.prn"
    config.write_mode(str(b / "mode.t3c"), mode)
    config.write_file_t3c(str(b / "file.t3c"), 0)
    O.run_reference(str(b), "prepare", "prep.prn")
    prep = P.read_prn(str(b / "prep.prn"))
    assert ref.head == prep.head
    for f in ref.bond.dtype.names:
        assert np.array_equal(ref.bond[f], prep.bond[f]), f
    # Marker temperature: in3mg interpolates its FP32 nodal temperature box to the marker
    # (in3mg.c:960-969), the builder evaluates the same linear profile at the marker; at 129^3
    # (7 % of the markers) the two differ by up to 2 FP32 roundings, which the Arrhenius
    # viscosity carries into the marker viscosity and the nodal viscosities and stresses (at most
    # 7.1e-6 relative measured).  Everything else is exact; at 17^3 and 33^3 all is.
    t_dep_marks, t_dep_nodes = ("k", "v"), ("nu", "nxx", "nxy", "nxz", "nyz", "tk")
    for f in P.MARK_FIELDS + ("t",):
        if f not in t_dep_marks:
            assert np.array_equal(ref.marks[f], prep.marks[f]), f
    ka = ref.marks["k"]
    assert np.max(np.abs(ka.astype(np.float64) - prep.marks["k"]) / np.spacing(np.abs(ka))) <= 2.0
    va = ref.marks["v"].astype(np.float64)
    assert np.max(np.abs(va - prep.marks["v"]) / np.maximum(np.abs(va), 1e-300)) <= 1e-5
    for f in P.NODE_FIELDS:
        a = ref.nodes[f].astype(np.float64)
        if f in t_dep_nodes:
            assert np.max(np.abs(a - prep.nodes[f]) / np.maximum(np.abs(a), 1e-300)) <= 1e-5, f
        else:
            assert np.array_equal(ref.nodes[f], prep.nodes[f]), f
    if n <= 33:
        with open(ref_path, "rb") as fa, open(str(b / "prep.prn"), "rb") as fb:
            assert fa.read() == fb.read()


def test_marker_restatement_matches_reference_bodies(tmp_path):
    """Box with bilinear faces, ellipsoid shell, cylinder along y, later bodies over earlier ones,
    on a 17 x 13 x 21 grid with 2 x 3 x 2 markers per cell: positions, rock types, markex, marke
    and temperatures of oracle/init_ref.py == the reference's initial-condition program."""
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import cases
    import init_ref
    from i3elvis_b200 import abi, model as M
    _, mode = cases.build("sphere13")          # two multigrid levels below the grid
    shape, size = (17, 13, 21), (120e3, 80e3, 150e3)
    spec = M.ModelSpec(shape=shape, size=size, mnum=(2, 3, 2), multinum=mode.multinum, nonstab=0,
                       t_top=300.0, t_bottom=1600.0)
    rocks = {t: M.Rock(nu=10.0 ** (20 + t % 4), ro=3000.0 + 50 * t) for t in (2, 5, 7, 9, 11)}
    tilted = abi.box_body(5, (0.1, 0.2, 0.15), (0.7, 0.6, 0.8), ex=0.25, e=0.5)
    for c in range(8):                       # lean the x faces with y and the y faces with x
        tilted.x[c] += 0.15 * tilted.y[c]
        tilted.y[c] += 0.1 * tilted.x[c] * tilted.z[c]
    bodies = [tilted,
              abi.sphere_body(7, (0.55, 0.45, 0.5), (0.3, 0.2, 0.25), 0.4, 1.0, ex=1.5, e=0.0),
              abi.sphere_body(9, (0.3, 0.5, 0.6), (0.12, 0.35, 0.1), 0.0, 1.0, cylinder=True, e=2.0),
              abi.box_body(11, (0.6, -0.05, 0.0), (1.05, 0.25, 0.4))]
    boxes = M.free_slip_boxes(*shape, spec.t_top, spec.t_bottom)
    _, ref = _in3mg(str(tmp_path), spec, rocks, 2, bodies, boxes, mode)
    bd = [dict(rock=b.rock, shape=b.shape, x=list(b.x), y=list(b.y), z=list(b.z), ex=b.ex, e=b.e) for b in bodies]
    mk = init_ref.markers(shape, size, spec.mnum, 0, (0.5,) * 3, 0, 2, bd, spec.t_top, spec.t_bottom)
    assert ref.head["marknum"] == mk["x"].size == 16 * 12 * 20 * 12
    for f in ("x", "y", "z", "t", "ex"):
        assert np.array_equal(ref.marks[f], mk[f]), f
    # temperature: the reference interpolates the nodal temperature box to the marker
    # (in3mg.c:960-969, tkcalc1), the restatement evaluates the same linear profile at the
    # marker: equal to one FP32 rounding
    k_ref = ref.marks["k"].astype(np.float64)
    assert np.max(np.abs(k_ref - mk["k"]) / np.spacing(np.abs(ref.marks["k"]))) <= 1.0
    # the file holds marke after the initial passes, whose viscosity computation keeps the
    # yielding state in its sign (mark3mg.c:1647-1658): negative, as none of these rocks yields
    assert np.array_equal(np.abs(ref.marks["e"]), mk["e"])
    assert not np.any(ref.marks["e"] > 0)
    # every body holds markers in the result
    for t in (2, 5, 7, 9, 11):
        assert np.count_nonzero(ref.marks["t"] == t) > 50, t
    # the boundary records of the expansion onto the levels
    ours = M.expand_bc(boxes, shape, mode.multinum)
    for f in ref.bond.dtype.names:
        assert np.array_equal(ref.bond[f], ours[f]), f


def test_reference_prn_reads_and_writes_back(tmp_path):
    """A .prn written by the reference's initial-condition program round-trips byte for byte
    through prn.py and through the C host program's reader and writer."""
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import cases
    from i3elvis_b200 import abi, model as M, prn as P
    _, mode = cases.build("sphere13")
    ours, spec = M.sinking_sphere(n=13, mnum=2, multinum=mode.multinum, nonstab=0)
    path, ref = _in3mg(str(tmp_path), spec, _rocks_of(ours, (M.MATRIX, M.SPHERE)), M.MATRIX,
                       [abi.sphere_body(M.SPHERE, (0.5, 0.5, 0.5), (0.2,) * 3)],
                       M.free_slip_boxes(13, 13, 13, spec.t_top, spec.t_bottom), mode)
    raw = open(path, "rb").read()
    P.write_prn(str(tmp_path / "py.prn"), ref)
    assert open(str(tmp_path / "py.prn"), "rb").read() == raw
    host = os.path.join(ROOT, "i3elvis_b200", "host", "i3g")
    if os.path.exists(host):
        subprocess.run([host, "-roundtrip", path, str(tmp_path / "c.prn")], check=True, timeout=120)
        assert open(str(tmp_path / "c.prn"), "rb").read() == raw
