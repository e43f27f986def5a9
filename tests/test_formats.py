"""File formats: .prn byte round trip and mode.t3c parsing with C atof/atoi semantics."""
import os

import numpy as np
import pytest

from i3elvis_b200 import config, model, prn as P


def test_prn_roundtrip(tmp_path):
    p, _ = model.sinking_sphere(n=9, mnum=2, multinum=1, seed=5)
    f1 = tmp_path / "a.prn"
    P.write_prn(f1, p)
    q = P.read_prn(f1)
    f2 = tmp_path / "b.prn"
    P.write_prn(f2, q)
    assert f1.read_bytes() == f2.read_bytes()
    # 4 size bytes + 176 header + rocks + 64 B/node + grid + 32 B/bond + 49 B/marker
    x, y, z = p.shape
    expect = 4 + 176 + 24 * 8 * p.head["rocknum"] + 64 * x * y * z + 4 * (x + y + z) + 32 * len(p.bond) + 49 * p.marknum
    assert os.path.getsize(f1) == expect


def test_prn_truncated(tmp_path):
    p, _ = model.sinking_sphere(n=9, mnum=1, multinum=1, seed=5)
    f = tmp_path / "a.prn"
    P.write_prn(f, p)
    data = f.read_bytes()
    (tmp_path / "t.prn").write_bytes(data[:-10])
    try:
        P.read_prn(tmp_path / "t.prn")
    except P.PrnFormatError:
        pass
    else:
        raise AssertionError("truncated file accepted")


def test_c_number_prefixes():
    assert config.c_atof("1e-04-DIVVMIN") == 1e-4
    assert config.c_atof("5e+01-STOKSMIN") == 50.0
    assert config.c_atof("0.0e-00-p2koef") == 0.0
    assert config.c_atoi("30000-cyc1max") == 30000
    assert config.c_atof("-3e-09-vyfluid") == -3e-9
    assert config.c_atof("abc") == 0.0


def test_mode_roundtrip(tmp_path):
    m = config.Mode(multinum=3, multinnn=((8, 16, 16, 0), (8, 16, 16, 64)),
                    files=[config.OutFile("o1.prn", maxxystep=123.5, multinum=3, multinum2=2)])
    f = tmp_path / "mode.t3c"
    config.write_mode(f, m)
    r = config.read_mode(f)
    assert r.multinnn == m.multinnn and r.files[0].maxxystep == 123.5 and r.files[0].multinum2 == 2
    assert r.water == m.water and r.HEATMIN == m.HEATMIN


def test_reference_mode_file_parses():
    """The reference's own mode.t3c specimen parses with the loadconf token order (runs where
    I3G_REFERENCE_DIR names a checkout of the reference sources)."""
    ref = os.path.join(os.environ.get("I3G_REFERENCE_DIR", ""), "mode.t3c")
    if not os.environ.get("I3G_REFERENCE_DIR") or not os.path.exists(ref):
        pytest.skip("I3G_REFERENCE_DIR does not name the reference sources")
    m = config.read_mode(ref)
    assert m.multinum == 4 and m.multinnn[1][4] == 64 and m.v0koef == 0.7
    assert len(m.files) > 100 and m.files[0].p0koef == 0.71


def test_level_geometry():
    assert model.level_dims(129, 4) == [129, 67, 36, 20, 12]
    assert model.level_dims(33, 2) == [33, 19, 12]
    g = np.arange(33, dtype=np.float64)
    lv = model.level_coords(g, 2)
    assert list(lv[1][:4]) == [0, 1, 2, 4] and lv[1][-1] == 32 and lv[2][3] == 6


def test_bc_expansion_counts():
    """Every Stokes row of every level is either interior or has a boundary record."""
    p, _ = model.sinking_sphere(n=13, mnum=1, multinum=2, seed=1)
    rows = set(p.bond["row"].tolist())
    nodenum = 13 ** 3
    trows = [r for r in rows if r >= 8 * nodenum]
    assert len(trows) > 0
    # the T rows cover the six faces of level 0
    assert len([r for r in trows if r - 8 * nodenum < nodenum]) == 13 ** 3 - 11 ** 3
