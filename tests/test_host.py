"""The C host loop (host/i3g): .prn and mode.t3c handling against the Python mirror, and a
GPU run of the program against runtime.run on the same run directory."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import cases
from i3elvis_b200 import abi, config, prn as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST = os.path.join(ROOT, "i3elvis_b200", "host", "i3g")


def _host():
    if not os.path.exists(HOST):
        from i3elvis_b200 import build
        build.build()
    return HOST


def _dump(path):
    out = subprocess.run([_host(), "-dump-mode", path], capture_output=True, text=True, check=True).stdout
    d, files = {}, []
    for line in out.splitlines():
        k, _, v = line.partition(" ")
        if k == "file":
            files.append(v.split())
        else:
            d[k] = v
    return d, files


@pytest.mark.parametrize("name", ["sphere13", "sphere17"])
def test_mode_parser_matches_python(tmp_path, name):
    _, mode = cases.build(name)
    mode.files.append(config.OutFile("second.prn", cyc0max=3, maxxystep=12.5, p1koef2=0.25, multstp=7))
    path = str(tmp_path / "mode.t3c")
    config.write_mode(path, mode)
    d, files = _dump(path)
    m = config.read_mode(path)
    par = abi.make_params(m)
    assert d["infile"] == m.infile and int(d["nfiles"]) == len(m.files)
    assert int(d["filesjob"]) == m.filesjob and int(d["cyc1max"]) == m.cyc1max
    for k in ("printmod", "movemod", "tempmod", "markmod", "gridmod", "outgrid", "densimod", "multicyc",
              "viscmod", "multicyct", "multittt0", "frictyn", "adiabyn"):
        assert int(d[k]) == getattr(par, k), k
    assert int(d["multinum"]) == par.multimax
    for k in ("stp100", "eroslev", "sedilev", "waterlev", "DIVVMIN", "STOKSMIN", "DIVVMAX", "STOKSMAX",
              "p0koef", "p1koef", "p2koef", "v0koef", "v1koef", "nubeg", "nuend", "nukoef", "HEATMIN",
              "t0koef", "heatdif", "zdeep", "vdeep", "tdeep", "nudeep", "healrate", "teclmin", "teclmax",
              "timebeg", "timeend"):
        assert float(d[k]) == getattr(par, k), k
    nnn = [int(v) for v in d["multinnn"].split()]
    assert nnn == list(m.multinnn[0]) + list(m.multinnn[1])
    for row, f in zip(files, m.files):
        fp = abi.make_file_params(f)
        assert row[0] == f.name and int(row[1]) == fp.cyc0max
        vals = [float(v) for v in row[2:13]]
        assert vals == [fp.maxxystep, fp.maxtkstep, fp.maxtmstep, fp.nubeg, fp.nuend, fp.p0koef, fp.p1koef,
                        fp.p2koef, fp.p0koef2, fp.p1koef2, fp.p2koef2]
        assert [int(v) for v in row[13:]] == [fp.multinum, fp.multstp, fp.multinum2]


def test_prn_roundtrip_matches_python_writer(tmp_path):
    p, _ = cases.build("sphere13")
    src = str(tmp_path / "in.prn")
    P.write_prn(src, p)
    c_out = str(tmp_path / "c.prn")
    subprocess.run([_host(), "-roundtrip", src, c_out], check=True)
    py_out = str(tmp_path / "py.prn")
    P.write_prn(py_out, abi.ModelBuffers(P.read_prn(src)).to_prn())
    a, b = open(c_out, "rb").read(), open(py_out, "rb").read()
    assert len(a) == len(b) and a == b


def test_prn_reader_rejects_truncated_file(tmp_path):
    p, _ = cases.build("sphere13")
    src = str(tmp_path / "in.prn")
    P.write_prn(src, p)
    raw = open(src, "rb").read()
    bad = str(tmp_path / "bad.prn")
    with open(bad, "wb") as fh:
        fh.write(raw[: len(raw) - 30])
    r = subprocess.run([_host(), "-roundtrip", bad, str(tmp_path / "o.prn")], capture_output=True, text=True)
    assert r.returncode != 0 and "truncated" in r.stderr


def _rundir(path, name, steps):
    """A run directory holding a prepared model (node fields from the reference's marker->node
    pass), like the .prn files the reference's initial-condition program writes."""
    from conftest import golden
    p, mode, _ = golden(name)
    mode.files[0].cyc0max = steps
    mode.infile = "in0.prn"
    P.write_prn(os.path.join(path, "in0.prn"), p)
    config.write_mode(os.path.join(path, "mode.t3c"), mode)
    config.write_file_t3c(os.path.join(path, "file.t3c"), 0)
    return mode


@pytest.mark.gpu
def test_host_program_matches_python_loop(tmp_path):
    from i3elvis_b200 import runtime
    a, b = tmp_path / "c", tmp_path / "py"
    a.mkdir(); b.mkdir()
    mode = _rundir(str(a), "sphere13", 2)
    _rundir(str(b), "sphere13", 2)
    r = subprocess.run([_host(), "-rtol", "1e-8"], cwd=str(a), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    runtime.run(str(b), stokes_rtol=1e-8)
    name = mode.files[0].name
    pc, pp = P.read_prn(str(a / name)), P.read_prn(str(b / name))
    assert open(str(a / "file.t3c")).read() == open(str(b / "file.t3c")).read() == "1 \n"
    assert pc.head == pp.head
    for f in P.NODE_FIELDS:
        np.testing.assert_allclose(pc.nodes[f], pp.nodes[f], rtol=1e-5, atol=1e-30, err_msg=f)
    for f in ("x", "y", "z", "k"):
        np.testing.assert_allclose(pc.marks[f], pp.marks[f], rtol=1e-6, err_msg=f)
    assert np.array_equal(pc.marks["t"], pp.marks["t"])
