"""``mode.t3c`` / ``file.t3c`` run configuration.

The token grammar is the reference's (``ffscanf`` in ``load3mg.c:1102-1127``): the file is
split on whitespace, tokens that begin with ``/`` are skipped, and each value token is read
with C ``atoi``/``atof`` prefix semantics, so ``1e-04-DIVVMIN`` reads as ``1e-4``.  Fields
are consumed in the order of ``loadconf`` (``load3mg.c:2-170``).
"""
from __future__ import annotations

import dataclasses
import re

from .prn import YEAR

_FLOAT_RE = re.compile(r"^[+-]?(\d+\.?\d*|\.\d+)([eE][+-]?\d+)?")
_INT_RE = re.compile(r"^[+-]?\d+")


def c_atof(tok: str) -> float:
    m = _FLOAT_RE.match(tok.strip())
    return float(m.group(0)) if m else 0.0


def c_atoi(tok: str) -> int:
    m = _INT_RE.match(tok.strip())
    return int(m.group(0)) if m else 0


@dataclasses.dataclass
class OutFile:
    """One row of the output-file table (``load3mg.c:25-58``)."""
    name: str
    cyc0max: int = 1          # time steps before this file is written
    maxxystep: float = 0.0    # CFL distance limit per step, m
    maxtkstep: float = 25.0   # temperature change limit per step, K
    maxtmstep_yr: float = 1e4
    nubeg: float = 1e18
    nuend: float = 1e24
    p0koef: float = 0.71
    p1koef: float = 1.0
    p2koef: float = 0.0
    p0koef2: float = 0.71
    p1koef2: float = 1.0
    p2koef2: float = 0.0
    multinum: int = 2
    multstp: int = 1000000    # outer iteration after which multinum2/p*koef2 apply
    multinum2: int = 2


@dataclasses.dataclass
class Mode:
    """All of ``mode.t3c`` that ``loadconf`` reads, with the shipped defaults
    (reference ``mode.t3c`` general, V_P and T blocks)."""
    infile: str = "in0.prn"
    files: list = dataclasses.field(default_factory=list)
    printmod: int = 0
    movemod: int = 1
    tempmod: int = 1
    markmod: int = 2
    gridmod: int = 1
    outgrid: int = 2
    densimod: int = 1
    stp100: float = 13500.0
    filesjob: int = 1000
    eroslev: float = -1e30
    sedilev: float = 1e30
    waterlev: float = -1e30
    cyc1max: int = 30000
    DIVVMIN: float = 1e-4
    STOKSMIN: float = 5e1
    DIVVMAX: float = 1e-8
    STOKSMAX: float = 1e-4
    multinum: int = 2
    multicyc: int = 4
    multinnn: tuple = ((8, 16, 16), (8, 16, 64))
    p0koef: float = 0.3
    p1koef: float = 0.1
    p2koef: float = 0.0
    v0koef: float = 0.7
    v1koef: float = 0.7
    nubeg: float = 1e18
    nuend: float = 1e25
    nukoef: float = 0.0
    viscmod: int = 0
    spheryn: int = 0
    cyc2max: int = 2500
    HEATMIN: float = 1e-3
    multinumt: int = 0
    multicyct: int = 1
    multittt: tuple = ((30,), (0,))
    t0koef: float = 1.0
    t1koef: float = 1.0
    heatdif: float = 1.0
    frictyn: int = 0
    adiabyn: int = 0
    water: tuple = (97300000.0, 75000, -3e-09, -3e-09, 1e-1, 1942.0, 100.0, 0.0, 760000.0,
                    770000.0, 1e21, 2e3, 2e3, 2e3, 100000, 4e4, 923, -0.0, 20000, 10000,
                    2.0, 10000.0, 873.15, 1.0e-15, 1e-2, 5e-1, 1e10, 673, 873)
    xvolc: float = 0.2
    xtkplut: float = 0.5
    timebeg_yr: float = 10e9
    timeend_yr: float = 15e9
    tempbeg: float = 2021.0
    convend_yr: float = 1e5

    WATER_NAMES = ("tkpor", "zmpor", "vyfluid", "vymelt", "dmwamin", "tdeep", "dtdeep", "drdeep",
                   "zdeep", "vdeep", "nudeep", "dxwater", "dywater", "dzwater", "dserp", "yserp",
                   "tserp", "lambmlt", "ydike", "dydike", "nusseltno", "circdepth", "circtemp",
                   "healrate", "meltmin", "maxwater", "maxpmelt", "teclmin", "teclmax")

    def water_param(self, name: str) -> float:
        return float(self.water[self.WATER_NAMES.index(name)])


def write_mode(path, m: Mode) -> None:
    """Write ``m`` as a ``mode.t3c`` that the reference's ``loadconf`` reads back."""
    L = ["/loadFILE_TYPE", f"{m.infile} b", "",
         "/SAVEFILE_TYPE_cyc0max_maxxystep_maxtkstep_maxtmstep_nubeg_nuend_p0k1_p1k1_p2k1__p0k2_p1k2_p2k2__multinum1_stp1_multinum2"]
    for f in m.files:
        L.append(f"{f.name} b {f.cyc0max} {f.maxxystep!r} {f.maxtkstep!r} {f.maxtmstep_yr!r} "
                 f"{f.nubeg!r} {f.nuend!r} {f.p0koef!r} {f.p1koef!r} {f.p2koef!r} "
                 f"{f.p0koef2!r} {f.p1koef2!r} {f.p2koef2!r} {f.multinum} {f.multstp} {f.multinum2}")
    L += ["~", "", "/GENERAL_PARAMETERS"]
    for k in ("printmod", "movemod", "tempmod", "markmod", "gridmod", "outgrid", "densimod",
              "stp100", "filesjob", "eroslev", "sedilev", "waterlev", "cyc1max", "DIVVMIN",
              "STOKSMIN", "DIVVMAX", "STOKSMAX", "multinum", "multicyc"):
        L.append(f"{getattr(m, k)!r}-{k}")
    assert len(m.multinnn[0]) == m.multinum + 1 and len(m.multinnn[1]) == m.multinum + 1
    L.append(" ".join(str(int(v)) for v in m.multinnn[0]))
    L.append(" ".join(str(int(v)) for v in m.multinnn[1]))
    for k in ("p0koef", "p1koef", "p2koef", "v0koef", "v1koef", "nubeg", "nuend", "nukoef",
              "viscmod", "spheryn", "cyc2max", "HEATMIN", "multinumt", "multicyct"):
        L.append(f"{getattr(m, k)!r}-{k}")
    assert len(m.multittt[0]) == m.multinumt + 1 and len(m.multittt[1]) == m.multinumt + 1
    L.append(" ".join(str(int(v)) for v in m.multittt[0]))
    L.append(" ".join(str(int(v)) for v in m.multittt[1]))
    for k in ("t0koef", "t1koef", "heatdif", "frictyn", "adiabyn"):
        L.append(f"{getattr(m, k)!r}-{k}")
    for name, v in zip(Mode.WATER_NAMES, m.water):
        L.append(f"{v!r}-{name}")
    for k in ("xvolc", "xtkplut", "timebeg_yr", "timeend_yr", "tempbeg", "convend_yr"):
        L.append(f"{getattr(m, k)!r}-{k}")
    L.append("")
    with open(path, "w") as fh:
        fh.write("\n".join(L))


def _tokens(path):
    with open(path) as fh:
        for tok in fh.read().split():
            if tok and tok[0] != "/":
                yield tok


def read_mode(path) -> Mode:
    """Parse ``mode.t3c`` exactly in ``loadconf`` order."""
    it = _tokens(path)
    nxt = lambda: next(it)
    m = Mode()
    m.infile = nxt(); nxt()
    m.files = []
    tok = nxt()
    while tok[0] != "~":
        f = OutFile(tok)
        nxt()
        f.cyc0max = c_atoi(nxt())
        f.maxxystep, f.maxtkstep, f.maxtmstep_yr = c_atof(nxt()), c_atof(nxt()), c_atof(nxt())
        f.nubeg, f.nuend = c_atof(nxt()), c_atof(nxt())
        f.p0koef, f.p1koef, f.p2koef = c_atof(nxt()), c_atof(nxt()), c_atof(nxt())
        f.p0koef2, f.p1koef2, f.p2koef2 = c_atof(nxt()), c_atof(nxt()), c_atof(nxt())
        f.multinum, f.multstp, f.multinum2 = c_atoi(nxt()), c_atoi(nxt()), c_atoi(nxt())
        m.files.append(f)
        tok = nxt()
    for k, conv in (("printmod", c_atoi), ("movemod", c_atoi), ("tempmod", c_atoi), ("markmod", c_atoi),
                    ("gridmod", c_atoi), ("outgrid", c_atoi), ("densimod", c_atoi), ("stp100", c_atof),
                    ("filesjob", c_atoi), ("eroslev", c_atof), ("sedilev", c_atof), ("waterlev", c_atof),
                    ("cyc1max", c_atoi), ("DIVVMIN", c_atof), ("STOKSMIN", c_atof), ("DIVVMAX", c_atof),
                    ("STOKSMAX", c_atof), ("multinum", c_atoi), ("multicyc", c_atoi)):
        setattr(m, k, conv(nxt()))
    a = tuple(c_atoi(nxt()) for _ in range(m.multinum + 1))
    b = tuple(c_atoi(nxt()) for _ in range(m.multinum + 1))
    m.multinnn = (a, b)
    for k, conv in (("p0koef", c_atof), ("p1koef", c_atof), ("p2koef", c_atof), ("v0koef", c_atof),
                    ("v1koef", c_atof), ("nubeg", c_atof), ("nuend", c_atof), ("nukoef", c_atof),
                    ("viscmod", c_atoi), ("spheryn", c_atoi), ("cyc2max", c_atoi), ("HEATMIN", c_atof),
                    ("multinumt", c_atoi), ("multicyct", c_atoi)):
        setattr(m, k, conv(nxt()))
    a = tuple(c_atoi(nxt()) for _ in range(m.multinumt + 1))
    b = tuple(c_atoi(nxt()) for _ in range(m.multinumt + 1))
    m.multittt = (a, b)
    m.t0koef, m.t1koef, m.heatdif = c_atof(nxt()), c_atof(nxt()), c_atof(nxt())
    m.frictyn, m.adiabyn = int(c_atof(nxt())), int(c_atof(nxt()))
    m.water = tuple(c_atof(nxt()) for _ in Mode.WATER_NAMES)
    m.xvolc, m.xtkplut = c_atof(nxt()), c_atof(nxt())
    m.timebeg_yr, m.timeend_yr, m.tempbeg = c_atof(nxt()), c_atof(nxt()), c_atof(nxt())
    m.convend_yr = c_atof(nxt())
    return m


def write_file_t3c(path, index: int) -> None:
    """``file.t3c`` holds the 1-based index of the next output file (``load3mg.c:1066-1068``)."""
    with open(path, "w") as fh:
        fh.write(f"{index} \n")


def maxtmstep_seconds(f: OutFile) -> float:
    return f.maxtmstep_yr * YEAR
