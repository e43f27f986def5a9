"""Small seeded models shared by the golden-fixture generator and the tests.

A case is rebuilt deterministically from its parameters (numpy PCG64 streams are stable);
the fixtures store only what the reference computed from it.
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from i3elvis_b200 import config, model  # noqa: E402

CASES = {
    # 13^3 sinking sphere, 2x2x2 markers per cell, levels 13 -> 9 -> 7
    "sphere13": dict(n=13, mnum=2, multinum=2, seed=1),
    # 17^3 sinking sphere, levels 17 -> 11 -> 8 -> 6
    "sphere17": dict(n=17, mnum=2, multinum=3, seed=3),
}


def build(name):
    """(Prn, Mode) of a case before the marker->node preparation."""
    c = CASES[name]
    prn, spec = model.sinking_sphere(n=c["n"], mnum=c["mnum"], multinum=c["multinum"], seed=c["seed"])
    mn = c["multinum"]
    mode = config.Mode(
        infile="in0.prn", multinum=mn, multicyc=1,
        multinnn=(tuple([8] * mn + [0]), tuple([8] * mn + [32])),
        p0koef=0.71, p1koef=1.0, v0koef=0.7, v1koef=0.7, nubeg=1e18, nuend=1e25,
        files=[config.OutFile("out1.prn", maxxystep=0.5 * 100e3 / (c["n"] - 1), maxtmstep_yr=1e9,
                              nubeg=1e18, nuend=1e25, p0koef=0.71, p1koef=1.0, multinum=mn, multinum2=mn)])
    return prn, mode


def level_sizes(prn, multinum):
    dims = [model.level_dims(n, multinum) for n in prn.shape]
    return [dims[0][l] * dims[1][l] * dims[2][l] for l in range(multinum + 1)]
