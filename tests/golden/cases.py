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
    "sphere13": dict(kind="sphere", n=13, mnum=2, multinum=2, seed=1),
    # 17^3 sinking sphere, levels 17 -> 11 -> 8 -> 6
    "sphere17": dict(kind="sphere", n=17, mnum=2, multinum=3, seed=3),
    # the CPU-runnable configuration of the benchmark: 100 km cube, 33^3 nodes, 3x3x3 markers
    # per cell (884,736), eta 1e23 / rho 3400 sphere of radius 20 km in eta 1e21 / rho 3300,
    # two coarse levels (33 -> 19 -> 12; the reference's 4-level cycle gives NaN at 33^3)
    "sphere33": dict(kind="sphere", n=33, mnum=3, multinum=2, seed=1, big=True),
    # 17^3, 200 km cube, 8 inclusions in an Arrhenius matrix (E = 500 kJ/mol, eta 1e18-1e24):
    # viscalc's thermally activated branch (mark3mg.c:1281-1299), the benchmark's rheology
    "incl17": dict(kind="incl", n=17, mnum=2, multinum=2, seed=5, count=8, r_km=(15.0, 35.0)),
    # 17^3 sphere below a Drucker-Prager matrix (sigma_y = 1e7 + 0.6 P, mark3mg.c:1148-1198)
    # with a dense sphere near the top so that markers above it yield
    "dp17": dict(kind="sphere", n=17, mnum=2, multinum=2, seed=2, plastic=(1e7, 0.6), sphere_rho=4300.0,
                 centre=(0.5, 0.3, 0.5)),
    # 17^3 sinking sphere on non-uniform grid lines (spacing 0.65 h .. 1.35 h): the binary
    # cell search instead of the uniform-spacing lookup, and stretched stencils
    "stretch17": dict(kind="sphere", n=17, mnum=2, multinum=2, seed=4, stretch=0.35),
}

# cases whose markers go through the reference's Stokes, advection, marker->node and heat steps
MARKER_CASES = ("sphere13", "sphere33", "incl17", "dp17", "stretch17")


def build(name):
    """(Prn, Mode) of a case before the marker->node preparation."""
    c = CASES[name]
    if c["kind"] == "incl":
        prn, spec = model.random_inclusions(n=c["n"], size_km=200.0, mnum=c["mnum"], multinum=c["multinum"],
                                            seed=c["seed"], count=c["count"], r_km=c["r_km"])
        size = 200e3
        nuend = 1e24
    else:
        prn, spec = model.sinking_sphere(n=c["n"], mnum=c["mnum"], multinum=c["multinum"], seed=c["seed"],
                                         stretch=c.get("stretch", 0.0), plastic=c.get("plastic"),
                                         sphere_rho=c.get("sphere_rho", 3400.0),
                                         centre_frac=c.get("centre", (0.5, 0.5, 0.5)))
        size = 100e3
        nuend = 1e25
    mn = c["multinum"]
    mode = config.Mode(
        infile="in0.prn", multinum=mn, multicyc=1,
        multinnn=(tuple([8] * mn + [0]), tuple([8] * mn + [32])),
        p0koef=0.71, p1koef=1.0, v0koef=0.7, v1koef=0.7, nubeg=1e18, nuend=nuend,
        files=[config.OutFile("out1.prn", maxxystep=0.5 * size / (c["n"] - 1), maxtmstep_yr=1e9,
                              nubeg=1e18, nuend=nuend, p0koef=0.71, p1koef=1.0, multinum=mn, multinum2=mn)])
    return prn, mode


def level_sizes(prn, multinum):
    dims = [model.level_dims(n, multinum) for n in prn.shape]
    return [dims[0][l] * dims[1][l] * dims[2][l] for l in range(multinum + 1)]
