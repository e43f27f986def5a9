"""Generate the golden fixtures from the reference itself (run in the build container, where
the reference sources exist): ``python tests/golden/make_golden.py``.

For each case in cases.py the reference harness (oracle/_ref/ref_harness, built from the
reference sources by oracle/build_ref.sh) is run single-threaded on the seeded model:

* ``prepare``  -> nodal fields and marker viscosities after marker->node averaging,
* ``assemble`` -> SHA-256 of the assembled rows of every multigrid level,
* ``vcycles 5``-> solution vector of every level after five V-cycles,
* ``solve``    -> level-0 solution at relative residual 1e-12.
"""
import hashlib
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle"))

import cases  # noqa: E402
import oracle as O  # noqa: E402
from i3elvis_b200 import config, prn as P  # noqa: E402


MARKER_CASES = ("sphere13",)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def make(name):
    p0, mode = cases.build(name)
    with tempfile.TemporaryDirectory() as d:
        P.write_prn(os.path.join(d, "in0.prn"), p0)
        config.write_mode(os.path.join(d, "mode.t3c"), mode)
        config.write_file_t3c(os.path.join(d, "file.t3c"), 0)
        O.run_reference(d, "prepare", "prep.prn")
        prep = P.read_prn(os.path.join(d, "prep.prn"))
        mode.infile = "prep.prn"
        config.write_mode(os.path.join(d, "mode.t3c"), mode)
        O.run_reference(d, "assemble", "a")
        csr = O.read_csr(os.path.join(d, "a.csr"))
        O.run_reference(d, "vcycles", 5, "v")
        vsol, vhist = O.read_sol(os.path.join(d, "v.sol"))
        info = O.run_reference(d, "solve", 1e-12, 3000, "s")
        ssol, shist = O.read_sol(os.path.join(d, "s.sol"))
        extra = {}
        digests = {}
        if name in MARKER_CASES:
            # reference vpiterate at its own (absolute) tolerance, then movemark + ronurecalc
            O.run_reference(d, "stokes", "m")
            flds = O.read_fields(os.path.join(d, "m.fields"))
            O.run_reference(d, "mover2n", repr(flds["timestep"]), "m")
            mk = O.read_marks(os.path.join(d, "m.marks"))
            nd = O.read_nodes(os.path.join(d, "m.nodes"))
            extra = dict(fld_pr=flds["pr"], fld=np.stack([flds[f] for f in O.FIELD_NAMES]),
                         fld_dt=np.array([flds["timestep"]]),
                         mk=np.stack([mk[f] for f in O.MARK_NAMES]), mk_t=mk["t"],
                         r2n=np.stack([nd[f] for f in O.NODE_NAMES]))
            # the reference's own titerate (absolute HEATMIN, evaluated on FP32 temperatures)
            O.run_reference(d, "titerate", repr(flds["timestep"]), "m", timeout=600)
            # and its heat rows solved tightly in FP64 (relative residual 1e-13)
            hinfo = O.run_reference(d, "heat", repr(flds["timestep"]), 1e-13, 5000, "h", timeout=600)
            hc = O.read_csr(os.path.join(d, "h.csr"))
            hsol, _ = O.read_sol(os.path.join(d, "h.sol"))
            digests["heat"] = dict(counts=sha(np.diff(hc["indptr"]).astype(np.int64)), cols=sha(hc["col"].astype(np.int64)),
                                   vals=sha(hc["val"]), rhs=sha(hc["rhs"]), info=hinfo)
            hm = O.read_marks(os.path.join(d, "m.marks"))
            hn = O.read_nodes(os.path.join(d, "m.nodes"))
            extra.update(heat_tk=hn["tk"], heat_mk=hm["k"], heat_sol=hsol)
    sizes = cases.level_sizes(p0, mode.multinum)
    offs = np.concatenate([[0], np.cumsum(sizes)]) * 4
    counts = np.diff(csr["indptr"])
    for l in range(len(sizes)):
        a, b = csr["indptr"][offs[l]], csr["indptr"][offs[l + 1]]
        digests[f"L{l}"] = dict(counts=sha(counts[offs[l]:offs[l + 1]].astype(np.int64)),
                                cols=sha(csr["col"][a:b].astype(np.int64)), vals=sha(csr["val"][a:b]))
    digests["rhs0"] = sha(csr["rhs"][:offs[1]])
    out = dict(nodes=np.stack([prep.nodes[f] for f in P.NODE_FIELDS]), markv=prep.marks["v"],
               vcyc_sol=vsol, vcyc_hist=vhist, solve_sol=ssol, solve_hist=shist, **extra)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    with open(os.path.join(HERE, f"{name}.json"), "w") as fh:
        json.dump(dict(case=cases.CASES[name], csr_sha256=digests, solve=info), fh, indent=1)
    print(name, "ok", info)


if __name__ == "__main__":
    for name in (sys.argv[1:] or cases.CASES):
        make(name)
