import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests", "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libi3g.so")


def golden(name):
    """Prepared (Prn, Mode, fixture dict) of a golden case: the seeded model with the nodal
    fields and marker viscosities the reference's marker->node pass produced."""
    import json
    import cases
    from i3elvis_b200 import prn as P
    p, mode = cases.build(name)
    fx = dict(np.load(os.path.join(ROOT, "tests", "golden", f"{name}.npz")))
    for i, f in enumerate(P.NODE_FIELDS):
        p.nodes[f] = fx["nodes"][i].copy()
    p.marks["v"] = fx["markv"].copy()
    with open(os.path.join(ROOT, "tests", "golden", f"{name}.json")) as fh:
        fx["meta"] = json.load(fh)
    mode.infile = "prep.prn"
    return p, mode, fx


# reference-generated cases small enough for the CPU oracle's tests (the 33^3 case runs in
# the oracle tests that stay fast and in the GPU tests)
SMALL_CASES = ["sphere13", "sphere17", "incl17", "dp17", "stretch17"]
ALL_CASES = SMALL_CASES + ["sphere33"]


@pytest.fixture(params=SMALL_CASES)
def golden_case(request):
    return (request.param,) + golden(request.param)
