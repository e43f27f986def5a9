"""Build the in-tree CUDA library (sm_100a) and the C host loop.

``python -m i3elvis_b200.build`` compiles ``csrc/*.cu`` into ``i3elvis_b200/libi3g.so``
with ``nvcc -gencode arch=compute_100a,code=sm_100a`` (cross-compiles without a GPU) and
the drop-in host program ``host/i3g`` with gcc.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def build(verbose: bool = False) -> None:
    jobs = str(min(8, os.cpu_count() or 1))
    out = None if verbose else subprocess.DEVNULL
    subprocess.run(["make", "-j", jobs, "-C", os.path.join(HERE, "csrc")], check=True, stdout=out)
    host = os.path.join(HERE, "host")
    if os.path.exists(os.path.join(host, "Makefile")):
        subprocess.run(["make", "-C", host], check=True, stdout=out)


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print("built", os.path.join(HERE, "libi3g.so"))
