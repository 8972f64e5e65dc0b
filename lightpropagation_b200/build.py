"""Build step for the native libraries (in-tree, so the built .so files travel with the tree).

    python -m lightpropagation_b200.build
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def build(verbose: bool = False) -> None:
    """Compile liblpcuda.so (sm_100a) and the C++ host library."""
    quiet = [] if verbose else ["-s"]
    subprocess.check_call(["make", *quiet, "-C", os.path.join(HERE, "csrc")])
    host = os.path.join(HERE, "csrc", "host")
    if os.path.isfile(os.path.join(host, "Makefile")):
        subprocess.check_call(["make", *quiet, "-C", host])


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
