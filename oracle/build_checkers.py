"""Test infrastructure: builds the CPU checkers of the VELO chain (oracle/Makefile).

    python oracle/build_checkers.py            # the plain-C restatement, and the reference CPU build
                                      # when the reference tree is found

The reference tree is taken from ALLEN_REFERENCE_ROOT, else from a directory named
``reference`` beside this repository's parent directory; where neither exists only the
restatement is built (the prebuilt oracle/_ref library, if any, is kept).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)


def reference_root() -> str | None:
    """The reference source tree, or None where it is not on this machine."""
    root = os.environ.get("ALLEN_REFERENCE_ROOT")
    if root is None:
        root = os.path.join(os.path.dirname(REPO), "reference")
    return root if os.path.isdir(root) else None


def build_oracle(ref_root: str | None = None, with_reference: bool = True) -> None:
    """The plain-C oracle, then (with_reference) the reference CPU build where its tree exists."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    root = ref_root or (reference_root() if with_reference else None)
    if root:
        subprocess.run(["make", "-s", "-j8", "-C", HERE, "ref", f"REF_ROOT={root}"], check=True)


def build_allen_harness(ref_root: str | None = None) -> None:
    """integration/VeloB200Chain.cu with the reference's headers and velo_kalman_filter, and the
    harness that runs them (tests/allen_harness), where the reference tree exists."""
    root = ref_root or reference_root()
    if root:
        subprocess.run(["make", "-s", "-j8", "-C", os.path.join(REPO, "tests", "allen_harness"), f"REF_ROOT={root}"],
                       check=True)


if __name__ == "__main__":
    build_oracle(sys.argv[1] if len(sys.argv) > 1 else None)
