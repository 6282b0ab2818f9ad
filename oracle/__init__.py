"""CPU oracle: test infrastructure only (tests, smoke() and bench.py's CPU baseline legs)."""
from __future__ import annotations

import os

# Where the build recipe looks for the reference source tree (cuStingerAlg) when compiling
# oracle/_ref. TC_REFERENCE_ROOT overrides it; on machines without the tree nothing under _ref is
# rebuilt and the prebuilt files are used as they are.
_DEFAULT_REFERENCE_TREE = "/root/reference"


def reference_tree() -> str | None:
    """Root of the reference source tree, or None when it is absent."""
    root = os.environ.get("TC_REFERENCE_ROOT") or _DEFAULT_REFERENCE_TREE
    return root if os.path.isfile(os.path.join(root, "tests", "cct.cpp")) else None


def make_args() -> list[str]:
    """`make` variables for oracle/Makefile: REF when the reference tree is present."""
    root = reference_tree()
    return [f"REF={root}"] if root else []
