"""Where the reference tree (lammps-tensormd) lies, for the checker scripts
that read it: oracle/build_ref.py, tests/golden/make_golden.py and the
plugin syntax check.  TEST INFRASTRUCTURE ONLY.

One environment variable, TMD_REFERENCE_TREE, names the tree; without it the
mount point of this build's read-only copy is used.  Scripts that find no
tree there skip what needs it.
"""
from __future__ import annotations

import os
from pathlib import Path

DEFAULT = "/root/reference"


def reference_tree() -> Path:
    return Path(os.environ.get("TMD_REFERENCE_TREE", DEFAULT))
