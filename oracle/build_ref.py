"""Build oracle/_ref/libtmdref.so: the reference's own CPU contraction code
(src/ML-TENSORMD/tensor_ops.cpp with its vendored Eigen), compiled from the
reference tree where it lies, plus oracle/ref_harness.cpp and the CBLAS shim
in oracle/ref_shim/.  Test infrastructure only (a second checker next to the
oracle restatement); nothing in the product links it.

    python oracle/build_ref.py [--force]

Needs the reference tree (TMD_REFERENCE_TREE, see oracle/reftree.py);
without it the build is skipped and the tests that use the library are
skipped too.  Output goes only to oracle/_ref/.
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
if str(HERE) not in sys.path:
    sys.path.insert(0, str(HERE))
from reftree import reference_tree  # noqa: E402

REF_SRC = reference_tree() / "src" / "ML-TENSORMD"
OUT_DIR = HERE / "_ref"
LIB = OUT_DIR / "libtmdref.so"


def build(force: bool = False) -> Path | None:
    src = REF_SRC / "tensor_ops.cpp"
    if not src.exists():
        return LIB if LIB.exists() else None
    deps = [src, REF_SRC / "tensor_ops.h", REF_SRC / "cppblas.hpp", HERE / "ref_harness.cpp",
            HERE / "ref_shim" / "cblas.h"]
    if LIB.exists() and not force and LIB.stat().st_mtime >= max(p.stat().st_mtime for p in deps):
        return LIB
    OUT_DIR.mkdir(exist_ok=True)
    # the shim directory comes first so cppblas.hpp's "cblas.h" resolves to it;
    # no USE_MKL_BATCH / EIGEN_USE_MKL_ALL: the plain loop and Eigen paths
    cmd = ["g++", "-O2", "-std=c++14", "-fPIC", "-shared", "-w",
           "-I", str(HERE / "ref_shim"), "-I", str(REF_SRC),
           str(HERE / "ref_harness.cpp"), str(src), "-o", str(LIB)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"reference build failed:\n{r.stderr[-4000:]}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
