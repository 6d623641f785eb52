"""The LAMMPS-side binding (pair style tensormd/b200 and its plugin entry)
compiles against the LAMMPS headers of the reference tree (syntax check with
the serial MPI stubs).  Skipped where that tree is not mounted."""
import shutil
import subprocess
from pathlib import Path

import pytest

from reftree import reference_tree
from tmd_testutil import ROOT

LAMMPS_SRC = reference_tree() / "src"


@pytest.mark.skipif(not (LAMMPS_SRC / "pair.h").exists() or shutil.which("g++") is None,
                    reason="LAMMPS headers not available")
@pytest.mark.parametrize("src", ["pair_tensormd_b200.cpp", "tensormd_b200_plugin.cpp",
                                 "compute_tensormd_density_b200.cpp"])
def test_plugin_compiles_against_lammps_headers(src):
    plug = ROOT / "lammps-tensormd_b200" / "lammps"
    cmd = ["g++", "-std=c++17", "-fsyntax-only", "-DLAMMPS_SMALLBIG",
           "-I", str(LAMMPS_SRC), "-I", str(LAMMPS_SRC / "STUBS"),
           "-I", str(ROOT / "include"), "-I", str(plug), str(plug / src)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
