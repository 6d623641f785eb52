"""The oracle against the reference's own CPU contraction code.

oracle/_ref/libtmdref.so is the reference's src/ML-TENSORMD/tensor_ops.cpp
(kernel_P, kernel_dEdG, kernel_dEdS, kernel_U, kernel_V, kernel_F1,
kernel_fused_F2 with calculate_dM) compiled from the reference tree with its
vendored Eigen (oracle/build_ref.py).  Fed the same per-pair geometry, radial
values and MLP gradients, it must reproduce the oracle's descriptor
invariants G and its forces to FP64 rounding (relative 1e-11), for one and two
elements, an orthogonal and a triclinic cell.  Skipped where neither the
library nor the reference tree exists."""
import numpy as np
import pytest

import refcheck
from pack import Oracle, load_npz
from tmd_b200 import synth
from tmd_testutil import GOLDEN, frac_wrap, read_data

REF = refcheck.load()
pytestmark = pytest.mark.skipif(REF is None, reason="reference CPU kernels unavailable")


def _case(tmp_path, nelt, lattice):
    p = tmp_path / f"pot{nelt}.npz"
    synth.gaussian_potential(p, nelt=nelt, num_filters=8, rc=5.0, max_moment=3,
                             hidden=(16, 16), actfn=1, seed=11 + nelt)
    if lattice == "triclinic":
        x, t, box = read_data(GOLDEN / "Mo8_Ni8_id3210.data")
        x = frac_wrap(x, box)
        t = ((t - 1) % nelt) + 1
    else:
        x, t, box, _ = synth.build_system(lattice, 3.6, (2, 2, 2), sigma=0.1, nelt=nelt, seed=5)
    return str(p), x, np.asarray(t), box


@pytest.mark.parametrize("nelt,lattice", [(1, "fcc"), (2, "fcc"), (2, "triclinic")])
def test_oracle_matches_reference_kernels(tmp_path, nelt, lattice):
    p, x, t, box = _case(tmp_path, nelt, lattice)
    orc = Oracle(p)
    nl = Oracle.neighbors(x, box, [1, 1, 1], orc.rmax)
    out = orc.compute(x, t - 1, box, [1, 1, 1], nlist=nl, want_G=True, want_dEdG=True)
    ref = refcheck.pair_forces(REF, load_npz(p), x, t - 1, box, nl, out["G"], out["dEdG"])
    Gr = refcheck.invariants(ref["P"], ref["T"]).reshape(len(x), -1)
    assert np.abs(Gr - out["G"]).max() <= 1e-11 * np.abs(out["G"]).max()
    fmax = np.abs(out["f"]).max()
    assert np.abs(ref["f"] - out["f"]).max() <= 1e-11 * fmax, np.abs(ref["f"] - out["f"]).max()


def test_check_detects_a_planted_error(tmp_path):
    """The comparison is sensitive: a 0.1% error planted in the MLP gradient
    handed to the reference kernels shows up far above the tolerance."""
    p, x, t, box = _case(tmp_path, 2, "fcc")
    orc = Oracle(p)
    nl = Oracle.neighbors(x, box, [1, 1, 1], orc.rmax)
    out = orc.compute(x, t - 1, box, [1, 1, 1], nlist=nl, want_G=True, want_dEdG=True)
    ref = refcheck.pair_forces(REF, load_npz(p), x, t - 1, box, nl, out["G"],
                               out["dEdG"] * 1.001)
    assert np.abs(ref["f"] - out["f"]).max() > 1e-5 * np.abs(out["f"]).max()
