"""FP32 MLP forms against the FP64 oracle on shapes the benchmark configs do
not reach.

The warp-tile form runs every MLP whose hidden layers are 64 wide and not
residual: each activation kind, several elements (weights reloaded when a
CTA's tiles change element), input widths that are not multiples of the
64-column GEMM pass (dE/dG columns masked), one and three hidden layers.  The
resident form runs the other widths and the residual MLPs.  Every case must
meet the plain-form bars (force relative RMS 1e-5, energy 5e-7 eV/atom, or
2e-7 of the per-atom energy where residual layers make it large, virial
1e-5)."""
import numpy as np
import pytest

from pack import Oracle, load_npz
from tmd_b200 import TensorMDModel, TensorMDSystem, synth
from tmd_testutil import rel_rms

pytestmark = pytest.mark.gpu


def _run(tmp_path, *, nelt, K, mm, hidden, actfn, resnet=0, seed=5, e_rel=0.0):
    p = tmp_path / "m.npz"
    syms = synth.gaussian_potential(p, nelt=nelt, num_filters=K, rc=5.5, max_moment=mm,
                                    hidden=hidden, actfn=actfn, resnet=resnet, seed=seed)
    x, t, box, _ = synth.build_system("fcc", 3.6, (6, 6, 6), sigma=0.08, nelt=nelt,
                                      seed=seed + 1)
    m = TensorMDModel(f"{p} {' '.join(syms)}")
    s = TensorMDSystem(m, len(x), 1.0)
    s.set_box(box, [1, 1, 1])
    s.set_atoms(x, t)
    out = s.compute(1, 1, 1.0)
    again = s.compute(1, 1, 1.0)
    assert np.array_equal(out["f"], again["f"])  # deterministic run to run
    ref = Oracle(load_npz(p)).compute(x, t - 1, box, [1, 1, 1], skin=1.0)
    assert rel_rms(out["f"], ref["f"]) <= 1e-5, rel_rms(out["f"], ref["f"])
    e_tol = max(5e-7, e_rel * abs(ref["energy"]) / len(x))
    assert abs(out["energy"] - ref["energy"]) / len(x) <= e_tol
    vr = np.linalg.norm(out["virial"] - ref["virial"]) / np.linalg.norm(ref["virial"])
    assert vr <= 1e-5, vr


@pytest.mark.parametrize("actfn", [0, 1, 2, 3])
def test_warp_tile_activations(tmp_path, actfn):
    # nin = 3 elements x 8 filters x 4 moments = 96: a full and a masked
    # 64-column pass of dE/dG
    _run(tmp_path, nelt=3, K=8, mm=3, hidden=(64, 64), actfn=actfn)


@pytest.mark.parametrize("hidden", [(64,), (64, 64, 64)])
def test_warp_tile_depths(tmp_path, hidden):
    _run(tmp_path, nelt=2, K=16, mm=2, hidden=hidden, actfn=2)


def test_resident_form_other_widths(tmp_path):
    _run(tmp_path, nelt=2, K=8, mm=3, hidden=(48, 48), actfn=2)


def test_residual_mlp_other_form(tmp_path):
    # residual layers carry their inputs forward, so the per-atom energies
    # are large (about -7 eV): the bar is the FP32 rounding of that sum
    _run(tmp_path, nelt=1, K=16, mm=3, hidden=(64, 64, 64), actfn=1, resnet=1, e_rel=2e-7)
