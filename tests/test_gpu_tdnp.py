"""Temperature-dependent potentials (tdnp = 1, TDNP of tdnp.cpp) on the GPU
through the C ABI, against the FP64 oracle's restatement.

The nets H, U, S replace the MLP; the energy is U, the forces those of the
free energy A = U - T S, and S and A are reported as the pair style's
eentropy and free_energy.  Bars (FP32 nets against FP64): forces relative
RMS 1e-5, energy 5e-7 eV/atom, entropy and free energy 1e-6 relative, at the
pair_coeff electron temperature and after changing it (fix tensormd/etemp),
in the plain and the Sommerfeld forms, two elements.
"""
import numpy as np
import pytest

from pack import Oracle, load_npz
from tmd_b200 import TensorMDModel, TensorMDSystem, synth
from tmd_testutil import rel_rms

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("sommerfeld", [0, 1])
def test_tdnp_against_the_oracle(tmp_path, sommerfeld):
    p = tmp_path / "tdnp.npz"
    syms = synth.tdnp_potential(p, nelt=2, num_filters=8, rc=5.0, h_hidden=(32, 32), ydim=8,
                                u_hidden=(16,), s_hidden=(16,), sommerfeld=sommerfeld, seed=5)
    x, t, box, _ = synth.build_system("fcc", 3.6, (4, 4, 4), sigma=0.08, nelt=2, seed=11)
    n = len(x)
    m = TensorMDModel(f"{p} {' '.join(syms)} etemp 5000")
    s = TensorMDSystem(m, n, 1.0)
    s.set_box(box)
    s.set_atoms(x, t)
    o = Oracle(load_npz(p), etemp=5000.0)
    for kelvin in (5000.0, 12000.0):
        if kelvin != 5000.0:
            s.set_etemp(kelvin)
            o.set_etemp(kelvin)
        out = s.compute(1, 1)
        ref = o.compute(x, t - 1, box, [1, 1, 1], skin=1.0)
        S, A = s.tdnp_energies()
        So, Ao = o.tdnp_totals()
        assert rel_rms(out["f"], ref["f"]) <= 1e-5, (kelvin, rel_rms(out["f"], ref["f"]))
        assert abs(out["energy"] - ref["energy"]) / n <= 5e-7
        assert S == pytest.approx(So, rel=1e-6, abs=1e-6 * n)
        assert A == pytest.approx(Ao, rel=1e-6, abs=1e-6 * n)
        vr = np.linalg.norm(out["virial"] - ref["virial"]) / np.linalg.norm(ref["virial"])
        assert vr <= 1e-5


def test_tdnp_refuses_tensor_core_forms(tmp_path):
    p = tmp_path / "tdnp.npz"
    syms = synth.tdnp_potential(p, nelt=1)
    with pytest.raises(Exception):
        TensorMDModel(f"{p} {' '.join(syms)} precision bf16")
