"""The oracle's fix nvt (Nose-Hoover chain of 3, fix_nh.cpp) on the CPU.

  t_damp -> infinity   the chain decouples and the run equals fix nve
                       (thermo and positions to 1e-9)
  conserved quantity   pe + ke + chain energy (FixNH::compute_scalar) stays
                       constant while the thermostat works: the random-weight
                       potential releases energy (the cell heats from 300 K to
                       ~4,800 K under NVE) and the chain takes it out; the
                       deviation is < 1e-3 of the absorbed ~62 eV over 0.3 ps
                       and falls ~4x when dt halves (second order)
  control              the temperature over the second half of the run is
                       far closer to the target than without the thermostat"""
import numpy as np

from pack import Oracle
from tmd_b200 import synth


def _system(tmp_path):
    p = tmp_path / "pot.npz"
    synth.gaussian_potential(p, nelt=1, num_filters=8, rc=5.0, max_moment=3,
                             hidden=(16, 16), actfn=2, seed=3)
    x, t, box, v = synth.build_system("fcc", 3.6, (3, 3, 3), sigma=0.05, T=300.0, seed=4,
                                      masses=[63.546])
    return Oracle(str(p)), x, t - 1, box, v


def test_nvt_with_infinite_damping_is_nve(tmp_path):
    orc, x, e, box, v = _system(tmp_path)
    xa, va, _, tha = orc.nve(x, v, e, box, [1, 1, 1], 0.001, 30)
    xb, vb, _, thb = orc.nvt(x, v, e, box, [1, 1, 1], 0.001, 30, 300.0, 300.0, 1e9)
    np.testing.assert_allclose(thb[:, :2], tha, rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(xb, xa, atol=1e-9)


def test_nvt_conserves_extended_energy_and_controls_temperature(tmp_path):
    orc, x, e, box, v = _system(tmp_path)
    n = len(x)
    dev = []
    for dt, nst in ((0.0005, 600), (0.00025, 1200)):  # the same 0.3 ps
        _, _, _, th = orc.nvt(x, v, e, box, [1, 1, 1], dt, nst, 700.0, 700.0, 0.05)
        H = th.sum(1)
        released = abs(th[-1, 2])  # energy the chain absorbed (~62 eV)
        assert released > 1.0
        dev.append(np.abs(H - H[0]).max())
        assert dev[-1] < 1e-3 * released, (dev[-1], released)
    # second-order integrator: halving dt cuts the deviation about 4x
    assert dev[0] / dev[1] > 3.0, dev
    _, _, _, th = orc.nvt(x, v, e, box, [1, 1, 1], 0.0005, 600, 700.0, 700.0, 0.05)
    T = 2.0 * th[:, 1] / ((3 * n - 3) * synth.BOLTZ)
    _, _, _, th_nve = orc.nve(x, v, e, box, [1, 1, 1], 0.0005, 600)
    T_nve = 2.0 * th_nve[:, 1] / ((3 * n - 3) * synth.BOLTZ)
    assert abs(T[300:].mean() - 700.0) < 0.5 * abs(T_nve[300:].mean() - 700.0)
