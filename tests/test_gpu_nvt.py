"""fix nvt on the device (tmd_nvt_run, tmd_batch_nvt_run) against the oracle.

  trajectory   40 steps of a 256-atom FCC cell heated from 300 K toward 500 K
               (t_damp 0.05 ps): pe within 1e-7 eV/atom (the plain form's
               FP32 energy bar), ke within 1e-7 relative, positions within
               1e-6 A and the chain energy within 1e-6 relative of the FP64
               oracle
  batch        per-cell thermostats (different targets) equal separate
               systems' runs within 1e-6 relative
  persistence  two runs of 20 steps continue the chain like one run of 40:
               thermo within 1e-9 relative"""
import numpy as np
import pytest

from pack import Oracle
from tmd_b200 import TensorMDBatch, TensorMDModel, TensorMDSystem, synth
from tmd_testutil import frac_wrap

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pot(tmp_path_factory):
    p = tmp_path_factory.mktemp("pot") / "nvt.npz"
    syms = synth.gaussian_potential(p, nelt=2, num_filters=16, rc=6.0, max_moment=3,
                                    hidden=(32, 32), actfn=2, seed=8)
    return str(p), syms


def _state(seed, cells=(4, 4, 4), T=300.0):
    return synth.build_system("fcc", 3.6, cells, sigma=0.05, T=T, nelt=2, seed=seed,
                              masses=[63.546, 58.6934])


def test_nvt_trajectory_matches_oracle(pot):
    p, syms = pot
    x, t, box, v = _state(1)
    m = TensorMDModel(f"{p} {' '.join(syms)}")
    s = TensorMDSystem(m, len(x), 1.0)
    s.set_box(box)
    s.set_atoms(x, t, v)
    th = s.nvt_run(40, 0.001, 300.0, 500.0, 0.05, thermo_every=1)
    xo, vo, fo, tho = Oracle(p).nvt(x, v, t - 1, box, [1, 1, 1], 0.001, 40, 300.0, 500.0, 0.05)
    n = len(x)
    assert np.abs(th[:, 0] - tho[:, 0]).max() <= 1e-7 * n  # FP32 energy: 1e-7 eV/atom
    np.testing.assert_allclose(th[:, 1], tho[:, 1], rtol=1e-7)
    assert s.nvt_energy()[0] == pytest.approx(tho[-1, 2], rel=1e-6, abs=1e-7 * n)
    xg = s.get()[0]
    d = frac_wrap(xg, box) - frac_wrap(xo, box)
    L = box[3:6]
    d -= L * np.round(d / L)
    assert np.abs(d).max() < 1e-6
    # the thermostat acted: the run is not NVE
    the = Oracle(p).nve(x, v, t - 1, box, [1, 1, 1], 0.001, 40)[3]
    assert abs(the[-1, 1] - tho[-1, 1]) > 1e-3 * tho[-1, 1]


def test_nvt_batch_cells_equal_separate_runs(pot):
    p, syms = pot
    m = TensorMDModel(f"{p} {' '.join(syms)}")
    cells = [_state(10 + c, cells=(3, 3, 3), T=300.0 + 100 * c) for c in range(4)]
    b = TensorMDBatch(m, [len(c[0]) for c in cells], 1.0)
    b.set_cells(np.stack([c[2] for c in cells]))
    b.set_atoms(np.concatenate([c[0] for c in cells]), np.concatenate([c[1] for c in cells]),
                np.concatenate([c[3] for c in cells]))
    tstart = np.array([300.0, 400.0, 500.0, 600.0])
    tstop = np.array([600.0, 400.0, 300.0, 900.0])
    th = b.nvt_run(30, 0.001, tstart, tstop, 0.05, thermo_every=10)
    for c, (x, t, box, v) in enumerate(cells):
        s = TensorMDSystem(m, len(x), 1.0)
        s.set_box(box)
        s.set_atoms(x, t, v)
        ref = s.nvt_run(30, 0.001, tstart[c], tstop[c], 0.05, thermo_every=10)
        np.testing.assert_allclose(th[:, c, :], ref, rtol=1e-6, atol=1e-6)


def test_nvt_chain_persists_between_runs(pot):
    p, syms = pot
    x, t, box, v = _state(2)
    m = TensorMDModel(f"{p} {' '.join(syms)}")
    one = TensorMDSystem(m, len(x), 1.0)
    one.set_box(box)
    one.set_atoms(x, t, v)
    th1 = one.nvt_run(40, 0.001, 400.0, 400.0, 0.05, thermo_every=40)
    two = TensorMDSystem(m, len(x), 1.0)
    two.set_box(box)
    two.set_atoms(x, t, v)
    two.nvt_run(20, 0.001, 400.0, 400.0, 0.05)
    th2 = two.nvt_run(20, 0.001, 400.0, 400.0, 0.05, thermo_every=20)
    np.testing.assert_allclose(th2[-1], th1[-1], rtol=1e-9)
