"""Pin the FP64 oracle to the reference's own published outputs.

The reference has no unit tests for pair_style tensormd; its only known
answers are the example logs and the force.yaml dump (read as text into
tests/golden/published.json by tests/golden/make_golden.py).  These tests run
the oracle on the same potentials and cells and require agreement to the
printed precision.
"""
import numpy as np
import pytest

from pack import Oracle
from tmd_testutil import GOLDEN, NKTV2P, kinetic_pressure, published, read_data, volume


@pytest.fixture(scope="module")
def pub():
    return published()


def test_moni_m3_energy_forces_pressure(pub):
    p = pub["MoNi_m3"]
    x, t, box = read_data(GOLDEN / "Mo8_Ni8_id3210.data")
    o = Oracle(str(GOLDEN / "MoNi_m3.npz"), interp=p["interp"])
    out = o.compute(x, t - 1, box, [1, 1, 1], skin=1.0)
    # 96,000-atom energy printed with 15 significant digits
    assert out["energy"] == pytest.approx(p["energy_total"] / p["replicas"], abs=1e-9)
    vir = out["virial"] / volume(box) * NKTV2P
    assert vir[0] == pytest.approx(p["pxx"], abs=1e-3)
    assert vir[1] == pytest.approx(p["pyy"], abs=1e-3)
    assert vir[2] == pytest.approx(p["pzz"], abs=1e-3)
    assert vir[:3].mean() == pytest.approx(p["press"], abs=1e-3)
    rows = np.array(pub["MoNi_m3_forces"]["rows"])
    # force.yaml holds a 2x2x2 replica: 8 copies of the 16 distinct atoms
    ref = rows[:16, 2:5]
    for k in range(1, 8):
        assert np.allclose(rows[16 * k:16 * (k + 1), 2:5], ref, atol=1e-8)
    assert np.abs(out["f"] - ref).max() < 1e-8  # printed to 8 decimals
    assert np.abs(out["f"]).max() == pytest.approx(p["fmax_component"], abs=1e-9)


def test_moni_squareplus_energy_pressure(pub):
    """MoNi_squareplus_500k on the Mo8Ni8 cell replicated 10 x 10 x 10: the
    step-0 energy (8 significant digits) within one unit of the last digit,
    the pressure (virial part plus the kinetic part at 100 K) within 2e-3 bar."""
    p = pub["MoNi_squareplus"]
    x, t, box = read_data(GOLDEN / "Mo8_Ni8_id3210.data")
    o = Oracle(str(GOLDEN / "MoNi_squareplus_500k.npz"), interp=p["interp"])
    out = o.compute(x, t - 1, box, [1, 1, 1])
    assert out["energy"] * p["replicas"] == pytest.approx(p["pe"], abs=0.01)
    p_vir = out["virial"][:3].mean() / volume(box) * NKTV2P
    p_kin = kinetic_pressure(p["natoms"], p["temp"], volume(box) * p["replicas"])
    assert p_vir + p_kin == pytest.approx(p["press"], abs=2e-3)


def test_almgsi_energy(pub):
    p = pub["AlMgSi"]
    x, t, box = read_data(GOLDEN / "AlMgSi.data")
    o = Oracle(str(GOLDEN / "AlMgSi.24aug13.npz"), interp=p["interp"])
    e = o.compute(x, t - 1, box, [1, 1, 1])["energy"]
    # thermo prints 8 significant digits of the 32,400-atom total
    assert e * p["replicas"] == pytest.approx(p["energy_total"], abs=0.5)


def test_w_k32_energy(pub):
    p = pub["W_k32"]
    a = p["lattice"]
    x = np.array([[0.0, 0.0, 0.0], [0.5 * a, 0.5 * a, 0.5 * a]])
    box = np.array([0, 0, 0, a, a, a, 0, 0, 0], dtype=float)
    o = Oracle(str(GOLDEN / "W_k32_snapshot.npz"), interp=p["interp"])
    out = o.compute(x, [0, 0], box, [1, 1, 1])
    e_atom = out["energy"] / 2
    assert e_atom * p["natoms"] == pytest.approx(p["energy_total"], abs=0.05)
    # step-0 pressure of the 300 K run: virial part plus the kinetic part
    p_vir = out["virial"][:3].mean() / a ** 3 * NKTV2P
    vol = p["natoms"] / 2 * a ** 3
    assert p_vir + kinetic_pressure(p["natoms"], p["temp"], vol) == pytest.approx(p["press"], abs=2e-3)
    # the 200,000,000-atom weak-scaling run of the same potential (perfect
    # lattice: the same energy per atom; 8 significant digits printed)
    big = pub["W_k32_200M"]
    assert e_atom * big["natoms"] == pytest.approx(big["pe"], abs=100.0)
    vol = big["natoms"] / 2 * a ** 3
    assert p_vir + kinetic_pressure(big["natoms"], big["temp"], vol) == pytest.approx(big["press"], abs=2e-3)


def test_w_m3_k64_energy_and_pressure(pub):
    """W_m3_k64_n128_squareplus (64 filters, residual squareplus MLP) on perfect
    BCC W of 46,080 to 115,200 atoms: every atom has the same environment, so
    the two-atom cell gives the energy per atom and the virial pressure.  The
    published step-0 energies (8 significant digits) within one unit of the
    last digit; the pressures (Press minus its kinetic part) within 2e-3 bar
    (printed to 1e-3 bar; the reference's FP32 virial moves the last digit)."""
    p = pub["W_m3_k64"]
    a = p["lattice"]
    x = np.array([[0.0, 0.0, 0.0], [0.5 * a, 0.5 * a, 0.5 * a]])
    box = np.array([0, 0, 0, a, a, a, 0, 0, 0], dtype=float)
    o = Oracle(str(GOLDEN / "W_m3_k64_n128_squareplus.npz"), interp=p["interp"])
    out = o.compute(x, [0, 0], box, [1, 1, 1])
    e_atom = out["energy"] / 2
    p_vir = out["virial"][:3].mean() / a ** 3 * NKTV2P
    for run in p["runs"]:
        unit = 10.0 ** (np.floor(np.log10(abs(run["pe"]))) - 7)
        assert e_atom * run["natoms"] == pytest.approx(run["pe"], abs=unit), run
        p_kin = kinetic_pressure(run["natoms"], run["temp"], run["volume"])
        assert p_vir + p_kin == pytest.approx(run["press"], abs=2e-3), run
