"""GPU parity of the CUDA path (through the C ABI) against the FP64 oracle.

Tolerances (plain FP32 form; FP64 only for the cutoff test, positions,
the MLP output layer, energy/virial sums and the position update):
  forces        relative RMS <= 1e-5
  energy        |dE| / N <= 1e-7 eV/atom for the benchmark potential shape
                (16 Gaussians, MLP 64-64-1 tanh); 5e-7 eV/atom for the other
                shapes (softplus/squareplus residual MLPs, the shipped FNN
                potentials whose table is rounded to FP32): FP32 weights of a
                deeper MLP shift every atom's energy by a few 1e-8..1e-7 eV
  virial        relative error of the 6-vector <= 1e-5
  neighbor set  bit-exact (same (i, j, image) tuples) at rc + skin
"""
import numpy as np
import pytest

from pack import Oracle, load_npz
from tmd_b200 import PairTensorMD, TensorMDModel, TensorMDSystem, synth
from tmd_testutil import (GOLDEN, NKTV2P, bcc_lattice, canonical_pairs, frac_wrap, kinetic_pressure,
                          published, read_data, rel_rms, volume)

pytestmark = pytest.mark.gpu

FORCE_RRMS = 1e-5
E_PER_ATOM = 1e-7
E_PER_ATOM_OTHER = 5e-7
VIR_REL = 1e-5


def _run(model_args, x, types, box, pbc=(1, 1, 1), skin=1.0, peratom=False):
    m = TensorMDModel(model_args)
    s = TensorMDSystem(m, len(x), skin)
    s.set_box(box, pbc)
    s.set_atoms(x, types)
    out = s.compute(1, 1, 1.0, peratom=peratom)
    return m, s, out


def _check(out, ref, n, e_tol=E_PER_ATOM):
    assert rel_rms(out["f"], ref["f"]) <= FORCE_RRMS, rel_rms(out["f"], ref["f"])
    de = abs(out["energy"] - ref["energy"]) / n
    assert de <= e_tol, (de, out["energy"], ref["energy"])
    vr = np.linalg.norm(out["virial"] - ref["virial"]) / np.linalg.norm(ref["virial"])
    assert vr <= VIR_REL, vr


@pytest.fixture(scope="module")
def fcc4k(tmp_path_factory):
    """4,000-atom FCC, 16 Gaussians, rc 6, rank <= 3, MLP 64-64-64-1 tanh."""
    c = synth.config("fcc4k")
    p = tmp_path_factory.mktemp("pot") / "fcc4k.npz"
    syms = synth.gaussian_potential(p, seed=1234, **c["pot"])
    x, t, box, v = synth.build_system(c["kind"], c["a"], c["cells"], sigma=c["sigma"],
                                      T=c["T"], nelt=c["nelt"], seed=42)
    return str(p), syms, x, t, box, v


def test_neighbor_set_bit_exact(fcc4k):
    p, syms, x, t, box, _ = fcc4k
    m, s, _ = _run(f"{p} {' '.join(syms)}", x, t, box)
    cut = m.cutmax + 1.0
    got = canonical_pairs(*s.neighbor_list(cut))
    ref = canonical_pairs(*Oracle.neighbors(x, box, [1, 1, 1], cut))
    assert np.array_equal(got, ref)


def test_neighbor_set_small_triclinic():
    x, t, box = read_data(GOLDEN / "Mo8_Ni8_id3210.data")
    x = frac_wrap(x, box)
    m, s, _ = _run(f"{GOLDEN}/MoNi_m3.npz Mo Ni interp 0.0001", x, t, box)
    cut = m.cutmax + 1.0
    got = canonical_pairs(*s.neighbor_list(cut))
    ref = canonical_pairs(*Oracle.neighbors(x, box, [1, 1, 1], cut))
    assert np.array_equal(got, ref)


def test_fcc4k_against_oracle(fcc4k):
    p, syms, x, t, box, _ = fcc4k
    _, _, out = _run(f"{p} {' '.join(syms)}", x, t, box)
    ref = Oracle(p).compute(x, t - 1, box, [1, 1, 1], skin=1.0)
    _check(out, ref, len(x))


def test_peratom_energy_virial(fcc4k):
    p, syms, x, t, box, _ = fcc4k
    _, _, out = _run(f"{p} {' '.join(syms)}", x, t, box, peratom=True)
    ref = Oracle(p).compute(x, t - 1, box, [1, 1, 1], skin=1.0)
    assert np.abs(out["eatom"] - ref["eatom"]).max() < 2e-6
    assert rel_rms(out["vatom"], ref["vatom"]) <= 2e-5
    assert np.sum(out["eatom"]) == pytest.approx(out["energy"], abs=1e-6)
    assert np.abs(out["vatom"].sum(0) - out["virial"]).max() < 1e-6 * np.abs(out["virial"]).max()


def test_moni_published_on_gpu():
    """GPU against the reference's published MoNi_m3 numbers."""
    pub = published()
    p = pub["MoNi_m3"]
    x, t, box = read_data(GOLDEN / "Mo8_Ni8_id3210.data")
    x = frac_wrap(x, box)
    _, _, out = _run(f"{GOLDEN}/MoNi_m3.npz Mo Ni interp 0.0001", x, t, box)
    assert out["energy"] == pytest.approx(p["energy_total"] / p["replicas"],
                                          abs=16 * E_PER_ATOM_OTHER)
    rows = np.array(pub["MoNi_m3_forces"]["rows"])[:16, 2:5]
    assert rel_rms(out["f"], rows) <= 2e-5
    press = out["virial"][:3].mean() / volume(box) * NKTV2P
    assert press == pytest.approx(p["press"], rel=2e-5)


def test_w_m3_k64_published_on_gpu():
    """GPU against the reference's published W_m3_k64_n128_squareplus numbers
    (64 filters, residual squareplus MLP): perfect BCC W, 24 x 24 x 40 cells =
    46,080 atoms.  Energy within 2e-7 of |E| (measured 1.2e-7: the FP32
    rounding of the radial table, the 64-filter sums and the MLP is the same
    in every atom of the perfect lattice, so it does not average out as it
    does over a disordered cell); the virial pressure plus LAMMPS's kinetic
    part at the run's 300 K within the virial bar; forces of the symmetric
    lattice vanish up to FP32 cancellation."""
    p = published()["W_m3_k64"]
    run = p["runs"][0]
    x, box = bcc_lattice(p["lattice"], 24, 24, 40)
    assert len(x) == run["natoms"]
    t = np.ones(len(x), dtype=np.int32)
    _, _, out = _run(f"{GOLDEN}/W_m3_k64_n128_squareplus.npz W interp 0.001", x, t, box)
    press = out["virial"][:3].mean() / volume(box) * NKTV2P + kinetic_pressure(
        run["natoms"], run["temp"], volume(box))
    fmax = np.abs(out["f"]).max()
    diag = (out["energy"], run["pe"], press, run["press"], fmax)
    assert out["energy"] == pytest.approx(run["pe"], rel=2e-7), diag
    assert press == pytest.approx(run["press"], rel=VIR_REL), diag
    assert fmax < 1e-3, diag


def test_moni_squareplus_published_on_gpu():
    """MoNi_squareplus_500k on the Mo8Ni8 cell: the GPU against the FP64
    oracle at the residual-MLP bars, and the published 16,000-atom step-0
    energy (the cell replicated 10 x 10 x 10)."""
    p = published()["MoNi_squareplus"]
    x, t, box = read_data(GOLDEN / "Mo8_Ni8_id3210.data")
    x = frac_wrap(x, box)
    _, _, out = _run(f"{GOLDEN}/MoNi_squareplus_500k.npz Mo Ni interp 0.0001", x, t, box)
    ref = Oracle(str(GOLDEN / "MoNi_squareplus_500k.npz"), interp=1e-4).compute(
        x, t - 1, box, [1, 1, 1])
    assert rel_rms(out["f"], ref["f"]) <= 2e-5
    assert abs(out["energy"] - ref["energy"]) / len(x) <= E_PER_ATOM_OTHER
    vr = np.linalg.norm(out["virial"] - ref["virial"]) / np.linalg.norm(ref["virial"])
    assert vr <= VIR_REL, vr
    assert out["energy"] * p["replicas"] == pytest.approx(
        p["pe"], abs=0.01 + p["natoms"] * E_PER_ATOM_OTHER)


def test_three_elements_against_oracle():
    pub = published()["AlMgSi"]
    x, t, box = read_data(GOLDEN / "AlMgSi.data")
    x = frac_wrap(x, box)
    _, _, out = _run(f"{GOLDEN}/AlMgSi.24aug13.npz Al Mg Si interp 0.0001", x, t, box)
    ref = Oracle(str(GOLDEN / "AlMgSi.24aug13.npz"), interp=1e-4).compute(x, t - 1, box, [1, 1, 1])
    # atomic energies of this potential are about -500 eV (its output bias):
    # the FP32 hidden layers bound the energy to ~1e-8 relative, not 1e-7 eV
    _check(out, ref, len(x), e_tol=1e-8 * abs(ref["energy"]) / len(x))
    assert out["energy"] * pub["replicas"] == pytest.approx(pub["energy_total"], abs=1.0)


def test_wide_mlp_streamed_weights_against_oracle(tmp_path):
    """The precision config's potential (4 elements, 32 filters, rc 6.5,
    512-128-128-128-1 softplus): its FP32 weights do not fit in shared
    memory, so the plain form streams them in chunks.  10,976 atoms = 172
    tiles of 64 atoms, more than one per SM."""
    p = tmp_path / "alloy.npz"
    syms = synth.gaussian_potential(p, seed=99, **synth.config("alloy432k")["pot"])
    x, t, box, _ = synth.build_system("fcc", 3.6, (14, 14, 14), sigma=0.05, nelt=4, seed=7)
    _, s, out = _run(f"{p} {' '.join(syms)}", x, t, box)
    ref = Oracle(load_npz(p)).compute(x, t - 1, box, [1, 1, 1], skin=1.0)
    _check(out, ref, len(x))
    again = s.compute(1, 1, 1.0)
    assert np.array_equal(again["f"], out["f"]) and again["energy"] == out["energy"]


@pytest.mark.parametrize("kw", [dict(actfn=1, resnet=1, hidden=(32, 32, 32)),
                                dict(actfn=3, resnet=0, hidden=(32, 32), fctype=1),
                                dict(actfn=2, resnet=0, hidden=(64, 64), max_moment=2),
                                dict(actfn=2, resnet=0, hidden=(64, 64), max_moment=1)])
def test_activation_and_rank_variants(tmp_path, kw):
    p = tmp_path / "v.npz"
    syms = synth.gaussian_potential(p, nelt=2, num_filters=8, rc=5.5, seed=3, **kw)
    x, t, box, _ = synth.build_system("bcc", 2.9, (6, 6, 6), sigma=0.1, nelt=2, seed=5)
    _, _, out = _run(f"{p} {' '.join(syms)}", x, t, box)
    ref = Oracle(load_npz(p)).compute(x, t - 1, box, [1, 1, 1], skin=1.0)
    _check(out, ref, len(x), e_tol=E_PER_ATOM_OTHER)


def test_set_positions_any_periodic_frame(fcc4k):
    """Positions handed over in another periodic frame (every atom shifted by
    -1, 0 or +1 box vectors per axis, as a caller that wraps at other times
    would hand them over) give the forces and energy of the original frame,
    to the FP64 rounding of the shift."""
    p, syms, x, t, box, _ = fcc4k
    m = TensorMDModel(f"{p} {' '.join(syms)}")
    s = TensorMDSystem(m, len(x), 1.0)
    s.set_box(box)
    s.set_atoms(x, t)
    ref = s.compute(1, 1)
    k = np.random.default_rng(3).integers(-1, 2, size=(len(x), 3))
    s.set_positions(x + k * np.array([box[3], box[4], box[5]]))
    out = s.compute(1, 1)
    assert rel_rms(out["f"], ref["f"]) <= 1e-12
    assert out["energy"] == pytest.approx(ref["energy"], rel=1e-12)
    np.testing.assert_allclose(out["virial"], ref["virial"], rtol=1e-10, atol=1e-10)


def test_deterministic_bitwise(fcc4k):
    p, syms, x, t, box, _ = fcc4k
    m = TensorMDModel(f"{p} {' '.join(syms)}")
    s = TensorMDSystem(m, len(x), 1.0)
    s.set_box(box)
    s.set_atoms(x, t)
    a = s.compute()
    b = s.compute()
    assert np.array_equal(a["f"], b["f"]) and a["energy"] == b["energy"]
    assert np.array_equal(a["virial"], b["virial"])


def test_nve_matches_oracle(fcc4k):
    p, syms, x, t, box, v = fcc4k
    m = TensorMDModel(f"{p} {' '.join(syms)}")
    s = TensorMDSystem(m, len(x), 1.0)
    s.set_box(box)
    s.set_atoms(x, t, v)
    th = s.nve_run(20, 0.001, thermo_every=10)
    xg, vg, fg, img = s.get()
    o = Oracle(p)
    xo, vo, fo, tho = o.nve(x, v, t - 1, box, [1, 1, 1], 0.001, 20, skin=1.0)
    # unwrap both through the box images before comparing
    L = box[3:6]
    dx = (xg - xo) - np.round((xg - xo) / L) * L
    assert np.abs(dx).max() < 1e-6
    assert np.abs(vg - vo).max() < 1e-4 * np.abs(vo).max()
    assert th[0, 0] == pytest.approx(tho[0, 0], abs=1e-7 * len(x))
    assert th[-1, 0] + th[-1, 1] == pytest.approx(tho[-1, 0] + tho[-1, 1], abs=2e-7 * len(x))


def test_nve_list_outgrows_its_capacity(tmp_path):
    """An imploding cell (density 0.02 A^-3 at the start, velocities toward
    the centre) outgrows the neighbor capacity sized at set_atoms during the
    run; the chunk is rolled back, the list grown and the steps rerun, so the
    run ends normally and follows the oracle, which has no capacity limit."""
    p = tmp_path / "pot.npz"
    syms = synth.gaussian_potential(p, nelt=1, num_filters=16, rc=6.0, max_moment=3,
                                    hidden=(32, 32), actfn=2, seed=21)
    a = 0.02 ** (-1.0 / 3.0)
    x, t, box, _ = synth.build_system("sc", a, (6, 6, 6), sigma=0.05, seed=3)
    c = box[3:6] / 2.0
    v = -30.0 * (x - c)  # 40% of the distance to the centre after 20 fs
    m = TensorMDModel(f"{p} {' '.join(syms)}")
    s = TensorMDSystem(m, len(x), 1.0)
    s.set_box(box)
    s.set_atoms(x, t, v)
    cap0 = max(np.diff(s.neighbor_list(m.cutmax + 1.0)[0]))
    th = s.nve_run(20, 0.001, thermo_every=10)
    cap1 = max(np.diff(s.neighbor_list(m.cutmax + 1.0)[0]))
    assert cap1 > 2 * cap0  # the rows grew well beyond the first estimate
    xo, vo, fo, tho = Oracle(str(p)).nve(x, v, t - 1, box, [1, 1, 1], 0.001, 20, skin=1.0)
    xg = s.get()[0]
    L = box[3:6]
    dx = (xg - xo) - np.round((xg - xo) / L) * L
    assert np.abs(dx).max() < 1e-5
    np.testing.assert_allclose(th[-1], tho[-1], rtol=1e-5)


def test_nve_energy_drift(fcc4k):
    """Total energy over 1,000 steps of 1 fs stays within 1e-5 eV/atom."""
    p, syms, x, t, box, v = fcc4k
    m = TensorMDModel(f"{p} {' '.join(syms)}")
    s = TensorMDSystem(m, len(x), 1.0)
    s.set_box(box)
    s.set_atoms(x, t, v)
    th = s.nve_run(1000, 0.001, thermo_every=100)
    etot = th[:, 0] + th[:, 1]
    assert np.abs(etot - etot[0]).max() / len(x) < 1e-5


def test_pair_style_interface(fcc4k):
    p, syms, x, t, box, _ = fcc4k
    pair = PairTensorMD()
    pair.settings()
    with pytest.raises(ValueError):
        pair.settings("bogus")
    pair.coeff(f"* * {p} {' '.join(syms)}")
    assert pair.init_one(1, 1) == pytest.approx(6.0)
    f = pair.compute(x, t, box, eflag=1, vflag=1, eflag_atom=1)
    ref = Oracle(p).compute(x, t - 1, box, [1, 1, 1])
    assert rel_rms(f, ref["f"]) <= FORCE_RRMS
    assert pair.eng_vdwl == pytest.approx(ref["energy"], abs=E_PER_ATOM * len(x))
    assert pair.eatom.shape == (len(x),)


def test_edge_cases(tmp_path):
    p = tmp_path / "e.npz"
    syms = synth.gaussian_potential(p, nelt=1, num_filters=8, rc=4.0, hidden=(8, 8), seed=2)
    m = TensorMDModel(f"{p} {' '.join(syms)}")
    o = Oracle(load_npz(p))
    big = np.array([0, 0, 0, 30.0, 30.0, 30.0, 0, 0, 0])
    # zero atoms
    s = TensorMDSystem(m, 4, 1.0)
    s.set_box(big)
    s.set_atoms(np.zeros((0, 3)), np.zeros(0, dtype=np.int32))
    assert s.compute()["energy"] == 0.0
    # one isolated atom: E = MLP(0), no force
    x1 = np.array([[5.0, 5.0, 5.0]])
    s.set_atoms(x1, [1])
    out = s.compute()
    ref = o.compute(x1, [0], big, [1, 1, 1])
    assert out["energy"] == pytest.approx(ref["energy"], abs=1e-6)
    assert np.abs(out["f"]).max() == 0.0
    # a pair across the periodic boundary, and the same pair non-periodic
    x2 = np.array([[0.5, 1.0, 1.0], [29.0, 1.2, 0.9]])
    s.set_atoms(x2, [1, 1])
    out = s.compute()
    ref = o.compute(x2, [0, 0], big, [1, 1, 1])
    assert np.allclose(out["f"], ref["f"], rtol=1e-5, atol=1e-7)
    assert np.abs(out["f"]).max() > 0
    s.set_box(big, (0, 0, 0))
    s.set_atoms(x2, [1, 1])
    assert np.abs(s.compute()["f"]).max() == 0.0
    # unmapped type is rejected
    with pytest.raises(Exception):
        s.set_atoms(x2, [1, 2])
