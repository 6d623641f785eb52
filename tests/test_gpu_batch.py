"""Multi-cell batches (tmd_batch_*) through the C ABI.

A batch of C cells must give, cell by cell, what C separate systems give:
  forces        bit-identical to the separate systems (same neighbor rows after
                sorting, same per-pair arithmetic, same per-atom MLP rows)
  energy/virial per-cell FP64 sums in another fixed order: relative 1e-12
  NVE runs     per cell bitwise the positions, velocities, forces and image
                counters of separate runs (a cell's list is rebuilt when its
                own atoms trigger it); thermo sums 1e-12 relative
and the FP64 oracle, cell by cell, within the plain-form tolerances
(force relative RMS 1e-5, energy 5e-7 eV/atom, virial 1e-5).
Cells cover FCC and BCC lattices, a triclinic cell and cells smaller than the
list cutoff (two images per axis)."""
import numpy as np
import pytest

from pack import Oracle
from tmd_b200 import TensorMDBatch, TensorMDModel, TensorMDSystem, TmdError, synth
from tmd_testutil import GOLDEN, frac_wrap, read_data, rel_rms

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pot2(tmp_path_factory):
    p = tmp_path_factory.mktemp("pot") / "cells.npz"
    syms = synth.gaussian_potential(p, seed=77, **synth.config("cells4096")["pot"])
    return str(p), syms


def _cells():
    """(x, types, box) of cells of several shapes and sizes."""
    rng = np.random.default_rng(5)
    out = []
    data = synth.batch_cells(4, 256, nelt=2, seed=3)
    for x, t, box, _ in data["cells"]:
        out.append((x, t, box))
    # 32-atom FCC cell (7.2 A box, list cutoff 7 A) and a 16-atom one (3.6 x
    # 3.6 x 14.4 A): two images per axis
    for cells in ((2, 2, 2), (1, 1, 4)):
        x, t, box, _ = synth.build_system("fcc", 3.6, cells, sigma=0.05, nelt=2,
                                          seed=int(rng.integers(1 << 30)))
        out.append((x, t, box))
    # the triclinic 16-atom cell of the reference's binary example
    x, t, box = read_data(GOLDEN / "Mo8_Ni8_id3210.data")
    out.append((frac_wrap(x, box), t, box))
    return out


def _batch(args, cells, skin=1.0, v=None):
    m = TensorMDModel(args)
    b = TensorMDBatch(m, [len(c[0]) for c in cells], skin)
    b.set_cells(np.stack([c[2] for c in cells]))
    b.set_atoms(np.concatenate([c[0] for c in cells]), np.concatenate([c[1] for c in cells]),
                v)
    return m, b


def _separate(args, x, t, box, skin=1.0, v=None):
    m = TensorMDModel(args)
    s = TensorMDSystem(m, len(x), skin)
    s.set_box(box)
    s.set_atoms(x, t, v)
    return m, s


def test_batch_equals_separate_systems(pot2):
    p, syms = pot2
    args = f"{p} {' '.join(syms)}"
    cells = _cells()
    m, b = _batch(args, cells)
    out = b.compute()
    off = b.offsets
    for c, (x, t, box) in enumerate(cells):
        _, s = _separate(args, x, t, box)
        ref = s.compute(1, 1)
        assert np.array_equal(out["f"][off[c]:off[c + 1]], ref["f"]), c
        assert out["energy"][c] == pytest.approx(ref["energy"], rel=1e-12, abs=1e-10)
        np.testing.assert_allclose(out["virial"][c], ref["virial"], rtol=1e-12, atol=1e-10)


def test_batch_non_periodic_cells(pot2):
    """A slab (periodic in x and y, the box 10 A taller than the atoms), a
    cluster (periodic in no direction) and a periodic cell in one batch: each
    cell's bin grid takes no image shift along its non-periodic axes.  Forces
    bit-identical to separate systems with the same boundaries."""
    p, syms = pot2
    args = f"{p} {' '.join(syms)}"
    x, t, box, _ = synth.build_system("fcc", 3.6, (3, 3, 3), sigma=0.05, nelt=2, seed=11)
    slab_box = box.copy()
    slab_box[5] += 10.0
    cl_box = box.copy()
    cl_box[3:6] += 12.0
    cells = [(x + np.array([0.0, 0.0, 5.0]), t, slab_box, (1, 1, 0)),
             (x + 6.0, t, cl_box, (0, 0, 0)),
             (x, t, box, (1, 1, 1))]
    m = TensorMDModel(args)
    b = TensorMDBatch(m, [len(c[0]) for c in cells], 1.0)
    b.set_cells(np.stack([c[2] for c in cells]), np.array([c[3] for c in cells]))
    b.set_atoms(np.concatenate([c[0] for c in cells]), np.concatenate([c[1] for c in cells]))
    out = b.compute()
    off = b.offsets
    for c, (xc, tc, bc, pbc) in enumerate(cells):
        s = TensorMDSystem(m, len(xc), 1.0)
        s.set_box(bc, pbc)
        s.set_atoms(xc, tc)
        ref = s.compute(1, 1)
        assert np.array_equal(out["f"][off[c]:off[c + 1]], ref["f"]), c
        assert out["energy"][c] == pytest.approx(ref["energy"], rel=1e-12, abs=1e-10)


def test_batch_against_oracle(pot2):
    p, syms = pot2
    cells = _cells()
    _, b = _batch(f"{p} {' '.join(syms)}", cells)
    out = b.compute()
    off = b.offsets
    orc = Oracle(p)
    for c in (0, 1, 4, 5):
        x, t, box = cells[c]
        ref = orc.compute(x, t - 1, box, [1, 1, 1], skin=1.0)
        f = out["f"][off[c]:off[c + 1]]
        assert rel_rms(f, ref["f"]) <= 1e-5, (c, rel_rms(f, ref["f"]))
        # 5e-7 eV/atom as for the other potential shapes of the single-system
        # tests (this one has two elements, MLP input 128)
        assert abs(out["energy"][c] - ref["energy"]) / len(x) <= 5e-7, c
        vr = np.linalg.norm(out["virial"][c] - ref["virial"]) / np.linalg.norm(ref["virial"])
        assert vr <= 1e-5, (c, vr)


def test_batch_triclinic_moni_against_oracle():
    """Triclinic cell with the shipped FNN potential, inside a batch."""
    x, t, box = read_data(GOLDEN / "Mo8_Ni8_id3210.data")
    x = frac_wrap(x, box)
    args = f"{GOLDEN}/MoNi_m3.npz Mo Ni interp 0.0001"
    cells = [(x, t, box), (x, t, box)]
    _, b = _batch(args, cells)
    out = b.compute()
    ref = Oracle(str(GOLDEN / "MoNi_m3.npz"), interp=1e-4).compute(x, t - 1, box, [1, 1, 1])
    for c in range(2):
        f = out["f"][16 * c:16 * (c + 1)]
        assert rel_rms(f, ref["f"]) <= 2e-5
        assert abs(out["energy"][c] - ref["energy"]) / 16 <= 5e-7


def test_batch_nve_matches_separate_runs(pot2):
    p, syms = pot2
    args = f"{p} {' '.join(syms)}"
    data = synth.batch_cells(6, 256, nelt=2, seed=21)
    cells = [(x, t, box) for x, t, box, _ in data["cells"]]
    _, b = _batch(args, cells, v=data["v"])
    th = b.nve_run(60, 0.001, thermo_every=20)
    assert th.shape == (4, 6, 2)
    bx, bv, bf, bimg = b.get()
    off = b.offsets
    for c, (x, t, box, v) in enumerate(data["cells"]):
        _, s = _separate(args, x, t, box, v=v)
        ref = s.nve_run(60, 0.001, thermo_every=20)
        # a cell rebuilds its list exactly when its own atoms trigger it, as
        # the separate system does, so the trajectories are the same bit for
        # bit; the thermo sums run in another order
        sx, sv, sf, simg = s.get()
        sl = slice(off[c], off[c + 1])
        assert np.array_equal(bx[sl], sx) and np.array_equal(bv[sl], sv), c
        assert np.array_equal(bf[sl], sf) and np.array_equal(bimg[sl], simg), c
        np.testing.assert_allclose(th[:, c, :], ref, rtol=1e-12, atol=1e-12)
    # total energy per cell is conserved over the run
    etot = th.sum(-1)
    assert np.abs(etot - etot[0]).max() < 1e-3 * 256


def test_batch_rejects_cells_below_three_images(pot2):
    p, syms = pot2
    m = TensorMDModel(f"{p} {' '.join(syms)}")
    b = TensorMDBatch(m, [4], 1.0)
    with pytest.raises(TmdError) as e:
        b.set_cells(np.array([[0, 0, 0, 2.0, 2.0, 2.0, 0, 0, 0]]))
    assert e.value.code == -1
    sysv = b.system()
    with pytest.raises(TmdError) as e:
        sysv.set_box([0, 0, 0, 10.0, 10.0, 10.0, 0, 0, 0])
    assert e.value.code == -7
