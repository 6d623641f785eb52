"""Ghost-aware mode (tmd_system_set_atoms_ghost): the pair style on a rank of
a domain-decomposed LAMMPS run, through the C ABI.

A periodic cell is cut into two slabs along x.  Each "rank" gets its local
atoms and the ghosts LAMMPS's border exchange gives it: every periodic image
of every atom within the ghost cutoff (rc + skin) of the slab, with the image
position x + s * L formed in FP64 as pack_border does.  Each rank's forces on
local and ghost atoms are then reverse-summed onto the owning atoms (what
LAMMPS's reverse communication does with newton_pair on).  The result must
equal the single periodic system's:
  forces        relative RMS <= 1e-6 (same pairs; rows, and with them the
                FP32 summation order, differ)
  energy        sum of the ranks' energies, |dE|/N <= 1e-8 eV/atom (the
                FP32 per-atom energies round differently with the row order)
  virial        sum of the ranks' virials, 1e-6 relative
  eatom/vatom   per atom after the reverse sum (ghost eatom is 0)
  descriptors   the local atoms' G rows (compute tensormd/density), 1e-5
"""
import numpy as np
import pytest

from tmd_b200 import TensorMDModel, TensorMDSystem, synth
from tmd_testutil import rel_rms

pytestmark = pytest.mark.gpu


def _rank_atoms(x, types, box, lo, hi, cut):
    """Local atoms of the slab lo <= x < hi of an orthogonal periodic cell and
    its ghosts out to `cut`: (xall, tall, owner) with the local atoms first;
    owner[k] is the atom that xall[k] is a copy of."""
    L = np.asarray(box[3:6])
    b0 = np.asarray(box[:3])
    xw = b0 + np.mod(x - b0, L)
    local = np.flatnonzero((xw[:, 0] >= lo) & (xw[:, 0] < hi))
    ext_lo = np.array([lo - cut, b0[1] - cut, b0[2] - cut])
    ext_hi = np.array([hi + cut, b0[1] + L[1] + cut, b0[2] + L[2] + cut])
    gx, gown = [], []
    rng = [int(np.ceil(cut / L[a])) for a in range(3)]
    for sx in range(-rng[0], rng[0] + 1):
        for sy in range(-rng[1], rng[1] + 1):
            for sz in range(-rng[2], rng[2] + 1):
                sh = np.array([sx, sy, sz]) * L
                p = xw + sh  # FP64, as pack_border's x + pbc * prd
                inside = np.all((p >= ext_lo) & (p < ext_hi), axis=1)
                if sx == 0 and sy == 0 and sz == 0:
                    inside[local] = False
                k = np.flatnonzero(inside)
                gx.append(p[k])
                gown.append(k)
    gx = np.concatenate(gx)
    gown = np.concatenate(gown)
    xall = np.concatenate([xw[local], gx])
    owner = np.concatenate([local, gown])
    return xall, types[owner], owner, len(local)


@pytest.fixture(scope="module")
def cell(tmp_path_factory):
    p = tmp_path_factory.mktemp("pot") / "ghost.npz"
    syms = synth.gaussian_potential(p, nelt=2, num_filters=16, rc=6.0, max_moment=3,
                                    hidden=(64, 64), actfn=2, seed=17)
    x, t, box, _ = synth.build_system("fcc", 3.61, (10, 10, 10), sigma=0.05, nelt=2, seed=8)
    return f"{p} {' '.join(syms)}", x, t, box


def test_two_slab_ranks_equal_the_periodic_cell(cell):
    args, x, t, box = cell
    m = TensorMDModel(args)
    n = len(x)
    s = TensorMDSystem(m, n, 1.0)
    s.set_box(box)
    s.set_atoms(x, t)
    ref = s.compute(1, 1, peratom=True)
    Gref = s.descriptors()
    cut = m.cutmax + 1.0
    L = box[3]
    f = np.zeros((n, 3))
    eatom = np.zeros(n)
    vatom = np.zeros((n, 6))
    energy, virial = 0.0, np.zeros(6)
    for lo, hi in ((box[0], box[0] + L / 2), (box[0] + L / 2, box[0] + L)):
        xall, tall, owner, nloc = _rank_atoms(x, t, box, lo, hi, cut)
        assert len(xall) > nloc  # there are ghosts
        r = TensorMDSystem(m, len(xall), 1.0)
        r.set_atoms_ghost(nloc, xall, tall)
        out = r.compute(1, 1, peratom=True)
        assert out["f"].shape == (len(xall), 3)
        assert np.all(out["eatom"][nloc:] == 0.0)
        # reverse communication: ghost forces and per-atom virials go home
        np.add.at(f, owner, out["f"])
        np.add.at(eatom, owner, out["eatom"])
        np.add.at(vatom, owner, out["vatom"])
        energy += out["energy"]
        virial += out["virial"]
        G = r.descriptors()
        assert G.shape == (nloc, m.n_desc)
        assert rel_rms(G, Gref[owner[:nloc]]) <= 1e-5
        # positions-only update in the same order (LAMMPS's forward
        # communication between reneighborings): same result
        r.set_positions(xall)
        again = r.compute(1, 1)
        assert rel_rms(again["f"], out["f"]) <= 1e-12
        r.close()
    assert rel_rms(f, ref["f"]) <= 1e-6, rel_rms(f, ref["f"])
    assert abs(energy - ref["energy"]) / n <= 1e-8
    assert np.linalg.norm(virial - ref["virial"]) <= 1e-6 * np.linalg.norm(ref["virial"])
    assert np.abs(eatom - ref["eatom"]).max() < 1e-6
    assert rel_rms(vatom, ref["vatom"]) <= 1e-5


def test_ghost_mode_refuses_md_and_leaves_with_set_atoms(cell):
    args, x, t, box = cell
    m = TensorMDModel(args)
    xall, tall, owner, nloc = _rank_atoms(x, t, box, box[0], box[0] + box[3] / 2, m.cutmax + 1.0)
    s = TensorMDSystem(m, len(x) + len(xall), 1.0)
    s.set_atoms_ghost(nloc, xall, tall)
    with pytest.raises(Exception):
        s.nve_run(1, 0.001)
    # back to the periodic mode
    s.set_box(box)
    s.set_atoms(x, t)
    s.nve_run(2, 0.001)


def test_slab_decomposition_on_the_device(cell):
    """The spatial decomposition driver (tmd_b200.decomp) over the
    ghost-aware device system, one rank holding the whole cell as one slab
    (its own periodic neighbour: every ghost is an image of a local atom):
    forces, energy and virial of the periodic cell, and 10 NVE steps with a
    re-decomposition after 5 against the device-resident fix nve run."""
    from tmd_b200.decomp import SlabDecomposition
    args, x, t, box = cell
    m = TensorMDModel(args)
    n = len(x)
    rng = np.random.default_rng(4)
    masses = np.concatenate([[0.0], [m.type_mass[k] for k in (1, 2)]])
    v = synth.maxwell(masses[t], 600.0, rng)
    s = TensorMDSystem(m, n, 1.0)
    s.set_box(box)
    s.set_atoms(x, t, v)
    ref = s.compute(1, 1)
    r = TensorMDSystem(m, 6 * n, 1.0)
    dec = SlabDecomposition(box, m.cutmax + 1.0, 1.0, r, rebuild_every=5)
    dec.set_atoms(x, t, v)
    f, e, vir = dec.compute()
    xg, vg, fg = dec.gather()
    assert rel_rms(fg, ref["f"]) <= 1e-6
    assert abs(e - ref["energy"]) / n <= 1e-8
    assert np.linalg.norm(vir - ref["virial"]) <= 1e-6 * np.linalg.norm(ref["virial"])
    dec.nve_run(10, 0.001, masses)
    s.nve_run(10, 0.001)
    xs = s.get()[0]
    xd = dec.gather()[0]
    L = box[3:6]
    d = xd - xs
    d -= np.round(d / L) * L
    assert np.abs(d).max() < 1e-7, np.abs(d).max()
