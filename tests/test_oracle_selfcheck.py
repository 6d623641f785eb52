"""Internal consistency of the oracle: forces and virial are exact derivatives
of its energy, the neighbor list equals a brute-force image enumeration, and
the rational table tracks the analytic radial functions."""
import numpy as np
import pytest

from pack import Oracle, load_npz
from tmd_b200 import synth
from tmd_testutil import canonical_pairs, frac_wrap


def _pot(tmp_path, **kw):
    p = tmp_path / "pot.npz"
    synth.gaussian_potential(p, **kw)
    return load_npz(p)


def _small_system(seed=3, tilt=(0.0, 0.0, 0.0), nelt=2):
    x, t, box, _ = synth.build_system("fcc", 3.6, (2, 2, 2), sigma=0.12, nelt=nelt, seed=seed)
    box = box.copy()
    box[6:9] = tilt
    x = frac_wrap(x, box)
    return x, t, box


@pytest.mark.parametrize("actfn,resnet,fctype", [(2, 0, 0), (1, 1, 0), (3, 1, 1), (0, 0, 0)])
def test_forces_are_energy_gradient(tmp_path, actfn, resnet, fctype):
    pot = _pot(tmp_path, nelt=2, num_filters=8, rc=5.0, hidden=(16, 16), actfn=actfn,
               resnet=resnet, fctype=fctype, seed=11)
    o = Oracle(pot)
    x, t, box = _small_system(tilt=(0.4, -0.3, 0.25))
    out = o.compute(x, t - 1, box, [1, 1, 1], skin=0.5)
    h = 1e-5
    rng = np.random.default_rng(0)
    for i in rng.choice(len(x), 4, replace=False):
        for a in range(3):
            xp = x.copy(); xp[i, a] += h
            xm = x.copy(); xm[i, a] -= h
            ep = o.compute(xp, t - 1, box, [1, 1, 1], skin=0.5)["energy"]
            em = o.compute(xm, t - 1, box, [1, 1, 1], skin=0.5)["energy"]
            fd = -(ep - em) / (2 * h)
            assert out["f"][i, a] == pytest.approx(fd, abs=2e-7, rel=2e-6)


def test_virial_is_strain_derivative(tmp_path):
    pot = _pot(tmp_path, nelt=1, num_filters=8, rc=5.0, hidden=(16, 16), actfn=2, seed=5)
    o = Oracle(pot)
    x, t, box = _small_system(nelt=1)
    out = o.compute(x, t - 1, box, [1, 1, 1])
    h = 1e-6
    for a in range(3):
        def energy(eps):
            s = np.ones(3); s[a] += eps
            b = box.copy(); b[3 + a] *= s[a]
            return o.compute(x * s, t - 1, b, [1, 1, 1])["energy"]
        w = -(energy(h) - energy(-h)) / (2 * h)
        assert out["virial"][a] == pytest.approx(w, rel=1e-6, abs=1e-8)


def _brute_list(x, box, cut):
    """All (i, j, s) with |x_j + s.h - x_i| <= cut, images built hop by hop."""
    n = len(x)
    xprd, yprd, zprd, xy, xz, yz = box[3:9]
    rows = []
    for i in range(n):
        for j in range(n):
            for sx in range(-3, 4):
                for sy in range(-3, 4):
                    for sz in range(-3, 4):
                        if i == j and sx == sy == sz == 0:
                            continue
                        px, py, pz = x[j]
                        st = 1.0 if sx > 0 else -1.0
                        for _ in range(abs(sx)):
                            px = px + st * xprd
                        st = 1.0 if sy > 0 else -1.0
                        for _ in range(abs(sy)):
                            px = px + st * xy; py = py + st * yprd
                        st = 1.0 if sz > 0 else -1.0
                        for _ in range(abs(sz)):
                            px = px + st * xz; py = py + st * yz; pz = pz + st * zprd
                        dx, dy, dz = x[i][0] - px, x[i][1] - py, x[i][2] - pz
                        if dx * dx + dy * dy + dz * dz <= cut * cut:
                            rows.append((i, j, sx, sy, sz))
    return np.array(sorted(rows), dtype=np.int64)


def test_neighbor_list_matches_brute_force():
    rng = np.random.default_rng(1)
    box = np.array([0.3, -0.2, 0.1, 5.1, 5.6, 4.9, 0.7, -0.4, 0.3])
    x = frac_wrap(rng.uniform(0, 5, size=(12, 3)), box)
    cut = 6.2
    off, ent = Oracle.neighbors(x, box, [1, 1, 1], cut)
    got = canonical_pairs(off, ent)
    ref = _brute_list(x, box, cut)
    assert got.shape == ref.shape
    assert np.array_equal(got, ref)


def test_table_tracks_analytic(tmp_path):
    pot = _pot(tmp_path, nelt=1, num_filters=8, rc=5.0, hidden=(16, 16), actfn=2, seed=9)
    x, t, box = _small_system(nelt=1)
    direct = Oracle(pot).compute(x, t - 1, box, [1, 1, 1])
    table = Oracle(pot, interp=1e-4).compute(x, t - 1, box, [1, 1, 1])
    assert table["energy"] == pytest.approx(direct["energy"], rel=1e-8)
    assert np.abs(table["f"] - direct["f"]).max() < 1e-6 * max(1.0, np.abs(direct["f"]).max())


def test_fire_restatement_relaxes_a_trained_cell():
    """min_style fire (LAMMPS defaults) in the oracle relaxes a perturbed
    Mo8Ni8 cell of the reference's trained MoNi potential to max |F_i| < 0.01
    eV/A, lowering the energy; the returned forces are those of the returned
    positions."""
    from tmd_testutil import GOLDEN, frac_wrap, read_data
    x, t, box = read_data(GOLDEN / "Mo8_Ni8_id3210.data")
    x = frac_wrap(x, box) + np.random.default_rng(2).normal(0.0, 0.1, size=x.shape)
    o = Oracle(str(GOLDEN / "MoNi_m3.npz"), interp=1e-4)
    e0 = o.compute(frac_wrap(x, box), t - 1, box, [1, 1, 1])["energy"]
    xo, fo, eo, it = o.fire(x, t - 1, box, [1, 1, 1], 0.001, 0.01, 1000)
    assert it < 1000
    assert np.linalg.norm(fo, axis=1).max() < 0.01
    assert eo < e0
    again = o.compute(xo, t - 1, box, [1, 1, 1])
    assert np.abs(again["f"] - fo).max() < 1e-12
    # capped run: exactly maxiter iterations when the tolerance is unreachable
    _, _, _, it2 = o.fire(x, t - 1, box, [1, 1, 1], 0.001, 1e-12, 30)
    assert it2 == 30


@pytest.mark.parametrize("sommerfeld", [0, 1])
def test_tdnp_forces_are_the_free_energy_gradient(tmp_path, sommerfeld):
    """TDNP restatement (tdnp.cpp, nnp.cu:295-318): the energy is the sum of
    U, the forces are -dA/dx with A = U - T S (S scaled by T in the Sommerfeld
    form), checked by central differences at T = 5000 K; A - U = -T S."""
    p = tmp_path / "t.npz"
    synth.tdnp_potential(p, nelt=2, sommerfeld=sommerfeld)
    o = Oracle(load_npz(p), etemp=5000.0)
    x, t, box, _ = synth.build_system("fcc", 3.6, (2, 2, 2), sigma=0.1, nelt=2, seed=3)
    r = o.compute(x, t - 1, box, [1, 1, 1])
    S, A = o.tdnp_totals()
    T = 5000.0 / 11604.522060401008
    assert A == pytest.approx(r["energy"] - T * S, rel=1e-12)
    h = 1e-5
    for i in (0, 17):
        for a in range(3):
            xp, xm = x.copy(), x.copy()
            xp[i, a] += h
            xm[i, a] -= h
            o.compute(xp, t - 1, box, [1, 1, 1])
            ap = o.tdnp_totals()[1]
            o.compute(xm, t - 1, box, [1, 1, 1])
            am = o.tdnp_totals()[1]
            assert r["f"][i, a] == pytest.approx(-(ap - am) / (2 * h), rel=1e-6, abs=1e-8)
