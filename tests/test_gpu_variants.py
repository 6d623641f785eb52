"""Kernel forms of the pair-force loop and of the descriptor
(tmd_system_set_variant / autotune).

Every combination of forms must meet the plain-form tolerances against the FP64 oracle
(force relative RMS 1e-5, energy 1e-7 eV/atom on the benchmark shape and
5e-7 on the others, virial 1e-5) on every radial kind (Gaussian, rational
table, the generic analytic forms), every monomial count (D = 1, 4, 10, 20),
more than one element and in multi-cell batches.  The forms sum in different
orders, so between forms the forces agree to FP32 rounding (relative RMS
5e-6 on the benchmark shape, where the two-stream descriptor adds its pairs
as two partial sums), and each form is bitwise deterministic run to run."""
import numpy as np
import pytest

from pack import Oracle, load_npz
from tmd_b200 import TensorMDBatch, TensorMDModel, TensorMDSystem, synth
from tmd_testutil import GOLDEN, frac_wrap, read_data, rel_rms

pytestmark = pytest.mark.gpu

FORMS = TensorMDSystem.FORCE_VARIANTS
DFORMS = TensorMDSystem.DESC_VARIANTS


def _check(out, ref, n, e_tol, f_tol=1e-5):
    assert rel_rms(out["f"], ref["f"]) <= f_tol, rel_rms(out["f"], ref["f"])
    assert abs(out["energy"] - ref["energy"]) / n <= e_tol
    vr = np.linalg.norm(out["virial"] - ref["virial"]) / np.linalg.norm(ref["virial"])
    assert vr <= 1e-5, vr


def _forms(args, x, t, box, pbc=(1, 1, 1)):
    m = TensorMDModel(args)
    s = TensorMDSystem(m, len(x), 1.0)
    s.set_box(box, pbc)
    s.set_atoms(x, t)
    outs = {}
    for dv in DFORMS:
        s.set_descriptor_variant(dv)
        assert s.descriptor_variant() == dv
        for v in FORMS:
            s.set_force_variant(v)
            assert s.force_variant() == v
            outs[(dv, v)] = s.compute(1, 1, 1.0)
            again = s.compute(1, 1, 1.0)
            assert np.array_equal(outs[(dv, v)]["f"], again["f"]), (dv, v)
    return outs


def _analytic(path, method, K=8, rc=5.5, seed=11):
    """A 2-element potential whose radial basis is descriptor::method 0, 1 or 2,
    with parameters that keep the descriptors O(1-100) as trained potentials
    do (a Morse basis far below r0 gives G ~ 1e4, where the FP32 form's
    relative error grows with the cancellation inside P)."""
    syms = synth.gaussian_potential(path, nelt=2, num_filters=K, rc=rc, seed=seed,
                                    hidden=(32, 32))
    d = dict(np.load(path))
    for k in ("descriptor::eta", "descriptor::omega"):
        d.pop(k)
    d["descriptor::method"] = np.int32(method)
    lin = np.linspace(0.0, 1.0, K)
    if method == 0:
        d["descriptor::rl"] = 1.5 + 2.5 * lin
        d["descriptor::pl"] = 1.0 + 2.0 * lin
    elif method == 1:
        d["descriptor::D"] = 0.5 + 0.5 * lin
        d["descriptor::gamma"] = 0.3 + 0.3 * lin
        d["descriptor::r0"] = 2.6 + 1.4 * lin
    else:
        d["descriptor::A"] = 1.0 - 0.5 * lin
        d["descriptor::beta"] = 1.0 + 2.0 * lin
        d["descriptor::re"] = 2.0 + 2.0 * lin
    np.savez(path, **d)
    return syms


@pytest.fixture(scope="module")
def fcc4k(tmp_path_factory):
    c = synth.config("fcc4k")
    p = tmp_path_factory.mktemp("pot") / "fcc4k.npz"
    syms = synth.gaussian_potential(p, seed=1234, **c["pot"])
    x, t, box, _ = synth.build_system(c["kind"], c["a"], c["cells"], sigma=c["sigma"],
                                      T=c["T"], nelt=c["nelt"], seed=42)
    return str(p), syms, x, t, box


def test_forms_on_benchmark_shape(fcc4k):
    p, syms, x, t, box = fcc4k
    outs = _forms(f"{p} {' '.join(syms)}", x, t, box)
    ref = Oracle(p).compute(x, t - 1, box, [1, 1, 1], skin=1.0)
    first = outs[(DFORMS[0], FORMS[0])]
    for v, out in outs.items():
        _check(out, ref, len(x), 1e-7)
        # the forms sum in different orders (pairs, filters, two pair streams)
        assert rel_rms(out["f"], first["f"]) <= 5e-6, v


def test_descriptor_forms_agree(fcc4k):
    """Both descriptor forms give the same G = T P^2 rows to FP32 rounding."""
    p, syms, x, t, box = fcc4k
    m = TensorMDModel(f"{p} {' '.join(syms)}")
    s = TensorMDSystem(m, len(x), 1.0)
    s.set_box(box, [1, 1, 1])
    s.set_atoms(x, t)
    G = {}
    for dv in DFORMS:
        s.set_descriptor_variant(dv)
        s.compute(1, 1, 1.0)
        G[dv] = s.descriptors()
    ref = Oracle(p).compute(x, t - 1, box, [1, 1, 1], skin=1.0, want_G=True)["G"]
    for dv, g in G.items():
        assert rel_rms(g, ref) <= 1e-6, (dv, rel_rms(g, ref))
    assert rel_rms(G[DFORMS[1]], G[DFORMS[0]]) <= 1e-6


@pytest.mark.parametrize("D,mm", [(1, 0), (4, 1), (10, 2)])
def test_forms_monomial_counts(tmp_path, D, mm):
    p = tmp_path / "v.npz"
    syms = synth.gaussian_potential(p, nelt=2, num_filters=8, rc=5.5, seed=3,
                                    max_moment=mm, hidden=(32, 32))
    x, t, box, _ = synth.build_system("bcc", 2.9, (6, 6, 6), sigma=0.1, nelt=2, seed=5)
    outs = _forms(f"{p} {' '.join(syms)}", x, t, box)
    ref = Oracle(load_npz(p)).compute(x, t - 1, box, [1, 1, 1], skin=1.0)
    for out in outs.values():
        _check(out, ref, len(x), 5e-7)


@pytest.mark.parametrize("method", [0, 1, 2])
def test_forms_generic_radial(tmp_path, method):
    p = tmp_path / "g.npz"
    syms = _analytic(p, method)
    x, t, box, _ = synth.build_system("fcc", 3.6, (5, 5, 5), sigma=0.08, nelt=2, seed=9)
    outs = _forms(f"{p} {' '.join(syms)}", x, t, box)
    ref = Oracle(load_npz(p)).compute(x, t - 1, box, [1, 1, 1], skin=1.0)
    for out in outs.values():
        _check(out, ref, len(x), 5e-7)


def test_forms_table_three_elements():
    x, t, box = read_data(GOLDEN / "AlMgSi.data")
    x = frac_wrap(x, box)
    outs = _forms(f"{GOLDEN}/AlMgSi.24aug13.npz Al Mg Si interp 0.0001", x, t, box)
    ref = Oracle(str(GOLDEN / "AlMgSi.24aug13.npz"), interp=1e-4).compute(x, t - 1, box,
                                                                          [1, 1, 1])
    for out in outs.values():
        _check(out, ref, len(x), 1e-8 * abs(ref["energy"]) / len(x))


def test_forms_small_triclinic_table():
    x, t, box = read_data(GOLDEN / "Mo8_Ni8_id3210.data")
    x = frac_wrap(x, box)
    outs = _forms(f"{GOLDEN}/MoNi_m3.npz Mo Ni interp 0.0001", x, t, box)
    ref = Oracle(str(GOLDEN / "MoNi_m3.npz"), interp=1e-4).compute(x, t - 1, box, [1, 1, 1])
    # 16 atoms near equilibrium: net forces ~0.03 eV/A are differences of pair
    # terms ~1 eV/A, so the FP32 rounding shows at 1e-5 relative (the same
    # 2e-5 bound as the published-number check of this cell)
    for out in outs.values():
        _check(out, ref, len(x), 5e-7, f_tol=2e-5)


def test_forms_in_a_batch(tmp_path):
    p = tmp_path / "c.npz"
    syms = synth.gaussian_potential(p, seed=77, **synth.config("cells4096")["pot"])
    m = TensorMDModel(f"{p} {' '.join(syms)}")
    rng = np.random.default_rng(4)
    cells = []
    for kind, a, rep in (("fcc", 3.6, (3, 3, 3)), ("bcc", 2.9, (2, 2, 2)), ("fcc", 3.5, (2, 2, 3))):
        x, t, box, _ = synth.build_system(kind, a, rep, sigma=0.1, nelt=len(syms),
                                          seed=int(rng.integers(1 << 30)))
        cells.append((x, t, box))
    b = TensorMDBatch(m, [len(c[0]) for c in cells])
    b.set_cells(np.array([c[2] for c in cells]), np.ones((len(cells), 3), dtype=np.int32))
    b.set_atoms(np.concatenate([c[0] for c in cells]), np.concatenate([c[1] for c in cells]))
    sysv = b.system()
    res = {}
    for dv in DFORMS:
        sysv.set_descriptor_variant(dv)
        for v in FORMS:
            sysv.set_force_variant(v)
            res[(dv, v)] = b.compute()
    off = 0
    for c, (x, t, box) in enumerate(cells):
        ref = Oracle(load_npz(p)).compute(x, t - 1, box, [1, 1, 1], skin=1.0)
        n = len(x)
        for v, r in res.items():
            out = {"f": r["f"][off:off + n], "energy": r["energy"][c], "virial": r["virial"][c]}
            _check(out, ref, n, 5e-7)
        off += n


def test_autotune_picks_the_fastest(fcc4k):
    p, syms, x, t, box = fcc4k
    m = TensorMDModel(f"{p} {' '.join(syms)}")
    s = TensorMDSystem(m, len(x), 1.0)
    s.set_box(box, [1, 1, 1])
    s.set_atoms(x, t)
    ms = s.autotune(reps=3)
    assert set(ms) == set(FORMS) and all(v > 0 for v in ms.values())
    assert s.force_variant() == min(ms, key=ms.get)
    md = s.autotune(reps=3, family="descriptor")
    assert set(md) == set(DFORMS) and all(v > 0 for v in md.values())
    assert s.descriptor_variant() == min(md, key=md.get)
    assert s.force_variant() == min(ms, key=ms.get)
    out = s.compute(1, 1, 1.0)
    ref = Oracle(p).compute(x, t - 1, box, [1, 1, 1], skin=1.0)
    _check(out, ref, len(x), 1e-7)
    # the captured MD step follows the chosen form
    th = s.nve_run(5, 0.001, thermo_every=5)
    assert np.all(np.isfinite(th))
