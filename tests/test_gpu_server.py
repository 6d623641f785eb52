"""Serving loop (tmd_server_*) through the C ABI.

  single-point jobs  forces bit-identical to a separate system of the same
                     atoms (the server runs them as cells of one batch, whose
                     per-cell results equal separate systems), energy and
                     virial to 1e-12 relative (sums in another order)
  NVE jobs           nsteps run; end state bitwise that of tmd_nve_run of the
                     same system (energy sums to 1e-12 relative)
  FIRE jobs          LAMMPS min_style fire (its defaults) against the FP64
                     oracle's restatement of min_fire.cpp: a 200-iteration
                     trajectory on a random-weight potential (positions
                     within 1e-4 A, energy 1e-6 eV/atom), and a relaxation on
                     the trained MoNi potential to max |F_i| < 0.01 eV/A in
                     the oracle's number of iterations
  concurrency        mixed jobs from several threads all complete; results
                     do not depend on what else was in flight
  mix independence   NVE and FIRE end states bitwise the same with other jobs
                     retiring and entering around them
  errors             unknown kind, job beyond the atom budget, box too small
                     for the cutoff, wait timeout"""
import threading
import time

import numpy as np
import pytest

from pack import Oracle, load_npz
from tmd_testutil import GOLDEN, frac_wrap, read_data
from tmd_b200 import TensorMDModel, TensorMDServer, TensorMDSystem, TmdError, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def model4(tmp_path_factory):
    p = tmp_path_factory.mktemp("pot") / "serve.npz"
    syms = synth.gaussian_potential(p, seed=31, nelt=4, num_filters=16, rc=6.0,
                                    max_moment=3, hidden=(64, 64), actfn=2)
    m = TensorMDModel(f"{p} {' '.join(syms)}")
    m.npz_path = str(p)
    return m


def _separate(model, x, t, box, v=None):
    s = TensorMDSystem(model, len(x), 1.0)
    s.set_box(box)
    s.set_atoms(x, t, v)
    return s


def test_single_point_jobs_equal_separate_systems(model4):
    rng = np.random.default_rng(1)
    srv = TensorMDServer(model4, max_atoms=200000, max_cells=256)
    jobs = [synth.serving_job(rng, kind=0, nmax=1200) for _ in range(12)]
    tickets = [srv.submit(0, x, t, box) for x, t, box, _ in jobs]
    for tk, (x, t, box, _) in zip(tickets, jobs):
        out = srv.wait(tk, timeout=120)
        ref = _separate(model4, x, t, box).compute(1, 1)
        assert np.array_equal(out["f"], ref["f"])
        assert out["energy"] == pytest.approx(ref["energy"], rel=1e-12, abs=1e-10)
        np.testing.assert_allclose(out["virial"], ref["virial"], rtol=1e-12, atol=1e-10)
        assert out["steps"] == 0 and out["latency"] > 0
    srv.close()


def test_bf16_single_point_jobs_equal_separate_systems(tmp_path):
    """The tensor-core MLP forms too: a job's result does not depend on the
    other jobs in the batch (MMA rows are independent atoms)."""
    p = tmp_path / "serve_bf16.npz"
    syms = synth.gaussian_potential(p, seed=31, nelt=4, num_filters=16, rc=6.0,
                                    max_moment=3, hidden=(64, 64), actfn=2)
    m = TensorMDModel(f"{p} {' '.join(syms)} precision bf16")
    rng = np.random.default_rng(5)
    srv = TensorMDServer(m, max_atoms=200000, max_cells=256)
    jobs = [synth.serving_job(rng, kind=0, nmax=900) for _ in range(8)]
    tickets = [srv.submit(0, x, t, box) for x, t, box, _ in jobs]
    for tk, (x, t, box, _) in zip(tickets, jobs):
        out = srv.wait(tk, timeout=120)
        ref = _separate(m, x, t, box).compute(1, 1)
        assert np.array_equal(out["f"], ref["f"])
        assert out["energy"] == pytest.approx(ref["energy"], rel=1e-12, abs=1e-10)
    srv.close()


def test_nve_job_matches_system_run(model4):
    rng = np.random.default_rng(2)
    x, t, box, v = synth.serving_job(rng, kind=1, nmin=500, nmax=600)
    srv = TensorMDServer(model4, max_atoms=100000, max_cells=64, steps_per_tick=8)
    tk = srv.submit(1, x, t, box, v=v, nsteps=100, dt=0.001)
    # a second job in flight at the same time
    x2, t2, box2, v2 = synth.serving_job(rng, kind=1, nmin=200, nmax=300)
    tk2 = srv.submit(1, x2, t2, box2, v=v2, nsteps=37, dt=0.001)
    out = srv.wait(tk, timeout=120)
    out2 = srv.wait(tk2, timeout=120)
    assert out["steps"] == 100 and out2["steps"] == 37
    s = _separate(model4, x, t, box, v)
    th = s.nve_run(100, 0.001, thermo_every=100)
    ref = s.compute(1, 1)
    # the job's cell is rebuilt when its own atoms trigger it and kicks and
    # drifts round as FixNVE on the device does: the trajectory is the
    # separate system's bit for bit (the energy sums run in another order)
    sx, sv, sf, _ = s.get()
    assert np.array_equal(out["x"], sx) and np.array_equal(out["v"], sv)
    assert np.array_equal(out["f"], sf)
    assert out["energy"] == pytest.approx(ref["energy"], rel=1e-12)
    m = model4.type_mass[t]
    ke = 0.5 * synth.MVV2E * np.sum(m[:, None] * out["v"] ** 2)
    assert ke == pytest.approx(th[-1, 1], rel=1e-12)
    srv.close()


@pytest.fixture(scope="module")
def model4_bf16(tmp_path_factory):
    p = tmp_path_factory.mktemp("pot") / "serve16.npz"
    syms = synth.gaussian_potential(p, seed=31, nelt=4, num_filters=16, rc=6.0,
                                    max_moment=3, hidden=(64, 64), actfn=2)
    return TensorMDModel(f"{p} {' '.join(syms)} precision bf16")


@pytest.mark.parametrize("form", ["fp32", "bf16"])
def test_trajectory_independent_of_the_mix(model4, model4_bf16, form):
    """An NVE and a FIRE job give bitwise the same end state run together
    and inside a batch whose other cells retire and are admitted while they
    run (three cells at most in flight, so retirements move them and admit
    queued jobs).  Moved cells keep their neighbor lists; a cell's list is
    rebuilt only when its own atoms trigger it; the MLP rows (FP32 or
    tensor-core) are independent atoms."""
    model4 = model4 if form == "fp32" else model4_bf16
    rng = np.random.default_rng(6)
    a = synth.serving_job(rng, kind=1, nmin=400, nmax=500)
    fj = synth.serving_job(rng, kind=2, nmin=150, nmax=250)
    fillers = [(int(k), synth.serving_job(rng, kind=int(k), nmin=50, nmax=700))
               for k in (1, 0, 1, 2, 0, 1, 0, 1, 1, 0)]

    def run(mixed):
        srv = TensorMDServer(model4, max_atoms=100000, max_cells=3, steps_per_tick=4)
        subs = [(1, a, 60), (2, fj, 80)]
        if mixed:
            subs = [(k, j, 5 + 7 * i) for i, (k, j) in enumerate(fillers[:3])] + subs[:1] \
                + [(k, j, 3 + 5 * i) for i, (k, j) in enumerate(fillers[3:7])] + subs[1:] \
                + [(k, j, 9 + 4 * i) for i, (k, j) in enumerate(fillers[7:])]
        tks = [(k, nst, srv.submit(k, x, t, box, v=v, nsteps=max(nst, 1), dt=0.002, fmax=1e-4))
               for k, (x, t, box, v), nst in subs]
        outs = [srv.wait(tk, timeout=300) for _, _, tk in tks]
        srv.close()
        pick = [o for (k, nst, _), o in zip(tks, outs) if (k, nst) in ((1, 60), (2, 80))]
        assert len(pick) == 2
        return pick

    alone, mixed = run(False), run(True)
    for o1, o2 in zip(alone, mixed):
        assert o1["steps"] == o2["steps"]
        for key in ("x", "v", "f"):
            assert np.array_equal(o1[key], o2[key]), key
        assert o1["energy"] == o2["energy"]
        assert np.array_equal(o1["virial"], o2["virial"])


def test_rows_grow_under_running_jobs(model4):
    """A job denser than the rows were sized for (FCC a = 3.3 A: 0.11
    atoms/A^3) arrives while an NVE job runs: every cell's rows move to the
    longer length (atom indices and partner slots re-based), and the running
    job's end state is bitwise the one it has without the dense neighbour."""
    rng = np.random.default_rng(12)
    a = synth.serving_job(rng, kind=1, nmin=400, nmax=500)
    dense = synth.build_system("fcc", 3.3, (3, 3, 3), sigma=0.05, nelt=2, seed=4)

    def run(with_dense):
        srv = TensorMDServer(model4, max_atoms=50000, max_cells=8, steps_per_tick=4)
        row0 = srv.footprint()["row_length"]
        x, t, box, v = a
        tk = srv.submit(1, x, t, box, v=v, nsteps=40, dt=0.002)
        if with_dense:
            while srv.stats()["active_atoms"] == 0:  # the first job is in flight
                time.sleep(0.0005)
            xd, td, boxd, vd = dense
            srv.wait(srv.submit(1, xd, td, boxd, v=vd, nsteps=8, dt=0.001), timeout=120)
            assert srv.footprint()["row_length"] > row0
        out = srv.wait(tk, timeout=120)
        srv.close()
        return out

    o1, o2 = run(False), run(True)
    for key in ("x", "v", "f"):
        assert np.array_equal(o1[key], o2[key]), key
    assert o1["energy"] == o2["energy"]


def test_fire_job_converges_as_the_oracle():
    """FIRE on a trained potential (the reference's MoNi_m3, whose lattice is
    a real minimum; the random-weight test potentials have none and collapse
    under any minimiser): a perturbed 16-atom Mo8Ni8 cell relaxed to
    max |F_i| < 0.01 eV/A in the server takes the oracle's number of
    iterations and ends at its positions; the returned forces are those of
    the returned positions."""
    x, t, box = read_data(GOLDEN / "Mo8_Ni8_id3210.data")
    x = frac_wrap(x, box) + np.random.default_rng(2).normal(0.0, 0.1, size=x.shape)
    model = TensorMDModel(f"{GOLDEN}/MoNi_m3.npz Mo Ni interp 0.0001")
    e0 = _separate(model, frac_wrap(x, box), t, box).compute(1, 1)["energy"]
    srv = TensorMDServer(model, max_atoms=10000, max_cells=8, steps_per_tick=16)
    fmax = 0.01
    out = srv.wait(srv.submit(2, x, t, box, nsteps=1000, dt=0.001, fmax=fmax), timeout=300)
    srv.close()
    xo, fo, eo, it = Oracle(str(GOLDEN / "MoNi_m3.npz"), interp=1e-4).fire(
        x, t - 1, box, [1, 1, 1], 0.001, fmax, 1000)
    assert it < 1000 and out["steps"] == it
    assert np.linalg.norm(out["f"], axis=1).max() < fmax
    assert out["energy"] < e0
    d = frac_wrap(out["x"], box) - frac_wrap(xo, box)
    assert np.abs(d).max() < 1e-5, np.abs(d).max()
    assert abs(out["energy"] - eo) / len(x) < 1e-6
    # a fresh system wraps atoms that crossed the box since the server's last
    # rebuild, which reorders their list rows (and the FP32 sums) and moves
    # forces by ~1e-7 eV/A; forces of a neighbouring FIRE step would differ
    # by far more
    ref = _separate(model, frac_wrap(out["x"], box), t, box).compute(1, 1)
    np.testing.assert_allclose(ref["f"], out["f"], rtol=0, atol=1e-6)


def test_fire_trajectory_follows_the_oracle(model4):
    """200 FIRE iterations of a 64-atom amorphous cell in the server against
    the FP64 oracle's min_style fire (same defaults, same start, v = 0):
    every P = F.v sign, step back and dt change must agree for the end
    positions to agree."""
    rng = np.random.default_rng(21)
    x, box = synth.random_packing(64, rng)
    t = rng.integers(1, 5, size=64).astype(np.int32)
    srv = TensorMDServer(model4, max_atoms=10000, max_cells=8, steps_per_tick=16)
    out = srv.wait(srv.submit(2, x, t, box, nsteps=200, dt=0.001, fmax=1e-9), timeout=300)
    srv.close()
    o = Oracle(load_npz(model4.npz_path))
    xo, fo, eo, it = o.fire(x, t - 1, box, [1, 1, 1], 0.001, 1e-9, 200)
    assert out["steps"] == it == 200
    L = box[3:6]
    d = (out["x"] - xo) - np.round((out["x"] - xo) / L) * L
    assert np.abs(d).max() < 1e-4, np.abs(d).max()
    assert abs(out["energy"] - eo) / len(x) < 1e-6
    assert eo < o.compute(x, t - 1, box, [1, 1, 1])["energy"]


def test_concurrent_mixed_jobs(model4):
    rng = np.random.default_rng(4)
    srv = TensorMDServer(model4, max_atoms=60000, max_cells=64, steps_per_tick=4)
    jobs = []
    for k in range(30):
        kind = (0, 0, 1, 2)[k % 4]
        jobs.append((kind, synth.serving_job(rng, kind=kind, nmax=800)))
    results = {}
    errors = []

    def client(part):
        try:
            for i in part:
                kind, (x, t, box, v) = jobs[i]
                tk = srv.submit(kind, x, t, box, v=v, nsteps=40 if kind == 1 else 400,
                                dt=0.001, fmax=0.2)
                results[i] = srv.wait(tk, timeout=300)
        except Exception as e:  # reported below
            errors.append(e)

    threads = [threading.Thread(target=client, args=(range(r, 30, 3),)) for r in range(3)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    assert not errors, errors
    assert len(results) == 30
    for i, (kind, (x, t, box, v)) in enumerate(jobs):
        if kind == 0:  # independent of what else was in flight
            ref = _separate(model4, x, t, box).compute(1, 1)
            assert np.array_equal(results[i]["f"], ref["f"])
        if kind == 1:
            assert results[i]["steps"] == 40
    st = srv.stats()
    assert st["submitted"] == 30 and st["completed"] == 30 and st["atom_steps"] > 0
    srv.close()


def test_hbm_budget_admission(model4):
    """A server sized from an HBM budget: its arrays fit the budget, jobs are
    admitted while their atoms fit (a queue forms beyond that), every job
    completes, and a job denser than the budget's row length is refused."""
    budget = 512 << 20
    srv = TensorMDServer(model4, hbm_bytes=budget, max_density=0.09, max_cells=64,
                         steps_per_tick=4)
    fp = srv.footprint()
    assert fp["device_bytes"] <= budget and fp["max_atoms"] > 5000
    rng = np.random.default_rng(9)
    jobs = [synth.serving_job(rng, kind=1, nmin=2000, nmax=4000) for _ in range(12)]
    assert sum(len(j[0]) for j in jobs) > fp["max_atoms"]  # not all fit at once
    tks = [srv.submit(1, x, t, box, v=v, nsteps=12, dt=0.001) for x, t, box, v in jobs]
    for tk in tks:
        assert srv.wait(tk, timeout=300)["steps"] == 12
    st = srv.stats()
    assert st["completed"] == 12 and st["active_atoms"] <= fp["max_atoms"]
    # a compressed lattice (about 0.34 atoms/A^3) needs longer rows than the budget
    x, t, box, _ = synth.build_system("fcc", 2.3, (4, 4, 4), sigma=0.0, nelt=1, seed=1)
    with pytest.raises(TmdError) as e:
        srv.submit(0, x, t, box)
    assert e.value.code == -4
    assert srv.footprint()["row_length"] == fp["row_length"]
    srv.close()


def test_server_errors(model4):
    srv = TensorMDServer(model4, max_atoms=1000, max_cells=8)
    x, t, box, _ = synth.serving_job(np.random.default_rng(5), kind=0, nmin=64, nmax=64)
    with pytest.raises(TmdError) as e:
        srv.submit(7, x, t, box)
    assert e.value.code == -1
    big, tb, boxb, _ = synth.build_system("fcc", 3.6, (8, 8, 8))
    with pytest.raises(TmdError) as e:
        srv.submit(0, big, tb, boxb)
    assert e.value.code == -4
    # a periodic box too small for the cutoff (rc + skin = 7 A needs more
    # than 3 images of a 2 A box) is refused at submit; the server goes on
    tiny = np.array([[0.0, 0.0, 0.0], [1.0, 1.0, 1.0]])
    with pytest.raises(TmdError) as e:
        srv.submit(0, tiny, np.array([1, 1]), np.array([0, 0, 0, 2.0, 2.0, 2.0, 0, 0, 0]))
    assert e.value.code == -1 and "cutoff" in str(e.value)
    out = srv.wait(srv.submit(0, x, t, box), timeout=120)
    assert np.isfinite(out["energy"])
    tk = srv.submit(1, x, t, box, nsteps=200000, dt=0.001)
    with pytest.raises(TmdError) as e:
        srv.wait(tk, timeout=0.0)
    assert e.value.code == -8
    srv.close()  # stops with the job unfinished
