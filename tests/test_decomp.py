"""Spatial decomposition of one periodic cell over ranks (tmd_b200.decomp) on
the CPU: gloo ranks on 127.0.0.1, each rank's device system replaced by the
FP64 oracle evaluating its local atoms among its ghosts (the oracle's
nlocal mode; the product's ghost-aware device system is checked against the
periodic cell on the GPU in test_gpu_ghost.py).

The decomposition (slab ownership, ghost images, reverse communication of
ghost forces, energy/virial reductions, migration) must reproduce the
periodic oracle: forces, energy and virial of one evaluation to 1e-10
relative, and a 12-step NVE run (atoms migrate between slabs, ghost lists
are rebuilt) to 1e-9 A in positions.  World sizes 1 (a rank is its own
periodic neighbour), 2 and 3 (slabs of 9.6 A for a 6 A ghost cutoff)."""
import json
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class OracleRank:
    """Stand-in for a rank's device system: the oracle on the rank's local
    atoms and ghosts in a non-periodic box around them."""

    def __init__(self, oracle, cut):
        self.o, self.cut = oracle, cut

    def set_atoms_ghost(self, nlocal, x, types):
        self.nlocal, self.x, self.t = nlocal, np.array(x), np.array(types)

    def set_positions(self, x):
        self.x = np.array(x)

    def compute(self, eflag=1, vflag=1, peratom=False):
        lo = self.x.min(0) - 2 * self.cut
        box = np.concatenate([lo, np.ptp(self.x, 0) + 4 * self.cut, [0.0, 0.0, 0.0]])
        return self.o.compute(self.x, self.t - 1, box, [0, 0, 0], nlocal=self.nlocal)


def _setup():
    for p in (ROOT / "lammps-tensormd_b200", ROOT / "oracle", ROOT / "tests"):
        if str(p) not in sys.path:
            sys.path.insert(0, str(p))
    import tempfile

    from pack import Oracle, load_npz
    from tmd_b200 import synth
    p = Path(tempfile.mkdtemp()) / "d.npz"
    syms = synth.gaussian_potential(p, nelt=2, num_filters=8, rc=5.0, max_moment=3,
                                    hidden=(16, 16), actfn=2, seed=17)
    x, t, box, v = synth.build_system("fcc", 3.6, (8, 4, 4), sigma=0.05, T=600.0, nelt=2,
                                      seed=8)
    return Oracle(load_npz(p)), syms, x, t, box, v


def _rank(rank, world, port, outdir):
    import datetime
    import os

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    if world > 1:
        dist.init_process_group("gloo", rank=rank, world_size=world,
                                timeout=datetime.timedelta(seconds=120))
    o, syms, x, t, box, v = _setup()
    from tmd_b200.decomp import SlabDecomposition
    cut = o.rmax + 1.0
    dec = SlabDecomposition(box, cut, 1.0, OracleRank(o, cut), rank=rank, world=world,
                            rebuild_every=5)
    dec.set_atoms(x, t, v)
    f, e, vir = dec.compute()
    xg, vg, fg = dec.gather()
    masses = np.concatenate([[0.0], o.masses])
    pe = dec.nve_run(12, 0.002, masses)
    xn, vn, fn = dec.gather()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        Path(outdir, "out.json").write_text(json.dumps(
            {"f": fg.tolist(), "e": e, "vir": vir.tolist(), "x": xn.tolist(),
             "v": vn.tolist(), "pe": pe.tolist(), "nlocal": len(dec.x)}))


@pytest.mark.parametrize("world", [1, 2, 3])
def test_slab_ranks_equal_the_periodic_cell(tmp_path, world):
    port = _free_port()
    if world == 1:
        _rank(0, 1, port, str(tmp_path))
    else:
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=_rank, args=(r, world, port, str(tmp_path)))
                 for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=300)
            assert p.exitcode == 0
    out = json.loads((tmp_path / "out.json").read_text())
    o, syms, x, t, box, v = _setup()
    ref = o.compute(x, t - 1, box, [1, 1, 1])
    f = np.array(out["f"])
    assert np.abs(f - ref["f"]).max() <= 1e-10 * np.abs(ref["f"]).max()
    assert out["e"] == pytest.approx(ref["energy"], rel=1e-12)
    np.testing.assert_allclose(out["vir"], ref["virial"], rtol=1e-10, atol=1e-10)
    xo, vo, fo, tho = o.nve(x, v, t - 1, box, [1, 1, 1], 0.002, 12, skin=1.0)
    L = box[3:6]
    d = np.array(out["x"]) - xo
    d -= np.round(d / L) * L
    assert np.abs(d).max() < 1e-9
    assert out["pe"][-1] == pytest.approx(tho[-1, 0], rel=1e-10)
