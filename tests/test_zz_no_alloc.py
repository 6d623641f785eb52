"""tmd_neighbor_list_noalloc: the neighbor list for host programs that may not
let a library allocate device memory (they manage every byte through their
own pool, or reserve the whole device up front).  The entry point uses only
the buffers the caller passes and the library's static 4 MiB scratch array;
it is synchronous and is called outside any stream capture.

Checked through the C ABI against the existing entry point
(tmd_system_* + tmd_neighbor_list): the same (i, j, image) set, bit for bit,
as every neighbor-set test here requires, on two calls in a row (the second
call finds the previous call's contents in the shared scratch array), for
periodic, slab and cluster cells and for a sparse box whose bins must be
merged to fit the scratch array's cell limit.  This file sorts last so a
failure here cannot hide the other tests."""
import ctypes

import numpy as np
import pytest

from tmd_b200 import TensorMDModel, TensorMDSystem, synth
from tmd_b200.lib import load_library
from tmd_testutil import GOLDEN, canonical_pairs, frac_wrap, read_data

pytestmark = pytest.mark.gpu

_pd = ctypes.POINTER(ctypes.c_double)
_pi = ctypes.POINTER(ctypes.c_int)


def _decode(counts, rows, cap):
    n = len(counts)
    off = np.zeros(n + 1, dtype=np.int64)
    off[1:] = np.cumsum(counts)
    ent = np.zeros((off[-1], 4), dtype=np.int32)
    for i in range(n):
        e = rows[i * cap:i * cap + counts[i]].astype(np.int64)
        code = e >> 23
        ent[off[i]:off[i + 1], 0] = e & 0x7FFFFF
        ent[off[i]:off[i + 1], 1] = code % 7 - 3
        ent[off[i]:off[i + 1], 2] = (code // 7) % 7 - 3
        ent[off[i]:off[i + 1], 3] = code // 49 - 3
    return off, ent


def _noalloc(x, box, pbc, cut, cap, expect=0):
    import torch
    lib = load_library()
    n = len(x)
    xd = torch.tensor(np.ascontiguousarray(x), dtype=torch.float64, device="cuda")
    counts = torch.zeros(n, dtype=torch.int32, device="cuda")
    rows = torch.zeros(n * cap, dtype=torch.int32, device="cuda")
    bx = np.ascontiguousarray(box, dtype=np.float64)
    pb = np.ascontiguousarray(pbc, dtype=np.int32)
    torch.cuda.synchronize()
    rc = lib.tmd_neighbor_list_noalloc(ctypes.c_void_p(xd.data_ptr()), n, bx.ctypes.data_as(_pd),
                                       pb.ctypes.data_as(_pi), cut, cap,
                                       ctypes.c_void_p(counts.data_ptr()),
                                       ctypes.c_void_p(rows.data_ptr()), None)
    assert rc == expect, rc
    return counts.cpu().numpy(), rows.cpu().numpy().view(np.uint32)


def _existing(pot_args, x, t, box, pbc, skin):
    m = TensorMDModel(pot_args)
    s = TensorMDSystem(m, len(x), skin)
    s.set_box(box, pbc)
    s.set_atoms(x, t)
    cut = m.cutmax + skin
    xs = s.get()[0]  # positions as the device holds them (inside the cell)
    return canonical_pairs(*s.neighbor_list(cut)), xs, cut


def _small_pot(tmp_path, rc=5.0):
    p = tmp_path / "pot.npz"
    syms = synth.gaussian_potential(p, nelt=1, num_filters=8, rc=rc, hidden=(8, 8))
    return f"{p} {' '.join(syms)}"


@pytest.mark.parametrize("case", ["fcc864", "triclinic16", "slab", "cluster", "sparse"])
def test_noalloc_list_equals_system_list(tmp_path, case):
    pbc = (1, 1, 1)
    if case == "triclinic16":
        x, t, box = read_data(GOLDEN / "Mo8_Ni8_id3210.data")
        x = frac_wrap(x, box)
        args = f"{GOLDEN}/MoNi_m3.npz Mo Ni interp 0.0001"
    elif case == "sparse":
        # 3,000 atoms in a periodic 200 A cube: bins of cut/2 would give
        # 57^3 = 185,193 cells, more than the scratch array holds, so the
        # call merges bins until the grid fits
        args = _small_pot(tmp_path, rc=6.0)
        rng = np.random.default_rng(5)
        box = np.array([0, 0, 0, 200.0, 200.0, 200.0, 0, 0, 0])
        x = rng.uniform(0.0, 200.0, size=(3000, 3))
        t = np.ones(len(x), dtype=np.int32)
    else:
        args = _small_pot(tmp_path)
        x, t, box, _ = synth.build_system("fcc", 3.6, (6, 6, 6), sigma=0.1, seed=9)
        if case != "fcc864":
            # non-periodic axes: a box 2 A wider than the atoms on each side;
            # one atom sits exactly on the upper face of the first free axis
            pbc = (1, 1, 0) if case == "slab" else (0, 0, 0)
            box = box.copy()
            for a in range(3):
                if not pbc[a]:
                    lo = x[:, a].min() - 2.0
                    box[a], box[3 + a] = lo, x[:, a].max() + 2.0 - lo
            a = 2
            x = x.copy()
            x[0, a] = box[a] + box[3 + a]
    ref, xs, cut = _existing(args, x, t, box, pbc, 1.0)
    cap = 512
    for _ in range(2):  # second call reuses the scratch left by the first
        counts, rows = _noalloc(xs, box, pbc, cut, cap)
        got = canonical_pairs(*_decode(counts, rows, cap))
        assert np.array_equal(got, ref)


def test_noalloc_row_overflow_reports_needed_length(tmp_path):
    args = _small_pot(tmp_path)
    x, t, box, _ = synth.build_system("fcc", 3.6, (6, 6, 6), sigma=0.1, seed=9)
    ref, xs, cut = _existing(args, x, t, box, (1, 1, 1), 1.0)
    longest = int(np.bincount(ref[:, 0]).max())
    _noalloc(xs, box, (1, 1, 1), cut, 16, expect=-4)
    buf = ctypes.create_string_buffer(256)
    load_library().tmd_last_error(buf, 256)
    assert f"needs {longest} entries".encode() in buf.value, buf.value


def test_noalloc_rejects_sizes_beyond_its_limit():
    lib = load_library()
    box = np.array([0, 0, 0, 10.0, 10.0, 10.0, 0, 0, 0])
    pbc = np.ones(3, dtype=np.int32)
    too_many = 262144 + 1
    dummy = ctypes.c_void_p(1)  # never dereferenced: the size check comes first
    rc = lib.tmd_neighbor_list_noalloc(dummy, too_many, box.ctypes.data_as(_pd),
                                       pbc.ctypes.data_as(_pi), 7.0, 64, dummy, dummy, None)
    assert rc == -4
    buf = ctypes.create_string_buffer(256)
    lib.tmd_last_error(buf, 256)
    assert b"limit" in buf.value
