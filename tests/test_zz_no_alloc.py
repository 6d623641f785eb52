"""tmd_neighbor_list_noalloc: the neighbor list for callers that may not
allocate device memory (code recorded into a CUDA graph, where cudaMalloc is
not allowed during capture, and hosts that manage all device memory through
their own pool).  The entry point uses only the buffers the caller passes and
the library's static 4 MiB scratch array.

Checked through the C ABI against the existing entry point
(tmd_system_* + tmd_neighbor_list): the same (i, j, image) set, bit for bit,
as every neighbor-set test here requires, on two calls in a row (the second
call finds the previous call's contents in the shared scratch array).  This
file sorts last so a failure here cannot hide the other tests."""
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


def _noalloc(x, box, pbc, cut, cap):
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
    assert rc == 0, rc
    return counts.cpu().numpy(), rows.cpu().numpy().view(np.uint32)


def _existing(pot_args, x, t, box, pbc, skin):
    m = TensorMDModel(pot_args)
    s = TensorMDSystem(m, len(x), skin)
    s.set_box(box, pbc)
    s.set_atoms(x, t)
    cut = m.cutmax + skin
    xs = s.get()[0]  # positions as the device holds them (inside the cell)
    return canonical_pairs(*s.neighbor_list(cut)), xs, cut


@pytest.mark.parametrize("case", ["fcc864", "triclinic16"])
def test_noalloc_list_equals_system_list(tmp_path, case):
    if case == "fcc864":
        p = tmp_path / "pot.npz"
        syms = synth.gaussian_potential(p, nelt=1, num_filters=8, rc=5.0, hidden=(8, 8))
        x, t, box, _ = synth.build_system("fcc", 3.6, (6, 6, 6), sigma=0.1, seed=9)
        args = f"{p} {' '.join(syms)}"
    else:
        x, t, box = read_data(GOLDEN / "Mo8_Ni8_id3210.data")
        x = frac_wrap(x, box)
        args = f"{GOLDEN}/MoNi_m3.npz Mo Ni interp 0.0001"
    ref, xs, cut = _existing(args, x, t, box, (1, 1, 1), 1.0)
    cap = 512
    for _ in range(2):  # second call reuses the scratch left by the first
        counts, rows = _noalloc(xs, box, (1, 1, 1), cut, cap)
        got = canonical_pairs(*_decode(counts, rows, cap))
        assert np.array_equal(got, ref)


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
