"""C-ABI library checks that need no GPU: it loads, exports every entry point
include/tmd_b200.h declares, and rejects bad pair_coeff arguments the way
PairTensorMD::coeff does (pair_tensormd.cpp:214-317) before touching a
device."""
import ctypes
import re

import pytest

from tmd_b200 import lib as tlib
from tmd_b200 import synth
from tmd_testutil import GOLDEN, ROOT


@pytest.fixture(scope="module")
def libtmd():
    if not tlib.library_path().exists():
        import build  # lammps-tensormd_b200/build.py
        build.build()
    return tlib.load_library()


def declared():
    txt = (ROOT / "include" / "tmd_b200.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:int|void|long)\s+(tmd_\w+)\s*\(", txt, re.M)))


def test_header_declares_entry_points():
    names = declared()
    assert "tmd_model_load" in names and "tmd_compute" in names and len(names) >= 15


def test_library_exports_every_declared_symbol(libtmd):
    for name in declared():
        assert hasattr(libtmd, name), name
    bound = {s[0] for s in tlib.SIGNATURES}
    assert bound == set(declared())


def _load(libtmd, args):
    h = ctypes.c_void_p()
    rc = libtmd.tmd_model_load(args.encode(), 0, ctypes.byref(h))
    buf = ctypes.create_string_buffer(512)
    libtmd.tmd_last_error(buf, 512)
    return rc, buf.value.decode()


def test_missing_file(libtmd, tmp_path):
    rc, msg = _load(libtmd, f"{tmp_path}/nope.npz Cu")
    assert rc == -6 and "cannot open" in msg


def test_bad_arguments(libtmd, tmp_path):
    p = tmp_path / "p.npz"
    synth.gaussian_potential(p, nelt=2, num_filters=8, hidden=(8, 8), symbols=["Cu", "Ni"])
    rc, msg = _load(libtmd, f"{p}")
    assert rc == -3 and "Incorrect args" in msg
    rc, msg = _load(libtmd, f"{p} Cu Xx")
    assert rc == -3 and "Xx" in msg
    rc, msg = _load(libtmd, f"{p} Cu Ni cmax bogus")
    assert rc == -3 and "cmax" in msg
    rc, msg = _load(libtmd, f"{p} Cu Ni interp 0.001 stray")
    assert rc == -3 and "stray" in msg
    rc, msg = _load(libtmd, f"{p} Cu Ni etemp -300")
    assert rc == -3 and "etemp" in msg
    # temperature-dependent files run the plain FP32 form only
    q = tmp_path / "t.npz"
    synth.tdnp_potential(q, nelt=2, symbols=["Cu", "Ni"])
    rc, msg = _load(libtmd, f"{q} Cu Ni etemp 3000 precision bf16")
    assert rc == -3 and "TDNP" in msg


def test_fnn_needs_interp(libtmd):
    rc, msg = _load(libtmd, f"{GOLDEN}/MoNi_m3.npz Mo Ni")
    assert rc == -3 and "interp" in msg


def test_filter_count_rule(libtmd, tmp_path):
    p = tmp_path / "k12.npz"
    synth.gaussian_potential(p, nelt=1, num_filters=12, hidden=(8, 8))
    rc, msg = _load(libtmd, f"{p} Cu")
    assert rc == -3 and "num_filters" in msg
