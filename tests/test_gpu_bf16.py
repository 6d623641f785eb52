"""Tensor-core MLP (tcgen05, BF16 operands) against the FP64 oracle.

Two forms run the MLP GEMMs on the tensor cores with FP32 accumulation in
tensor memory; descriptors, the force contraction, the output layer and all
sums keep their FP32/FP64 precision:
  bf16x3  split BF16 products (hi*hi + hi*lo + lo*hi), about 17 significant
          bits per operand.  Bounds: force RMS error <= 1e-3 eV/A (the target
          of the precision study), energy <= 1e-4 eV/atom, virial relative
          error <= 1e-2.  Measured on the 4,000-atom FCC case: 3.6e-4 eV/A,
          5.8e-6 eV/atom, 3.5e-3.
  bf16    single BF16 products.  On these random-weight potentials the
          first layer (descriptor x weights) dominates the error.  Bounds:
          force RMS <= 8e-3 eV/A, energy <= 5e-3 eV/atom, virial relative
          error <= 5e-2.  Measured: 4.0e-3 eV/A, 3.3e-3 eV/atom, 2.1e-2 (FCC);
          2.0e-3 eV/A, 2.4e-3 eV/atom, 2.8e-2 (MoNi_m3).
"""
import numpy as np
import pytest

from pack import Oracle, load_npz
from tmd_b200 import TensorMDModel, TensorMDSystem, synth
from tmd_testutil import GOLDEN, frac_wrap, read_data

pytestmark = pytest.mark.gpu

BOUNDS = {"bf16x3": (1e-3, 1e-4, 1e-2), "bf16": (8e-3, 5e-3, 5e-2)}


def _run(args, prec, x, t, box):
    m = TensorMDModel(args + f" precision {prec}")
    s = TensorMDSystem(m, len(x), 1.0)
    s.set_box(box)
    s.set_atoms(x, t)
    return s, s.compute(1, 1, peratom=True)


def _errors(out, ref, n):
    frms = float(np.sqrt(np.mean((out["f"] - ref["f"]) ** 2)))
    de = abs(out["energy"] - ref["energy"]) / n
    vr = float(np.linalg.norm(out["virial"] - ref["virial"]) / np.linalg.norm(ref["virial"]))
    return frms, de, vr


def _assert_bounds(prec, errs):
    fb, eb, vb = BOUNDS[prec]
    frms, de, vr = errs
    assert frms <= fb, (prec, errs)
    assert de <= eb, (prec, errs)
    assert vr <= vb, (prec, errs)


@pytest.fixture(scope="module")
def fcc4k(tmp_path_factory):
    c = synth.config("fcc4k")
    p = tmp_path_factory.mktemp("pot") / "fcc4k.npz"
    syms = synth.gaussian_potential(p, seed=1234, **c["pot"])
    x, t, box, _ = synth.build_system(c["kind"], c["a"], c["cells"], sigma=c["sigma"],
                                      nelt=1, seed=42)
    ref = Oracle(str(p)).compute(x, t - 1, box, [1, 1, 1], skin=1.0)
    return str(p), syms, x, t, box, ref


@pytest.mark.parametrize("prec", ["bf16x3", "bf16"])
def test_tc_fcc4k(fcc4k, prec):
    p, syms, x, t, box, ref = fcc4k
    _, out = _run(f"{p} {' '.join(syms)}", prec, x, t, box)
    _assert_bounds(prec, _errors(out, ref, len(x)))


@pytest.mark.parametrize("prec", ["bf16x3", "bf16"])
def test_tc_residual_wide_descriptor(prec):
    """MoNi_m3: 512 descriptor columns (backward output in 4 chunks),
    residual softplus MLP, two elements."""
    x, t, box = read_data(GOLDEN / "Mo8_Ni8_id3210.data")
    x = frac_wrap(x, box)
    _, out = _run(f"{GOLDEN}/MoNi_m3.npz Mo Ni interp 0.0001", prec, x, t, box)
    ref = Oracle(str(GOLDEN / "MoNi_m3.npz"), interp=1e-4).compute(x, t - 1, box, [1, 1, 1])
    _assert_bounds(prec, _errors(out, ref, len(x)))


def test_tc_deterministic(fcc4k):
    p, syms, x, t, box, _ = fcc4k
    s, a = _run(f"{p} {' '.join(syms)}", "bf16", x, t, box)
    b = s.compute(1, 1, peratom=True)
    assert np.array_equal(a["f"], b["f"]) and a["energy"] == b["energy"]


def test_tc_partial_tiles(tmp_path):
    """Atom counts that are not multiples of the 128-atom tile, two elements."""
    p = tmp_path / "two.npz"
    syms = synth.gaussian_potential(p, nelt=2, num_filters=8, rc=5.0, hidden=(64, 64),
                                    actfn=2, seed=4)
    x, t, box, _ = synth.build_system("bcc", 2.9, (5, 5, 5), sigma=0.1, nelt=2, seed=2)
    _, out = _run(f"{p} {' '.join(syms)}", "bf16x3", x, t, box)
    ref = Oracle(load_npz(p)).compute(x, t - 1, box, [1, 1, 1], skin=1.0)
    _assert_bounds("bf16x3", _errors(out, ref, len(x)))
