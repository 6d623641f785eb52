"""Failure detection of the tensor-core MLP kernels, without a GPU fault.

Every mbarrier wait in the tcgen05 kernels is bounded; a wait that runs out
sets a status bit, the kernel drains what it issued, frees its TMEM and
returns, and tmd_compute reports TMD_ERR_TIMEOUT.  tmd_system_set_wait_probe
makes every CTA first wait, with a short limit, on a barrier that nothing
arrives on, before it issues any MMA or copy: the timeout path runs with no
asynchronous work in flight.  Each kernel form must then report the timeout,
and the same system must compute the same results as before once the probe
is off (the context stays usable).
"""
import numpy as np
import pytest

from tmd_b200 import TensorMDModel, TensorMDSystem, TmdError, synth

pytestmark = pytest.mark.gpu

TMD_ERR_TIMEOUT = -8

CASES = {
    # weight-resident persistent kernel (k_mlp_tcp)
    "persistent-bf16": (dict(nelt=1, num_filters=16, rc=6.0, max_moment=3, hidden=(64, 64),
                             actfn=2), "bf16"),
    "persistent-bf16x3": (dict(nelt=1, num_filters=16, rc=6.0, max_moment=3,
                               hidden=(64, 64), actfn=2), "bf16x3"),
    # streamed-weight persistent kernel (k_mlp_tcs): 512-128-128-128 per element
    "streamed-bf16": (dict(nelt=4, num_filters=32, rc=6.5, max_moment=3,
                           hidden=(128, 128, 128), actfn=1), "bf16"),
    # one CTA per tile (k_mlp_tc): residual layers
    "tiled-residual": (dict(nelt=1, num_filters=16, rc=6.0, max_moment=3,
                            hidden=(64, 64, 64), actfn=1, resnet=1), "bf16"),
    # FP8 kernel (k_mlp_fp8)
    "fp8": (dict(nelt=1, num_filters=16, rc=6.0, max_moment=3, hidden=(64, 64), actfn=2),
            "fp8"),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_wait_timeout_is_reported_and_recovers(tmp_path, case):
    kw, prec = CASES[case]
    p = tmp_path / "pot.npz"
    syms = synth.gaussian_potential(p, seed=5, **kw)
    x, t, box, _ = synth.build_system("fcc", 3.6, (6, 6, 6), sigma=0.05, nelt=kw["nelt"],
                                      seed=3)
    m = TensorMDModel(f"{p} {' '.join(syms)} precision {prec}")
    s = TensorMDSystem(m, len(x), 1.0)
    s.set_box(box)
    s.set_atoms(x, t)
    ref = s.compute(1, 1)
    assert s.lib.tmd_system_set_wait_probe(s.h, 2000) == 0
    with pytest.raises(TmdError) as err:
        s.compute(1, 1)
    assert err.value.code == TMD_ERR_TIMEOUT
    assert s.lib.tmd_system_set_wait_probe(s.h, 0) == 0
    again = s.compute(1, 1)
    assert np.array_equal(again["f"], ref["f"])
    assert again["energy"] == ref["energy"]
