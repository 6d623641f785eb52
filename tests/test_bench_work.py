"""bench.py's algorithmic work per launch (the roofline numerators), on CPU.

Force step at the 128,000-atom benchmark shape (K = 16, D = 20, one element,
76.2 pairs inside rc per atom): per pair the U/V contractions 4 K D = 1,280,
radial 10 K = 160, F1 2K + 3 = 35, F2 2D + 3 = 43, monomial derivatives
6 D = 120 FLOP; per atom dE/dP (2M + 1) D K = 2,880 FLOP -> 127.7 kFLOP per
atom.  Bytes of the pair-lane form: per atom P 1,280 + G and dE/dG 512 +
virial 48 + active-pair counts 4 B, per pair 32 + 16 B."""
import sys
from pathlib import Path

import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
import bench  # noqa: E402


def test_force_step_work_at_the_benchmark_shape():
    n, pairs, nlist = 128000, 9_750_000, 15_500_000
    flops, nbytes = bench.algorithmic({"natoms": n}, pairs, nlist, 1, 16, 20, 64, "pair_lane8")
    per_pair = 4 * 16 * 20 + 10 * 16 + (2 * 16 + 3) + (2 * 20 + 3) + 6 * 20
    assert flops == pytest.approx(pairs * per_pair + n * 9 * 20 * 16)
    assert flops / n == pytest.approx(127.7e3, rel=2e-3)
    assert nbytes == n * (1280 + 512 + 48 + 4) + pairs * 48


def test_whole_job_value_of_replicas():
    # 4 replicas of 1,000 atoms, 10 steps each, the slowest took 2 ms
    assert bench.replicas_value(1000, 10, 4, 2.0) == pytest.approx(2.0e7)
