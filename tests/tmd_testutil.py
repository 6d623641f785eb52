"""Shared helpers of the test suite (fixtures, data files, tolerances)."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

from tmd_b200.synth import frac_wrap, read_data  # noqa: F401  (re-exported)

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
NKTV2P = 1.6021765e6  # metal units, update.cpp:187-206


def published():
    return json.loads((GOLDEN / "published.json").read_text())


def volume(box):
    return box[3] * box[4] * box[5]


def canonical_pairs(off, ent):
    """Sorted (i, j, sx, sy, sz) tuples of a neighbor list."""
    n = len(off) - 1
    i = np.repeat(np.arange(n), np.diff(off))
    t = np.concatenate([i[:, None], ent[:, :4]], 1).astype(np.int64)
    order = np.lexsort(t.T[::-1])
    return t[order]


def rel_rms(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(np.sqrt(np.mean((a - b) ** 2)) / max(np.sqrt(np.mean(b ** 2)), 1e-300))
