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


def kinetic_pressure(natoms, temp, vol):
    """Kinetic part of LAMMPS's pressure in bar: dof k_B T / (3 V) with
    dof = 3 N - 3 (ComputeTemp::dof_compute, compute_temp.cpp:58-62, extra_dof
    = dimension, compute.cpp:84) and metal k_B (update.cpp:188)."""
    return (3 * natoms - 3) * 8.617343e-5 * temp / (3 * vol) * NKTV2P


def bcc_lattice(a, nx, ny, nz):
    """Perfect BCC cells (LAMMPS `lattice bcc a` + `create_atoms`): positions
    and the orthogonal box as (xlo, ylo, zlo, xhi, yhi, zhi, xy, xz, yz)."""
    g = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"),
                 -1).reshape(-1, 3).astype(float)
    x = np.concatenate([g, g + 0.5]) * a
    return x, np.array([0, 0, 0, nx * a, ny * a, nz * a, 0, 0, 0], dtype=float)


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
