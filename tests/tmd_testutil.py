"""Shared helpers of the test suite (fixtures, data files, tolerances)."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
NKTV2P = 1.6021765e6  # metal units, update.cpp:187-206


def published():
    return json.loads((GOLDEN / "published.json").read_text())


def read_data(path):
    """Atoms of a LAMMPS data file (atomic style): x, types, box[9]."""
    lo = [0.0, 0.0, 0.0]
    prd = [0.0, 0.0, 0.0]
    tilt = [0.0, 0.0, 0.0]
    atoms = []
    sec = None
    for line in Path(path).read_text().splitlines():
        t = line.split()
        if "xlo" in line:
            lo[0], prd[0] = float(t[0]), float(t[1]) - float(t[0])
        elif "ylo" in line:
            lo[1], prd[1] = float(t[0]), float(t[1]) - float(t[0])
        elif "zlo" in line:
            lo[2], prd[2] = float(t[0]), float(t[1]) - float(t[0])
        elif "xy xz yz" in line:
            tilt = [float(t[0]), float(t[1]), float(t[2])]
        elif line.strip().startswith("Atoms"):
            sec = "atoms"
            continue
        elif line.strip() and line.strip()[0].isalpha():
            sec = None
        if sec == "atoms" and len(t) >= 5:
            atoms.append([int(t[0]), int(t[1]), float(t[2]), float(t[3]), float(t[4])])
    a = np.array(sorted(atoms, key=lambda r: r[0]))
    return a[:, 2:5].copy(), a[:, 1].astype(np.int32), np.array(lo + prd + tilt)


def frac_wrap(x, box):
    """Wrap positions into a (possibly triclinic) periodic cell."""
    lo = np.asarray(box[:3])
    xprd, yprd, zprd, xy, xz, yz = box[3:9]
    d = x - lo
    fz = d[:, 2] / zprd
    fy = (d[:, 1] - fz * yz) / yprd
    fx = (d[:, 0] - fy * xy - fz * xz) / xprd
    f = np.stack([fx, fy, fz], 1)
    s = np.floor(f)
    out = x.copy()
    out[:, 0] -= s[:, 0] * xprd + s[:, 1] * xy + s[:, 2] * xz
    out[:, 1] -= s[:, 1] * yprd + s[:, 2] * yz
    out[:, 2] -= s[:, 2] * zprd
    return out


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
