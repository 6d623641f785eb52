"""Seeded synthetic potentials and atom systems.

Potential files use the key layout the reference reads (nnp.cpp:110-145,
descriptor.h:45-85, tensormd.cpp:109-177, pair_tensormd.cpp:376-399), so the
same .npz drives the reference and this package.  Weights are random (no
trained checkpoint is available): N(0, 1/fan_in) with a fixed seed.

Lattices, displacements and Maxwell-Boltzmann velocities follow LAMMPS metal
units (update.cpp:187-206): boltz = 8.617343e-5 eV/K, mvv2e = 1.0364269e-4.
"""
from __future__ import annotations

import numpy as np
from pathlib import Path

BOLTZ = 8.617343e-5
MVV2E = 1.0364269e-4
NKTV2P = 1.6021765e6

SYMBOLS = ["Cu", "Ni", "Al", "Fe", "Mo", "W", "Ti", "Co"]
MASSES = {"Cu": 63.546, "Ni": 58.6934, "Al": 26.9815, "Fe": 55.845, "Mo": 95.95,
          "W": 183.84, "Ti": 47.867, "Co": 58.9332}


def gaussian_potential(path, *, nelt=1, num_filters=16, rc=6.0, max_moment=3,
                       hidden=(64, 64), actfn=2, resnet=0, seed=1234, symbols=None,
                       precision=64, fctype=0, output_bias=1):
    """Write an analytic (descriptor::method = 3, Gaussian SF) potential.

    Centers omega uniform on [0, rc]; eta so neighbouring Gaussians overlap at
    one standard deviation (sigma = spacing):  exp(-eta (r-omega)^2 / rc^2)."""
    rng = np.random.default_rng(seed)
    symbols = list(symbols or SYMBOLS[:nelt])
    K = num_filters
    M = max_moment + 1
    nin = nelt * K * M
    ft = np.float32 if precision == 32 else np.float64
    omega = np.linspace(0.0, rc, K)
    spacing = rc / (K - 1)
    eta = np.full(K, 0.5 * (rc / spacing) ** 2)
    sizes = [nin] + list(hidden) + [1]
    d = {
        "precision": np.int32(precision),
        "rmax": ft(rc),
        "nelt": np.int32(nelt),
        "max_moment": np.int32(max_moment),
        "masses": np.array([MASSES.get(s, 50.0) for s in symbols], dtype=ft),
        "numbers": np.array(sum(([ord(s[0]), ord(s[1]) if len(s) > 1 else 0]
                                 for s in symbols), []), dtype=np.int32),
        "tdnp": np.int32(0),
        "use_fnn": np.int32(0),
        "fctype": np.int32(fctype),
        "is_T_symmetric": np.int32(0),
        "descriptor::method": np.int32(3),
        "descriptor::eta": eta.astype(ft),
        "descriptor::omega": omega.astype(ft),
        "nlayers": np.int32(len(sizes) - 1),
        "actfn": np.int32(actfn),
        "layer_sizes": np.array(sizes[1:], dtype=np.int32),
        "use_resnet_dt": np.int32(resnet),
        "apply_output_bias": np.int32(output_bias),
    }
    for e in range(nelt):
        for l in range(len(sizes) - 1):
            w = rng.normal(0.0, 1.0 / np.sqrt(sizes[l]), size=(sizes[l], sizes[l + 1]))
            d[f"weights_{e}_{l}"] = (w if sizes[l + 1] > 1 else w[:, 0]).astype(ft)
            if l < len(sizes) - 2 or output_bias:
                b = rng.normal(0.0, 0.1, size=sizes[l + 1])
                d[f"biases_{e}_{l}"] = (b if sizes[l + 1] > 1 else b.reshape(())).astype(ft)
    np.savez(path, **d)
    return symbols


def tdnp_potential(path, *, nelt=1, num_filters=8, rc=5.0, max_moment=3, h_hidden=(32,),
                   ydim=8, u_hidden=(16,), s_hidden=(16,), actfn=1, sommerfeld=0, seed=77,
                   symbols=None):
    """Write a temperature-dependent (tdnp = 1) potential with random weights:
    the Gaussian descriptor of gaussian_potential, and three nets per element
    in the layout tdnp.cpp reads (H::*, U::*, S::*; tdnp::Sommerfeld): H maps
    the descriptor to ydim - 1 values (the reference appends the electron
    temperature as column ydim - 1), U and S map the ydim values to the
    atom's internal energy and entropy.  No main NNP keys (TDNP replaces it)."""
    rng = np.random.default_rng(seed)
    symbols = gaussian_potential(path, nelt=nelt, num_filters=num_filters, rc=rc,
                                 max_moment=max_moment, hidden=(4,), actfn=actfn,
                                 seed=seed, symbols=symbols)
    with np.load(path) as z:
        d = {k: z[k] for k in z.files if not (k.startswith(("weights_", "biases_"))
                                               or k in ("nlayers", "actfn", "layer_sizes",
                                                        "use_resnet_dt", "apply_output_bias"))}
    d["tdnp"] = np.int32(1)
    d["tdnp::Sommerfeld"] = np.int32(sommerfeld)
    nin = nelt * num_filters * (max_moment + 1)
    nets = {"H": [nin] + list(h_hidden) + [ydim - 1],
            "U": [ydim] + list(u_hidden) + [1],
            "S": [ydim] + list(s_hidden) + [1]}
    for scope, sizes in nets.items():
        d[f"{scope}::nlayers"] = np.int32(len(sizes) - 1)
        d[f"{scope}::layer_sizes"] = np.array(sizes[1:], dtype=np.int32)
        d[f"{scope}::actfn"] = np.int32(actfn)
        d[f"{scope}::use_resnet_dt"] = np.int32(0)
        d[f"{scope}::apply_output_bias"] = np.int32(1)
        for e in range(nelt):
            for l in range(len(sizes) - 1):
                w = rng.normal(0.0, 1.0 / np.sqrt(sizes[l]), size=(sizes[l], sizes[l + 1]))
                d[f"{scope}::weights_{e}_{l}"] = (w if sizes[l + 1] > 1 else w[:, 0])
                b = rng.normal(0.0, 0.1, size=sizes[l + 1])
                d[f"{scope}::biases_{e}_{l}"] = b if sizes[l + 1] > 1 else b.reshape(())
    np.savez(path, **d)
    return symbols


def _lattice_basis(kind):
    if kind == "fcc":
        return np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    if kind == "bcc":
        return np.array([[0, 0, 0], [0.5, 0.5, 0.5]])
    if kind == "sc":
        return np.array([[0.0, 0.0, 0.0]])
    raise ValueError(kind)


def lattice(kind, a, nx, ny, nz):
    """Positions of an orthogonal nx x ny x nz lattice and its box[9]."""
    basis = _lattice_basis(kind)
    g = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz),
                             indexing="ij"), -1).reshape(-1, 3)
    x = (g[:, None, :] + basis[None, :, :]).reshape(-1, 3) * a
    box = np.array([0.0, 0.0, 0.0, nx * a, ny * a, nz * a, 0.0, 0.0, 0.0])
    return x, box


def wrap(x, box):
    """Wrap positions into an orthogonal box (Domain::remap for orthogonal)."""
    lo = box[:3]
    prd = box[3:6]
    return lo + np.mod(x - lo, prd)


def maxwell(masses, T, rng):
    """Velocities (A/ps) drawn from Maxwell-Boltzmann at T, zero momentum, then
    scaled so the temperature with dof = 3N - 3 is exactly T (LAMMPS
    velocity create ... dist gaussian, mom yes, rot no)."""
    n = len(masses)
    v = rng.normal(size=(n, 3)) / np.sqrt(masses)[:, None]
    p = (masses[:, None] * v).sum(0) / masses.sum()
    v -= p
    ke = 0.5 * MVV2E * (masses[:, None] * v * v).sum()
    dof = 3 * n - 3
    t_now = 2.0 * ke / (dof * BOLTZ) if dof > 0 else 0.0
    if t_now > 0:
        v *= np.sqrt(T / t_now)
    return v


def temperature(masses, v):
    n = len(masses)
    ke = 0.5 * MVV2E * (masses[:, None] * v * v).sum()
    return 2.0 * ke / ((3 * n - 3) * BOLTZ)


def build_system(kind, a, cells, *, sigma=0.0, T=0.0, nelt=1, seed=7, masses=None):
    """Lattice + Gaussian displacements + random equal-fraction occupancy.

    Returns x, types (1-based), box, v."""
    rng = np.random.default_rng(seed)
    x, box = lattice(kind, a, *cells)
    n = len(x)
    if sigma > 0:
        x = x + rng.normal(0.0, sigma, size=x.shape)
        x = wrap(x, box)
    if nelt > 1:
        types = (np.arange(n) % nelt) + 1
        rng.shuffle(types)
    else:
        types = np.ones(n, dtype=np.int32)
    types = types.astype(np.int32)
    v = np.zeros_like(x)
    if T > 0:
        m = np.ones(n) * 50.0 if masses is None else np.asarray(masses)[types - 1]
        v = maxwell(m, T, rng)
    return x, types, box, v


def batch_cells(ncells=4096, natoms=256, *, nelt=2, sigma=0.1, t_range=(300.0, 1200.0),
                seed=11, masses=None):
    """Multi-cell workload: half FCC (a = 3.6 A, 4x4x4 cells), half BCC
    (a = 2.87 A, 4x4x8 cells), natoms = 256 atoms each, random equal-fraction
    occupancy of nelt elements, Gaussian displacements sigma, per-cell
    temperature uniform in t_range.  Returns per-cell lists
    (x, types, box, v) and the concatenated arrays."""
    if natoms != 256:
        raise ValueError("the FCC/BCC cells of this workload hold 256 atoms")
    rng = np.random.default_rng(seed)
    xs, ts, boxes, vs = [], [], [], []
    m_el = np.asarray(masses if masses is not None
                      else [MASSES[s] for s in SYMBOLS[:nelt]], dtype=np.float64)
    for c in range(ncells):
        if c % 2 == 0:
            x, box = lattice("fcc", 3.6, 4, 4, 4)
        else:
            x, box = lattice("bcc", 2.87, 4, 4, 8)
        n = len(x)
        x = wrap(x + rng.normal(0.0, sigma, size=x.shape), box)
        t = (np.arange(n) % nelt) + 1
        rng.shuffle(t)
        T = rng.uniform(*t_range)
        v = maxwell(m_el[t - 1], T, rng)
        xs.append(x); ts.append(t.astype(np.int32)); boxes.append(box); vs.append(v)
    return dict(x=np.concatenate(xs), types=np.concatenate(ts), boxes=np.stack(boxes),
                v=np.concatenate(vs), natoms=np.full(ncells, 256, dtype=np.int32),
                cells=list(zip(xs, ts, boxes, vs)))


def random_packing(n, rng, density=0.085, dmin=2.0, h=0.25, attempts=5):
    """n atoms in a periodic cube at `density` (1/A^3), no pair closer than
    dmin: random sequential addition (rejection sampling).  0.085 A^-3 with
    dmin = 2 A is a volume fraction of 0.356, close to the jamming limit of
    sequential addition (about 0.38), where uniform candidates are almost all
    rejected; candidates are therefore drawn uniformly inside voxels (side ~h)
    that no accepted atom fully excludes yet, then tested exactly against the
    accepted atoms and the round's earlier candidates.  Returns x[n, 3], box[9]."""
    from scipy.spatial import cKDTree
    L = (n / density) ** (1.0 / 3.0)
    g = max(1, int(np.ceil(L / h)))
    h = L / g
    # voxel offsets entirely within dmin of any point of the centre voxel
    r = int(np.ceil(dmin / h))
    o = np.stack(np.meshgrid(*(np.arange(-r, r + 1),) * 3, indexing="ij"), -1).reshape(-1, 3)
    o = o[np.linalg.norm(o, axis=1) * h + h * np.sqrt(3.0) < dmin]
    for _ in range(attempts):
        free = np.ones(g ** 3, dtype=bool)
        pts = np.zeros((0, 3))
        while len(pts) < n:
            fi = np.flatnonzero(free)
            if len(fi) == 0:
                break
            m = min(len(fi), max(2048, 4 * (n - len(pts))))
            pick = np.unique(fi[rng.integers(len(fi), size=m)])
            m = len(pick)
            vox = np.stack(np.unravel_index(pick, (g, g, g)), -1)
            cand = (vox + rng.uniform(size=(m, 3))) * h
            if len(pts):
                d, _ = cKDTree(pts, boxsize=L).query(cand, k=1)
                ok = d >= dmin
                free[pick[~ok & (d < dmin - h * np.sqrt(3.0))]] = False
                cand, vox = cand[ok], vox[ok]
            taken = np.ones(len(cand), dtype=bool)
            if len(cand) > 1:
                close = cKDTree(cand, boxsize=L).query_pairs(dmin, output_type="ndarray")
                if len(close):
                    taken[np.max(close, axis=1)] = False  # the later one of a close pair
            keep = np.nonzero(taken)[0][: n - len(pts)]
            pts = np.concatenate([pts, cand[keep]])
            blk = (vox[keep][:, None, :] + o[None, :, :]) % g
            free[np.ravel_multi_index((blk[..., 0], blk[..., 1], blk[..., 2]), (g, g, g))] = False
        if len(pts) >= n:
            return pts, np.array([0.0, 0.0, 0.0, L, L, L, 0.0, 0.0, 0.0])
    raise RuntimeError("random packing did not reach the requested density")


def _near_cubic(cells):
    """nx, ny, nz with nx*ny*nz close to `cells`, as cubic as possible."""
    c = max(1, int(round(cells)))
    best = (1, 1, c)
    for nx in range(1, int(round(c ** (1 / 3))) + 2):
        for ny in range(nx, int(round((c / nx) ** 0.5)) + 2):
            nz = max(ny, int(round(c / (nx * ny))))
            if abs(nx * ny * nz - c) < abs(best[0] * best[1] * best[2] - c) or (
                    nx * ny * nz == best[0] * best[1] * best[2] and nz - nx < best[2] - best[0]):
                best = (nx, ny, nz)
    return best


def serving_job(rng, *, kind, nmin=32, nmax=4096, max_elements=4, packings=None):
    """One job of the serving workload: N log-uniform in [nmin, nmax], an FCC
    (a = 3.6 A) or BCC (a = 2.87 A) lattice or a random packing (0.085 A^-3,
    dmin 2 A; `packings` may hold prepared ones by size), 1..max_elements
    elements.  NVE jobs get Maxwell-Boltzmann velocities at T in [300, 1200] K
    and FIRE jobs displaced positions (sigma 0.1 A).  Returns x, types, box, v."""
    n = int(round(np.exp(rng.uniform(np.log(nmin), np.log(nmax)))))
    shape = rng.integers(3)
    if shape == 0:
        x, box = lattice("fcc", 3.6, *_near_cubic(n / 4))
    elif shape == 1:
        x, box = lattice("bcc", 2.87, *_near_cubic(n / 2))
    else:
        if packings:
            sizes = np.array(sorted(packings))
            x, box = packings[int(sizes[np.argmin(np.abs(sizes - n))])]
        else:
            x, box = random_packing(n, rng)
    n = len(x)
    ne = int(rng.integers(1, max_elements + 1))
    types = rng.integers(1, ne + 1, size=n).astype(np.int32)
    v = np.zeros_like(x)
    if kind == 2:
        x = wrap(x + rng.normal(0.0, 0.1, size=x.shape), box)
    else:
        x = wrap(x + rng.normal(0.0, 0.05, size=x.shape), box)
    if kind == 1:
        m = np.array([MASSES[s] for s in SYMBOLS[:max_elements]])[types - 1]
        v = maxwell(m, rng.uniform(300.0, 1200.0), rng)
    return x, types, box, v


def config(name):
    """The workloads this path is measured on (shapes from the task spec)."""
    if name == "fcc4k":  # plain CPU config: 4,000 atoms
        return dict(kind="fcc", a=3.61, cells=(10, 10, 10), sigma=0.05, T=300.0, nelt=1,
                    pot=dict(nelt=1, num_filters=16, rc=6.0, max_moment=3,
                             hidden=(64, 64), actfn=2))
    if name == "bcc128k":  # plain FP32 GPU config: 128,000 atoms
        return dict(kind="bcc", a=2.87, cells=(40, 40, 40), sigma=0.08, T=600.0, nelt=1,
                    pot=dict(nelt=1, num_filters=16, rc=6.0, max_moment=3,
                             hidden=(64, 64), actfn=2))
    if name == "cells4096":  # batched config: 4,096 cells x 256 atoms, 2 elements
        return dict(kind="cells", ncells=4096, natoms=256, sigma=0.1, t_range=(300.0, 1200.0),
                    nelt=2, pot=dict(nelt=2, num_filters=16, rc=6.0, max_moment=3,
                                     hidden=(64, 64), actfn=2))
    if name == "alloy432k":  # precision config: 4 elements, 432,000 atoms
        return dict(kind="fcc", a=3.6, cells=(60, 60, 30), sigma=0.05, T=300.0, nelt=4,
                    pot=dict(nelt=4, num_filters=32, rc=6.5, max_moment=3,
                             hidden=(128, 128, 128), actfn=1))
    if name == "alloy55k":  # the precision config's potential on 55,296 atoms (profiling)
        c = config("alloy432k")
        c["cells"] = (24, 24, 24)
        return c
    raise KeyError(name)


def read_data(path):
    """Atoms of a LAMMPS data file (atomic style): x, types, box[9]
    (lo xyz, lengths, tilts xy xz yz)."""
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
