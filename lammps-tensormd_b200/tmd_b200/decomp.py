"""Spatial decomposition of one periodic cell over ranks, one GPU each.

The reference runs large cells under LAMMPS's MPI domain decomposition: each
rank owns the atoms of its subdomain, receives ghost copies of the atoms
within the ghost cutoff (border exchange), evaluates its local atoms over a
full list that includes the ghosts (pair_tensormd.cpp:141-184), writes forces
on ghosts and sends them back to their owners (reverse communication, with
the force sum of kernel.cu:1760-1789).  Here the same decomposition drives the
ghost-aware device system (tmd_system_set_atoms_ghost) of each rank:

  * the cell (orthogonal, periodic in x, y and z) is cut into `world` slabs
    along x; rank r owns the atoms with lo_r <= x < hi_r (wrapped), each slab
    at least `cut` wide;
  * ghosts of a rank are every periodic image of an atom that lies within
    `cut` (rc + skin) of its slab and is not one of its own local atoms
    (shift 0): images of its own atoms across the y and z faces (and the x
    faces when it holds the whole cell), and the other ranks' boundary atoms
    (those within `cut` of their slab's x faces), which every rank shares by
    one all-gather per exchange;
  * after the force evaluation the forces on ghosts go home: images of own
    atoms are summed locally, forces on other ranks' boundary atoms are added
    into a buffer over the gathered boundary atoms that one all-reduce sums;
  * energy and virial: one all-reduce of 7 numbers.

Between re-decompositions (atom migration and new ghost lists, at most every
`rebuild_every` steps and whenever an atom moved more than skin/2) the ghost
set is kept and only positions travel (the gathered boundary atoms' new
positions, the same images), as LAMMPS's forward communication does.  The
collectives run over torch.distributed (NCCL over NVLink between GPUs, gloo
on the host); no collective runs inside a kernel.

`backend` is the rank's device system: an object with set_atoms_ghost(nlocal,
x, types), set_positions(x) and compute(eflag, vflag, peratom=False) returning
dict(f, energy, virial) for all of its atoms (tmd_b200.TensorMDSystem).
"""
from __future__ import annotations

import numpy as np

from .synth import MVV2E

__all__ = ["slab_ghosts", "SlabDecomposition"]


def slab_ghosts(cand_x, cand_owner, local_mask, box, lo, hi, cut):
    """Ghost images of candidate atoms for the slab lo <= x < hi of an
    orthogonal periodic box: every image cand_x[k] + s * L (s in Z^3, formed
    in FP64 as LAMMPS's pack_border adds the box length) inside
    [lo - cut, hi + cut) x [ylo - cut, yhi + cut) x [zlo - cut, zhi + cut),
    except the local atoms themselves (local_mask[k] and s = 0).  Returns
    (positions[m, 3], candidate index[m], shift[m, 3])."""
    L = np.asarray(box[3:6], dtype=np.float64)
    b0 = np.asarray(box[:3], dtype=np.float64)
    ext_lo = np.array([lo - cut, b0[1] - cut, b0[2] - cut])
    ext_hi = np.array([hi + cut, b0[1] + L[1] + cut, b0[2] + L[2] + cut])
    reach = [int(np.ceil(cut / L[a])) + 1 for a in range(3)]
    px, pk, ps = [], [], []
    for sx in range(-reach[0], reach[0] + 1):
        for sy in range(-reach[1], reach[1] + 1):
            for sz in range(-reach[2], reach[2] + 1):
                s = np.array([sx, sy, sz])
                p = cand_x + s * L
                inside = np.all((p >= ext_lo) & (p < ext_hi), axis=1)
                if sx == 0 and sy == 0 and sz == 0:
                    inside &= ~local_mask
                k = np.flatnonzero(inside)
                if len(k):
                    px.append(p[k])
                    pk.append(k)
                    ps.append(np.repeat(s[None, :], len(k), axis=0))
    if not px:
        return np.zeros((0, 3)), np.zeros(0, dtype=np.int64), np.zeros((0, 3), dtype=np.int64)
    return np.concatenate(px), np.concatenate(pk), np.concatenate(ps)


class SlabDecomposition:
    """One rank's part of a periodic orthogonal cell split into slabs along x.

    set_atoms(x, types, v, ids) hands every rank the whole system (setup);
    each keeps its slab's atoms.  compute() evaluates forces, energy and
    virial of the distributed system; nve_run(nsteps, dt, masses) runs
    velocity Verlet (fix nve) with re-decomposition as atoms move.  gather()
    returns the whole system's state on every rank (ordered by global id)."""

    def __init__(self, box, cut, skin, backend, rank=0, world=1, group=None,
                 rebuild_every=20, device=None):
        import torch
        self.torch = torch
        self.box = np.asarray(box, dtype=np.float64).copy()
        if np.any(self.box[6:9] != 0.0):
            raise ValueError("slab decomposition needs an orthogonal box")
        self.L = self.box[3:6].copy()
        self.cut = float(cut)
        self.skin = float(skin)
        self.backend = backend
        self.rank, self.world, self.group = rank, world, group
        self.rebuild_every = int(rebuild_every)
        self.device = device if device is not None else torch.device("cpu")
        w = self.L[0] / world
        if w < self.cut:
            raise ValueError(f"slabs of {w:.3f} A are narrower than the ghost cutoff {self.cut}")
        self.lo = self.box[0] + rank * w
        self.hi = self.box[0] + (rank + 1) * w if rank < world - 1 else self.box[0] + self.L[0]
        self.bounds = [self.box[0] + r * w for r in range(world)] + [self.box[0] + self.L[0]]

    # ---- collectives (no-ops on one rank) ----
    def _all_reduce(self, a):
        if self.world == 1:
            return a
        t = self.torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(self.device)
        self.torch.distributed.all_reduce(t, group=self.group)
        return t.cpu().numpy()

    def _all_gather_rows(self, a, width):
        """Concatenate every rank's rows (float64[n_r, width]) in rank order."""
        if self.world == 1:
            return a.copy(), np.array([len(a)])
        dist = self.torch.distributed
        n = self.torch.tensor([len(a)], dtype=self.torch.int64, device=self.device)
        ns = [self.torch.zeros_like(n) for _ in range(self.world)]
        dist.all_gather(ns, n, group=self.group)
        ns = np.array([int(v.item()) for v in ns])
        m = max(int(ns.max()), 1)
        buf = np.zeros((m, width))
        buf[:len(a)] = a
        t = self.torch.from_numpy(buf).to(self.device)
        out = [self.torch.zeros_like(t) for _ in range(self.world)]
        dist.all_gather(out, t, group=self.group)
        rows = np.concatenate([o.cpu().numpy()[:k] for o, k in zip(out, ns)])
        return rows, ns

    # ---- ownership and ghost lists ----
    def _wrap(self, x):
        b0 = self.box[:3]
        return b0 + np.mod(x - b0, self.L)

    def set_atoms(self, x, types, v=None, ids=None):
        x = self._wrap(np.asarray(x, dtype=np.float64))
        n = len(x)
        ids = np.arange(n) if ids is None else np.asarray(ids)
        v = np.zeros_like(x) if v is None else np.asarray(v, dtype=np.float64)
        mine = (x[:, 0] >= self.lo) & (x[:, 0] < self.hi)
        self.natoms = n
        self.x, self.v = x[mine].copy(), v[mine].copy()
        self.types = np.asarray(types, dtype=np.int32)[mine].copy()
        self.ids = ids[mine].copy()
        self.f = np.zeros_like(self.x)
        self._decompose()

    def _decompose(self):
        """New ghost lists from the current local atoms of every rank."""
        nloc = len(self.x)
        self.x = self._wrap(self.x)
        # boundary atoms: within cut of this slab's x faces (other ranks' ghosts)
        bnd = np.flatnonzero((self.x[:, 0] < self.lo + self.cut) |
                             (self.x[:, 0] >= self.hi - self.cut))
        rows = np.concatenate([self.x[bnd], self.types[bnd, None].astype(np.float64),
                               np.full((len(bnd), 1), float(self.rank)),
                               bnd[:, None].astype(np.float64)], axis=1)
        allb, counts = self._all_gather_rows(rows, 6)
        self.bnd = bnd
        self.bnd_counts = counts
        self.bnd_off = np.concatenate([[0], np.cumsum(counts)])
        others = allb[:, 4] != self.rank
        # candidates: own atoms (ghost images through the periodic faces) and
        # the other ranks' boundary atoms
        cand_x = np.concatenate([self.x, allb[others, :3]])
        cand_t = np.concatenate([self.types, allb[others, 3].astype(np.int32)])
        # reference of each candidate: own local index, or gathered row index
        cand_src = np.concatenate([np.arange(nloc), np.flatnonzero(others)])
        cand_own = np.concatenate([np.ones(nloc, dtype=bool), np.zeros(others.sum(), dtype=bool)])
        gx, gk, gs = slab_ghosts(cand_x, cand_own, cand_own, self.box, self.lo, self.hi, self.cut)
        self.g_own = cand_own[gk]         # ghost is an image of an own atom
        self.g_src = cand_src[gk]         # local index, or gathered row
        self.g_shift = gs
        self.g_types = cand_t[gk]
        self.nghost = len(gx)
        xall = np.concatenate([self.x, gx])
        tall = np.concatenate([self.types, self.g_types])
        self.backend.set_atoms_ghost(nloc, xall, tall)
        self.x_build = self.x.copy()
        self.steps_since = 0

    def _ghost_positions(self):
        """Positions of the current ghost set (forward communication)."""
        rows = np.concatenate([self.x[self.bnd], np.zeros((len(self.bnd), 3))], axis=1)
        allb, _ = self._all_gather_rows(rows, 6)
        src = np.where(self.g_own[:, None], self.x[np.where(self.g_own, self.g_src, 0)],
                       allb[np.where(self.g_own, 0, self.g_src), :3])
        return src + self.g_shift * self.L

    # ---- evaluation ----
    def compute(self, forward=True):
        """Forces on the local atoms (self.f), and the whole system's energy
        and virial (every rank gets them)."""
        if forward:
            xall = np.concatenate([self.x, self._ghost_positions()])
            self.backend.set_positions(xall)
        out = self.backend.compute(1, 1)
        nloc = len(self.x)
        fall = np.asarray(out["f"])
        f = fall[:nloc].copy()
        fg = fall[nloc:]
        # reverse communication: images of own atoms locally, other ranks'
        # boundary atoms through one all-reduce over the gathered rows
        own = self.g_own
        np.add.at(f, self.g_src[own], fg[own])
        buf = np.zeros((int(self.bnd_off[-1]), 3))
        np.add.at(buf, self.g_src[~own], fg[~own])
        red = self._all_reduce(np.concatenate([buf.ravel(), [out["energy"]],
                                               np.asarray(out["virial"])]))
        nb = buf.size
        mine = red[:nb].reshape(-1, 3)[self.bnd_off[self.rank]:self.bnd_off[self.rank + 1]]
        np.add.at(f, self.bnd, mine)
        self.f = f
        self.energy = float(red[nb])
        self.virial = red[nb + 1:nb + 7].copy()
        return self.f, self.energy, self.virial

    def _migrate(self):
        """Hand atoms that left the slab to their new owners (an all-gather of
        the leavers) and rebuild the ghost lists."""
        self.x = self._wrap(self.x)
        gone = (self.x[:, 0] < self.lo) | (self.x[:, 0] >= self.hi)
        rows = np.concatenate([self.x[gone], self.v[gone], self.f[gone],
                               self.types[gone, None].astype(np.float64),
                               self.ids[gone, None].astype(np.float64)], axis=1)
        allr, _ = self._all_gather_rows(rows, 11)
        keep = ~gone
        self.x, self.v, self.f = self.x[keep], self.v[keep], self.f[keep]
        self.types, self.ids = self.types[keep], self.ids[keep]
        take = (allr[:, 0] >= self.lo) & (allr[:, 0] < self.hi)
        if take.any():
            r = allr[take]
            self.x = np.concatenate([self.x, r[:, 0:3]])
            self.v = np.concatenate([self.v, r[:, 3:6]])
            self.f = np.concatenate([self.f, r[:, 6:9]])
            self.types = np.concatenate([self.types, r[:, 9].astype(np.int32)])
            self.ids = np.concatenate([self.ids, r[:, 10].astype(np.int64)])
        self._decompose()

    def nve_run(self, nsteps, dt, masses):
        """Velocity Verlet (fix_nve.cpp:64-141, metal units) of the
        distributed system; masses[type] per LAMMPS type (index 0 unused).
        Returns the potential energy after each step (every rank)."""
        m = np.asarray(masses, dtype=np.float64)[self.types][:, None]
        dtf = 0.5 * dt / MVV2E
        pe = []
        if not hasattr(self, "energy"):
            self.compute()
        for _ in range(nsteps):
            self.v += dtf / m * self.f
            self.x += dt * self.v
            self.steps_since += 1
            moved = np.max(np.sum((self.x - self.x_build) ** 2, axis=1), initial=0.0)
            need = self._all_reduce(np.array([float(moved > (0.5 * self.skin) ** 2)]))[0] > 0
            if need or self.steps_since >= self.rebuild_every:
                self._migrate()
                m = np.asarray(masses, dtype=np.float64)[self.types][:, None]
                self.compute(forward=False)
            else:
                self.compute()
            self.v += dtf / m * self.f
            pe.append(self.energy)
        return np.array(pe)

    def gather(self):
        """(x, v, f) of the whole system in global-id order, on every rank."""
        rows = np.concatenate([self.ids[:, None].astype(np.float64), self.x, self.v, self.f],
                              axis=1)
        allr, _ = self._all_gather_rows(rows, 10)
        order = np.argsort(allr[:, 0])
        allr = allr[order]
        return allr[:, 1:4], allr[:, 4:7], allr[:, 7:10]
