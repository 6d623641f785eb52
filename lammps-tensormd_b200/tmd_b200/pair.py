"""PairTensorMD-shaped host interface over libtmd_b200.so.

Mirrors the LAMMPS pair style of src/ML-TENSORMD/pair_tensormd.cpp:
  settings()            no arguments allowed            (pair_tensormd.cpp:205-208)
  coeff("* * f.npz El1 El2 [interp dx] [cmax ...]")      (:214-317)
  init_one(i, j)        returns the cutoff rmax           (:336-341)
  compute(eflag, vflag) energy -> eng_vdwl, forces -> f, virial via the
                        fdotr convention, eatom / vatom   (:141-184)
  extract("scale")      the fix-adapt scale factor        (:415-425)
Atoms are handed over as LAMMPS would hold them for one rank with periodic
images handled on the device: local positions x[n][3], 1-based types, box.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .lib import check, load_library

_pd = ctypes.POINTER(ctypes.c_double)
_pi = ctypes.POINTER(ctypes.c_int)


def _dp(a):
    return None if a is None else a.ctypes.data_as(_pd)


def _ip(a):
    return None if a is None else a.ctypes.data_as(_pi)


class TensorMDModel:
    """A loaded potential (pair_coeff) on one CUDA device."""

    def __init__(self, coeff_args: str, device: int = 0):
        self.lib = load_library()
        h = ctypes.c_void_p()
        check(self.lib.tmd_model_load(coeff_args.encode(), device, ctypes.byref(h)))
        self.h = h
        cut = ctypes.c_double()
        nelt, ntypes, nd, k, m = (ctypes.c_int() for _ in range(5))
        check(self.lib.tmd_model_info(h, ctypes.byref(cut), ctypes.byref(nelt),
                                      ctypes.byref(ntypes), ctypes.byref(nd),
                                      ctypes.byref(k), ctypes.byref(m)))
        self.cutmax = cut.value
        self.nelt, self.ntypes, self.n_desc = nelt.value, ntypes.value, nd.value
        self.num_filters, self.mmax = k.value, m.value
        tmap = np.zeros(self.ntypes + 1, dtype=np.int32)
        tmass = np.zeros(self.ntypes + 1, dtype=np.float64)
        check(self.lib.tmd_model_type_map(h, _ip(tmap), _dp(tmass)))
        self.type_map, self.type_mass = tmap, tmass

    def close(self):
        if getattr(self, "h", None):
            self.lib.tmd_model_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class TensorMDSystem:
    """Device-resident periodic cell (atoms, velocities, neighbor list)."""

    def __init__(self, model: TensorMDModel, natoms_cap: int, skin: float = 1.0):
        self.model = model
        self.lib = model.lib
        h = ctypes.c_void_p()
        check(self.lib.tmd_system_create(model.h, int(natoms_cap), float(skin),
                                         ctypes.byref(h)))
        self.h = h
        self.n = 0

    def close(self):
        if getattr(self, "h", None) and getattr(self, "_owned", True):
            self.lib.tmd_system_free(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_box(self, box, pbc=(1, 1, 1)):
        b = np.ascontiguousarray(box, dtype=np.float64)
        p = np.ascontiguousarray(pbc, dtype=np.int32)
        check(self.lib.tmd_system_set_box(self.h, _dp(b), _ip(p)))

    def set_atoms(self, x, types, v=None):
        x = np.ascontiguousarray(x, dtype=np.float64)
        t = np.ascontiguousarray(types, dtype=np.int32)
        vv = None if v is None else np.ascontiguousarray(v, dtype=np.float64)
        self.n = x.shape[0]
        self.nlocal = self.n
        check(self.lib.tmd_system_set_atoms(self.h, self.n, _dp(x), _ip(t), _dp(vv)))

    def set_positions(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        check(self.lib.tmd_system_set_positions(self.h, _dp(x)))

    def set_atoms_ghost(self, nlocal, x, types):
        """Ghost-aware mode (multi-rank LAMMPS): x[nall, 3] and types[nall]
        hold the rank's local atoms first, then its ghosts; compute() then
        returns forces for all nall atoms and the energy of the local ones."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        t = np.ascontiguousarray(types, dtype=np.int32)
        self.n = x.shape[0]
        self.nlocal = int(nlocal)
        check(self.lib.tmd_system_set_atoms_ghost(self.h, int(nlocal), self.n - int(nlocal),
                                                  _dp(x), _ip(t)))

    def get(self):
        n = self.n
        x, v, f = (np.zeros((n, 3)) for _ in range(3))
        img = np.zeros((n, 3), dtype=np.int32)
        check(self.lib.tmd_system_get(self.h, _dp(x), _dp(v), _dp(f), _ip(img)))
        return x, v, f, img

    def compute(self, eflag=1, vflag=1, scale=1.0, peratom=False, forces=True):
        n = self.n
        e = np.zeros(1)
        vir = np.zeros(6)
        f = np.zeros((n, 3)) if forces else None
        ea = np.zeros(n) if peratom else None
        va = np.zeros((n, 6)) if peratom else None
        check(self.lib.tmd_compute(self.h, int(eflag), int(vflag), float(scale), _dp(e),
                                   _dp(vir), _dp(f), _dp(ea), _dp(va)))
        out = dict(energy=float(e[0]), virial=vir, f=f)
        if peratom:
            out["eatom"], out["vatom"] = ea, va
        return out

    def nve_run(self, nsteps, dt, thermo_every=0):
        rows = 0
        th = None
        if thermo_every:
            rows = 1 + nsteps // thermo_every + (1 if nsteps % thermo_every else 0)
            th = np.zeros((rows, 2))
        check(self.lib.tmd_nve_run(self.h, int(nsteps), float(dt), int(thermo_every), _dp(th)))
        return th

    def nvt_run(self, nsteps, dt, t_start, t_stop, t_damp, thermo_every=0):
        """fix nvt temp t_start t_stop t_damp for nsteps (Nose-Hoover chain)."""
        th = None
        if thermo_every:
            rows = 1 + nsteps // thermo_every + (1 if nsteps % thermo_every else 0)
            th = np.zeros((rows, 2))
        check(self.lib.tmd_nvt_run(self.h, int(nsteps), float(dt), float(t_start), float(t_stop),
                                   float(t_damp), int(thermo_every), _dp(th)))
        return th

    def nvt_energy(self, ngroups=1):
        """Thermostat chain energy per group after the last nvt run."""
        e = np.zeros(ngroups)
        check(self.lib.tmd_nvt_energy(self.h, _dp(e)))
        return e

    def neighbor_list(self, cut):
        n = self.n
        counts = np.zeros(max(n, 1), dtype=np.int32)
        tot = ctypes.c_long()
        check(self.lib.tmd_neighbor_list(self.h, float(cut), _ip(counts), None, 0,
                                         ctypes.byref(tot)))
        ent = np.zeros((max(tot.value, 1), 4), dtype=np.int32)
        check(self.lib.tmd_neighbor_list(self.h, float(cut), _ip(counts), _ip(ent),
                                         tot.value, ctypes.byref(tot)))
        off = np.zeros(n + 1, dtype=np.int64)
        off[1:] = np.cumsum(counts[:n])
        return off, ent[: tot.value]

    def descriptors(self):
        G = np.zeros((getattr(self, "nlocal", self.n), self.model.n_desc))
        check(self.lib.tmd_get_descriptors(self.h, _dp(G)))
        return G

    # kernel forms of the force loop (tmd_system_set_variant, family 0)
    FORCE_VARIANTS = ("filter_lane", "pair_lane8", "pair_lane16", "pair_lane32")

    def set_force_variant(self, variant):
        v = self.FORCE_VARIANTS.index(variant) if isinstance(variant, str) else int(variant)
        check(self.lib.tmd_system_set_variant(self.h, 0, v))

    def force_variant(self) -> str:
        v = ctypes.c_int()
        check(self.lib.tmd_system_get_variant(self.h, 0, ctypes.byref(v)))
        return self.FORCE_VARIANTS[v.value]

    # kernel forms of the descriptor (family 1)
    DESC_VARIANTS = ("filter4", "wide", "wide2", "split")

    def set_descriptor_variant(self, variant):
        v = self.DESC_VARIANTS.index(variant) if isinstance(variant, str) else int(variant)
        check(self.lib.tmd_system_set_variant(self.h, 1, v))

    def descriptor_variant(self) -> str:
        v = ctypes.c_int()
        check(self.lib.tmd_system_get_variant(self.h, 1, ctypes.byref(v)))
        return self.DESC_VARIANTS[v.value]

    def autotune(self, reps: int = 5, family: str = "force"):
        """Time every form of a kernel family ("force" or "descriptor") on the
        current atoms, keep the fastest; returns {form: ms per launch}."""
        names = self.FORCE_VARIANTS if family == "force" else self.DESC_VARIANTS
        ms = np.zeros(4)
        check(self.lib.tmd_system_autotune(self.h, 0 if family == "force" else 1, int(reps),
                                           _dp(ms)))
        return dict(zip(names, ms[:len(names)].tolist()))

    def stream(self) -> int:
        p = ctypes.c_void_p()
        check(self.lib.tmd_system_stream(self.h, ctypes.byref(p)))
        return p.value or 0

    def launches(self) -> int:
        return int(self.lib.tmd_system_launches(self.h))

    def set_etemp(self, kelvin):
        """Electron temperature of a tdnp = 1 potential, in K (fix tensormd/etemp)."""
        check(self.lib.tmd_system_set_etemp(self.h, float(kelvin) / 11604.522060401008))

    def tdnp_energies(self):
        """(entropy, free energy) of the last compute of a tdnp = 1 potential."""
        s_, a_ = ctypes.c_double(), ctypes.c_double()
        check(self.lib.tmd_system_tdnp_energies(self.h, ctypes.byref(s_), ctypes.byref(a_)))
        return s_.value, a_.value

    def rebuilds(self) -> int:
        """Neighbor-list rebuilds run since the system was created."""
        c = ctypes.c_long()
        check(self.lib.tmd_system_rebuilds(self.h, ctypes.byref(c)))
        return int(c.value)

    PROFILE_FAMILIES = ("neighbor", "descriptor", "mlp", "force", "gather", "nve", "reduce",
                        "dedp")

    def profile(self, enable: bool):
        check(self.lib.tmd_profile_enable(self.h, int(bool(enable))))

    def profile_read(self, reset=True):
        """{family: (launch-group count, summed device ms)} since the last reset."""
        n = np.zeros(len(self.PROFILE_FAMILIES), dtype=np.int64)
        ms = np.zeros(len(self.PROFILE_FAMILIES))
        check(self.lib.tmd_profile_read(self.h, n.ctypes.data_as(ctypes.POINTER(ctypes.c_long)),
                                        _dp(ms), int(bool(reset))))
        return {f: (int(c), float(t)) for f, c, t in zip(self.PROFILE_FAMILIES, n, ms)}


class TensorMDBatch:
    """Many small periodic cells evaluated together (tmd_batch_*).

    natoms[c] atoms per cell; atom arrays are concatenated cell by cell."""

    def __init__(self, model: TensorMDModel, natoms, skin: float = 1.0):
        self.model = model
        self.lib = model.lib
        na = np.ascontiguousarray(natoms, dtype=np.int32)
        self.natoms = na
        self.ncells = len(na)
        self.n = int(na.sum())
        self.offsets = np.concatenate([[0], np.cumsum(na)]).astype(np.int64)
        h = ctypes.c_void_p()
        check(self.lib.tmd_batch_create(model.h, self.ncells, _ip(na), float(skin),
                                        ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.tmd_batch_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_cells(self, boxes, pbc=None):
        b = np.ascontiguousarray(boxes, dtype=np.float64).reshape(self.ncells, 9)
        p = (np.ones((self.ncells, 3), dtype=np.int32) if pbc is None
             else np.ascontiguousarray(pbc, dtype=np.int32).reshape(self.ncells, 3))
        check(self.lib.tmd_batch_set_cells(self.h, _dp(b), _ip(p)))

    def set_atoms(self, x, types, v=None):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(self.n, 3)
        t = np.ascontiguousarray(types, dtype=np.int32)
        vv = None if v is None else np.ascontiguousarray(v, dtype=np.float64)
        check(self.lib.tmd_batch_set_atoms(self.h, _dp(x), _ip(t), _dp(vv)))

    def get(self):
        x, v, f = (np.zeros((self.n, 3)) for _ in range(3))
        img = np.zeros((self.n, 3), dtype=np.int32)
        check(self.lib.tmd_batch_get(self.h, _dp(x), _dp(v), _dp(f), _ip(img)))
        return x, v, f, img

    def compute(self, forces=True):
        e = np.zeros(self.ncells)
        vir = np.zeros((self.ncells, 6))
        f = np.zeros((self.n, 3)) if forces else None
        check(self.lib.tmd_batch_compute(self.h, _dp(e), _dp(vir), _dp(f)))
        return dict(energy=e, virial=vir, f=f)

    def nve_run(self, nsteps, dt, thermo_every=0):
        th = None
        if thermo_every:
            rows = 1 + nsteps // thermo_every + (1 if nsteps % thermo_every else 0)
            th = np.zeros((rows, self.ncells, 2))
        check(self.lib.tmd_batch_nve_run(self.h, int(nsteps), float(dt), int(thermo_every),
                                         _dp(th)))
        return th

    def nvt_run(self, nsteps, dt, t_start, t_stop, t_damp, thermo_every=0):
        """fix nvt per cell: t_start / t_stop scalars or one value per cell."""
        ts = np.ascontiguousarray(np.broadcast_to(np.asarray(t_start, dtype=np.float64),
                                                  (self.ncells,)))
        te = np.ascontiguousarray(np.broadcast_to(np.asarray(t_stop, dtype=np.float64),
                                                  (self.ncells,)))
        th = None
        if thermo_every:
            rows = 1 + nsteps // thermo_every + (1 if nsteps % thermo_every else 0)
            th = np.zeros((rows, self.ncells, 2))
        check(self.lib.tmd_batch_nvt_run(self.h, int(nsteps), float(dt), _dp(ts), _dp(te),
                                         float(t_damp), int(thermo_every), _dp(th)))
        return th

    def system(self) -> "TensorMDSystem":
        """The underlying system handle (stream, launches, profile, lists)."""
        h = ctypes.c_void_p()
        check(self.lib.tmd_batch_system(self.h, ctypes.byref(h)))
        s = TensorMDSystem.__new__(TensorMDSystem)
        s.model, s.lib, s.h, s.n = self.model, self.lib, h, self.n
        s._owned = False  # the batch frees it
        s._batch = self
        return s


class TensorMDServer:
    """Job server (tmd_server_*): continuous batching of small systems.

    submit() may be called from any thread; wait() returns the job's results."""

    ENERGY, NVE, FIRE = 0, 1, 2

    def __init__(self, model: TensorMDModel, max_atoms: int = 0, max_cells: int = 8192,
                 skin: float = 1.0, steps_per_tick: int = 8, hbm_bytes: int = 0,
                 max_density: float = 0.0):
        """Capacity either as max_atoms, or as an HBM budget (hbm_bytes) for
        jobs up to max_density atoms per A^3 (tmd_server_create_bytes)."""
        self.model = model
        self.lib = model.lib
        h = ctypes.c_void_p()
        if hbm_bytes:
            check(self.lib.tmd_server_create_bytes(model.h, int(hbm_bytes), float(max_density),
                                                   int(max_cells), float(skin),
                                                   int(steps_per_tick), ctypes.byref(h)))
        else:
            check(self.lib.tmd_server_create(model.h, int(max_atoms), int(max_cells),
                                             float(skin), int(steps_per_tick), ctypes.byref(h)))
        self.h = h
        self._n = {}

    def footprint(self):
        """dict(device_bytes, max_atoms, row_length) (tmd_server_footprint)."""
        b = ctypes.c_size_t()
        na, cap = ctypes.c_int(), ctypes.c_int()
        check(self.lib.tmd_server_footprint(self.h, ctypes.byref(b), ctypes.byref(na),
                                            ctypes.byref(cap)))
        return dict(device_bytes=b.value, max_atoms=na.value, row_length=cap.value)

    def close(self):
        if getattr(self, "h", None):
            self.lib.tmd_server_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, kind, x, types, box, pbc=(1, 1, 1), v=None, nsteps=0, dt=0.001,
               fmax=0.01) -> int:
        x = np.ascontiguousarray(x, dtype=np.float64)
        t = np.ascontiguousarray(types, dtype=np.int32)
        vv = None if v is None else np.ascontiguousarray(v, dtype=np.float64)
        b = np.ascontiguousarray(box, dtype=np.float64)
        p = np.ascontiguousarray(pbc, dtype=np.int32)
        tk = ctypes.c_long()
        check(self.lib.tmd_server_submit(self.h, int(kind), len(x), _dp(x), _ip(t), _dp(vv),
                                         _dp(b), _ip(p), int(nsteps), float(dt), float(fmax),
                                         ctypes.byref(tk)))
        self._n[tk.value] = len(x)
        return tk.value

    def wait(self, ticket: int, timeout: float = -1.0):
        """dict(energy, virial, x, v, f, steps, latency); raises TmdError (code -8
        when the job is not done within timeout seconds)."""
        n = self._n[ticket]
        e = np.zeros(1)
        vir = np.zeros(6)
        x, v, f = (np.zeros((n, 3)) for _ in range(3))
        steps = ctypes.c_int()
        lat = np.zeros(1)
        check(self.lib.tmd_server_wait(self.h, int(ticket), float(timeout), _dp(e), _dp(vir),
                                       _dp(x), _dp(v), _dp(f), ctypes.byref(steps), _dp(lat)))
        del self._n[ticket]
        return dict(energy=float(e[0]), virial=vir, x=x, v=v, f=f, steps=steps.value,
                    latency=float(lat[0]))

    def stats(self):
        sub, comp, act = ctypes.c_long(), ctypes.c_long(), ctypes.c_long()
        ast, busy = np.zeros(1), np.zeros(1)
        check(self.lib.tmd_server_stats(self.h, ctypes.byref(sub), ctypes.byref(comp),
                                        ctypes.byref(act), _dp(ast), _dp(busy)))
        return dict(submitted=sub.value, completed=comp.value, active_atoms=act.value,
                    atom_steps=float(ast[0]), busy_s=float(busy[0]))

    def timing(self):
        """Worker seconds by phase: relayout, admission evaluation, steps, results."""
        t = np.zeros(4)
        check(self.lib.tmd_server_timing(self.h, _dp(t)))
        return dict(zip(("relayout", "admission_eval", "steps", "results"), t.tolist()))


class PairTensorMD:
    """The pair_style tensormd call surface, single rank, periodic on device."""

    def __init__(self, device: int = 0, skin: float = 1.0):
        self.device = device
        self.skin = skin
        self.model = None
        self.system = None
        self.scale = 1.0
        self.eng_vdwl = 0.0
        self.virial = np.zeros(6)
        self.eatom = None
        self.vatom = None

    def settings(self, *args):
        if args:
            raise ValueError("Illegal pair_style command")

    def coeff(self, args: str):
        tok = args.split()
        if len(tok) < 4 or tok[0] != "*" or tok[1] != "*":
            raise ValueError("Incorrect args for pair coefficients")
        self.model = TensorMDModel(" ".join(tok[2:]), self.device)
        self.system = None

    def init_one(self, i: int, j: int) -> float:
        return self.model.cutmax

    def extract(self, name: str):
        if name == "scale":
            return self.scale
        return None

    def compute(self, x, types, box, pbc=(1, 1, 1), eflag=1, vflag=1, eflag_atom=0,
                vflag_atom=0):
        """Forces f[n][3] for local atoms; sets eng_vdwl, virial, eatom, vatom."""
        x = np.asarray(x, dtype=np.float64)
        n = x.shape[0]
        if self.system is None or n > self._cap:
            self._cap = max(n, 1)
            self.system = TensorMDSystem(self.model, self._cap, self.skin)
            self._box = None
        bx = tuple(np.asarray(box, dtype=np.float64).tolist()) + tuple(int(p) for p in pbc)
        if self._box != bx:
            self.system.set_box(box, pbc)
            self._box = bx
            self.system.set_atoms(x, types)
        else:
            self.system.set_atoms(x, types)
        out = self.system.compute(eflag, vflag, self.scale, peratom=bool(eflag_atom or vflag_atom))
        self.eng_vdwl = out["energy"] if eflag else 0.0
        self.virial = out["virial"]
        self.eatom = out.get("eatom")
        self.vatom = out.get("vatom")
        return out["f"]
