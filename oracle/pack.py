"""Python side of the FP64 oracle (TEST INFRASTRUCTURE ONLY).

Loads a tensormd ``.npz`` potential, builds the rational-interpolation table
the way the reference does at ``pair_coeff ... interp dx`` time, packs the
model into a flat (ints, doubles) blob and drives ``tmd_oracle.c`` through
ctypes.  Only tests, ``__graft_entry__.smoke()`` and the cpu_baseline leg of
``bench.py`` may import this module; the product never does.

Reference behaviour restated here (paths relative to the lammps-tensormd
tree):
  * npz keys and layer layout       src/ML-TENSORMD/nnp.cpp:110-145,
                                    fnn.cpp:32-55, descriptor.h:45-85
  * residual rule                   nnp.cpp:176-181
  * FNN forward on the grid         src/ML-TENSORMD/gpu/cuda/nnp.cu:59-116
                                    (bias + activation only for softplus and
                                    squareplus; output bias if requested)
  * grid, cutoff product            fnn.cpp:77-105, descriptor.cpp:143-171
  * table coefficients [y,s,c1,c2]  ration.hpp:166-225
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libtmd_oracle.so"

__all__ = ["Oracle", "load_npz", "build_table", "pack_model", "build_oracle"]


def build_oracle(force: bool = False) -> Path:
    """Compile tmd_oracle.c into oracle/libtmd_oracle.so (gcc, OpenMP)."""
    src = HERE / "tmd_oracle.c"
    if LIB_PATH.exists() and not force and LIB_PATH.stat().st_mtime >= src.stat().st_mtime:
        return LIB_PATH
    cmd = ["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared",
           str(src), "-o", str(LIB_PATH), "-lm"]
    subprocess.check_call(cmd)
    return LIB_PATH


def load_npz(path) -> dict:
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


def _scalar_dtype(pot: dict):
    if "precision" in pot and int(np.asarray(pot["precision"]).ravel()[0]) == 32:
        return np.float32
    return np.float64


def _softplus(z):
    thr = np.log(np.finfo(z.dtype).eps) + 2.0
    ex = np.exp(z)
    return np.where(z < -thr, np.log1p(ex), z)


def _squareplus(z):
    return 0.5 * (z + np.sqrt(z * z + 4.0))


def _cutoff(pot, r, dt):
    rc = dt(np.asarray(pot["rmax"]).ravel()[0])
    if int(np.asarray(pot["fctype"]).ravel()[0]) == 0:
        z = np.minimum(r / rc, dt(1.0)) * dt(np.pi)
        return dt(0.5) + dt(0.5) * np.cos(z)
    g = dt(5.0)
    z = np.minimum(r / rc, dt(np.pi))
    z5 = z ** 5
    return dt(1) + g * z5 * z - (g + dt(1)) * z5


def _fnn_grid(pot, x, dt):
    nl = int(pot["fnn::nlayers"])
    sizes = [1] + [int(s) for s in np.asarray(pot["fnn::layer_sizes"]).ravel()]
    act = int(pot["fnn::actfn"])
    outb = int(pot["fnn::apply_output_bias"])
    res_raw = int(pot["fnn::use_resnet_dt"])
    n_res = sum(1 for i in range(nl) if i > 0 and sizes[i] == sizes[i + 1])
    res = bool(res_raw and n_res > 0)
    h = x.reshape(-1, 1).astype(dt)
    for i in range(nl):
        W = np.asarray(pot[f"fnn::weights_0_{i}"], dtype=dt).reshape(sizes[i], sizes[i + 1])
        z = h @ W
        if i < nl - 1:
            if act in (1, 3):
                z = z + np.asarray(pot[f"fnn::biases_0_{i}"], dtype=dt).reshape(-1)
                z = _softplus(z) if act == 1 else _squareplus(z)
                if i > 0 and res and sizes[i] == sizes[i + 1]:
                    z = z + h
            h = z
        else:
            if outb:
                z = z + np.asarray(pot[f"fnn::biases_0_{i}"], dtype=dt).reshape(-1)
            h = z
    return h


def _analytic_grid(pot, r, dt):
    method = int(pot.get("descriptor::method", 0))
    rc = dt(np.asarray(pot["rmax"]).ravel()[0])
    r = r.reshape(-1, 1)
    if method == 0:
        rl = np.asarray(pot["descriptor::rl"], dtype=dt).ravel()
        pl = np.asarray(pot["descriptor::pl"], dtype=dt).ravel()
        f = np.exp(-((r / rl) ** pl))
    elif method == 1:
        D = np.asarray(pot["descriptor::D"], dtype=dt).ravel()
        g = np.asarray(pot["descriptor::gamma"], dtype=dt).ravel()
        r0 = np.asarray(pot["descriptor::r0"], dtype=dt).ravel()
        gdr = g * (r - r0)
        f = D * (np.exp(-2 * gdr) - 2 * np.exp(-gdr))
    elif method == 2:
        A = np.asarray(pot["descriptor::A"], dtype=dt).ravel()
        b = np.asarray(pot["descriptor::beta"], dtype=dt).ravel()
        re = np.asarray(pot["descriptor::re"], dtype=dt).ravel()
        f = A * np.exp(-b * ((r - re) / re))
    else:
        eta = np.asarray(pot["descriptor::eta"], dtype=dt).ravel()
        om = np.asarray(pot["descriptor::omega"], dtype=dt).ravel()
        f = np.exp(-eta * (r - om) ** 2 / (rc * rc))
    return f.astype(dt)


def build_table(pot: dict, delta: float):
    """Return (n, dx, params[n, 4, K]) for ``interp delta``."""
    dt = _scalar_dtype(pot)
    rmax = dt(np.asarray(pot["rmax"]).ravel()[0])
    delta = dt(delta)
    n = int(rmax / delta) + 1
    x = np.arange(n, dtype=dt) * delta
    use_fnn = int(pot["use_fnn"])
    y = _fnn_grid(pot, x, dt) if use_fnn else _analytic_grid(pot, x, dt)
    y = (y * _cutoff(pot, x, dt).reshape(-1, 1)).astype(dt)
    K = y.shape[1]
    xdx = dt(1.0) / delta
    prm = np.zeros((n, 4, K), dtype=dt)
    prm[:, 0, :] = y
    s = np.zeros((n, K), dtype=dt)
    s[: n - 1] = (y[1:] - y[:-1]) * xdx
    prm[:, 1, :] = s
    c1 = np.zeros((n, K), dtype=dt)
    c2 = np.zeros((n, K), dtype=dt)
    half = dt(2)
    for i in range(n - 1):
        si = s[i]
        if i == 0:
            sp = s[1]
            cond = si * (si - (sp - si) / half) <= 0
            c2[i] = np.where(cond, si * xdx, (sp - si) * xdx / half)
            c1[i] = 0
        elif i == n - 2:
            sm = s[i - 1]
            c1[i] = (si - sm) * xdx / half
            c2[i] = 0
        else:
            sm = s[i - 1]
            sp = s[i + 1]
            if i == 1:
                cond = sm * (sm - (si - sm) / half) <= 0
                c1[i] = np.where(cond, (si - half * sm) * xdx, (si - sm) * xdx / half)
            else:
                c1[i] = (si - sm) * xdx / half
            c2[i] = (sp - si) * xdx / half
    prm[:, 2, :] = c1
    prm[:, 3, :] = c2
    return n, float(delta), prm


def pack_model(pot: dict, interp: float | None = None):
    """Flatten a potential dict into the (ints, doubles) blob of tmd_oracle.c."""
    nelt = int(pot["nelt"])
    mm = int(pot["max_moment"])
    use_fnn = int(pot["use_fnn"])
    if use_fnn:
        K = int(pot["fnn::num_filters"])
    else:
        method = int(pot.get("descriptor::method", 0))
        key = {0: "descriptor::rl", 1: "descriptor::D", 2: "descriptor::A",
               3: "descriptor::eta"}[method]
        K = int(np.asarray(pot[key]).size)
    if use_fnn and not interp:
        raise ValueError("FNN radial basis requires interp dx")
    tdnp = "tdnp" in pot and int(np.asarray(pot["tdnp"]).ravel()[0]) == 1
    if tdnp:  # the TDNP nets replace the NNP (tensormd.cpp:129-132,471-484)
        nl, sizes = 0, []
        n_in = int(np.asarray(pot["H::weights_0_0"]).shape[0])
    else:
        nl = int(pot["nlayers"])
        sizes = [int(s) for s in np.asarray(pot["layer_sizes"]).ravel()]
        n_in = int(np.asarray(pot["weights_0_0"]).shape[0])
    ints = [1, nelt, mm, K, int(pot["fctype"]), 1 if interp else 0,
            int(pot.get("descriptor::method", 0)) if not use_fnn else 0,
            int(pot.get("is_T_symmetric", 0)), nl, 0 if tdnp else int(pot["actfn"]),
            0 if tdnp else int(pot["use_resnet_dt"]),
            0 if tdnp else int(pot["apply_output_bias"]), n_in, 0]
    ints += sizes
    dbl = [float(np.asarray(pot["rmax"]).ravel()[0]), 0.0]
    p = np.zeros((3, K))
    if not use_fnn:
        method = int(pot.get("descriptor::method", 0))
        names = {0: ("rl", "pl"), 1: ("D", "gamma", "r0"), 2: ("A", "beta", "re"),
                 3: ("eta", "omega")}[method]
        for a, nm in enumerate(names):
            p[a] = np.asarray(pot["descriptor::" + nm], dtype=np.float64).ravel()
    tab = np.zeros(0)
    if interp:
        n, dx, prm = build_table(pot, interp)
        ints[13] = n
        dbl[1] = dx
        tab = prm.astype(np.float64).ravel()
    parts = [np.asarray(dbl), p.ravel(), tab]
    full = [n_in] + sizes
    outb = 0 if tdnp else int(pot["apply_output_bias"])
    for e in range(nelt):
        for l in range(nl):
            parts.append(np.asarray(pot[f"weights_{e}_{l}"], dtype=np.float64).ravel())
            if parts[-1].size != full[l] * full[l + 1]:
                raise ValueError(f"weights_{e}_{l} has {parts[-1].size} values, "
                                 f"expected {full[l]}x{full[l + 1]}")
            if l < nl - 1 or outb:
                parts.append(np.asarray(pot[f"biases_{e}_{l}"], dtype=np.float64).ravel())
    return np.asarray(ints, dtype=np.int32), np.concatenate(parts).astype(np.float64)


def pack_tdnp(pot: dict):
    """The H, U, S nets of a tdnp = 1 potential (tdnp.cpp:46-139) as the blob
    of tmd_oracle.c tmdo_model_set_tdnp; H gets the zero weight column of the
    electron temperature (tdnp.cpp:80-97)."""
    nelt = int(pot["nelt"])
    som = int(np.asarray(pot.get("tdnp::Sommerfeld", 0)).ravel()[0])
    hs = [int(v) for v in np.asarray(pot["H::layer_sizes"]).ravel()]
    ydim = hs[-1] + 1
    ints = [som, ydim]
    parts = []
    for scope in ("H", "U", "S"):
        nl = int(pot[f"{scope}::nlayers"])
        ls = [int(v) for v in np.asarray(pot[f"{scope}::layer_sizes"]).ravel()]
        n_in = int(np.asarray(pot[f"{scope}::weights_0_0"]).shape[0])
        sizes = [n_in] + ls
        if scope == "H":
            sizes[-1] += 1
        outb = int(pot[f"{scope}::apply_output_bias"])
        ints += [nl, int(pot[f"{scope}::actfn"]), int(pot[f"{scope}::use_resnet_dt"]), outb]
        ints += sizes
        for e in range(nelt):
            for l in range(nl):
                w = np.asarray(pot[f"{scope}::weights_{e}_{l}"], dtype=np.float64)
                w = w.reshape(sizes[l], -1)
                if scope == "H" and l == nl - 1:
                    w = np.concatenate([w, np.zeros((sizes[l], 1))], axis=1)
                parts.append(w.ravel())
                if l < nl - 1 or outb:
                    b = np.asarray(pot[f"{scope}::biases_{e}_{l}"], dtype=np.float64).ravel()
                    if scope == "H" and l == nl - 1:
                        b = np.concatenate([b, [0.0]])
                    parts.append(b)
    return np.asarray(ints, dtype=np.int32), np.concatenate(parts).astype(np.float64)


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


class Oracle:
    """FP64 CPU oracle of the tensormd force path (checker, not product)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            build_oracle()
            L = ctypes.CDLL(str(LIB_PATH))
            L.tmdo_model_new.restype = ctypes.c_void_p
            L.tmdo_model_new.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_double), ctypes.c_int]
            L.tmdo_model_free.argtypes = [ctypes.c_void_p]
            L.tmdo_model_dims.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
            L.tmdo_neighbors.restype = ctypes.c_long
            L.tmdo_neighbors.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                         ctypes.POINTER(ctypes.c_double),
                                         ctypes.POINTER(ctypes.c_int), ctypes.c_double,
                                         ctypes.POINTER(ctypes.c_int),
                                         ctypes.POINTER(ctypes.c_int), ctypes.c_long]
            L.tmdo_compute.restype = ctypes.c_double
            L.tmdo_compute.argtypes = [ctypes.c_void_p, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_double),
                                       ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_double),
                                       ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_long),
                                       ctypes.POINTER(ctypes.c_int), ctypes.c_double,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
            L.tmdo_nve.restype = ctypes.c_int
            L.tmdo_nve.argtypes = [ctypes.c_void_p, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_int),
                                   ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_int), ctypes.c_double,
                                   ctypes.c_int, ctypes.c_double,
                                   ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
            L.tmdo_nvt.restype = ctypes.c_int
            L.tmdo_nvt.argtypes = [ctypes.c_void_p, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_int),
                                   ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_int), ctypes.c_double,
                                   ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_double,
                                   ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
            L.tmdo_model_set_tdnp.restype = ctypes.c_int
            L.tmdo_model_set_tdnp.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                              ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                              ctypes.c_int]
            L.tmdo_set_etemp.argtypes = [ctypes.c_void_p, ctypes.c_double]
            L.tmdo_tdnp_totals.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
            L.tmdo_fire.restype = ctypes.c_int
            L.tmdo_fire.argtypes = [ctypes.c_void_p, ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_double),
                                    ctypes.POINTER(ctypes.c_int),
                                    ctypes.POINTER(ctypes.c_double),
                                    ctypes.POINTER(ctypes.c_double),
                                    ctypes.POINTER(ctypes.c_int), ctypes.c_double,
                                    ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                    ctypes.POINTER(ctypes.c_double),
                                    ctypes.POINTER(ctypes.c_double)]
            cls._lib = L
        return cls._lib

    def __init__(self, pot, interp: float | None = None, etemp: float = 0.0):
        """etemp: electron temperature in K (pair_coeff keyword etemp, used by
        tdnp = 1 potentials; converted to eV as pair_tensormd.cpp:33,246)."""
        if not isinstance(pot, dict):
            pot = load_npz(pot)
        self.pot = pot
        ints, dbl = pack_model(pot, interp)
        self._ints, self._dbl = ints, dbl
        L = self.lib()
        self.h = L.tmdo_model_new(_p(ints, ctypes.c_int), ints.size,
                                  _p(dbl, ctypes.c_double), dbl.size)
        if not self.h:
            raise ValueError("oracle rejected the model")
        self.tdnp = "tdnp" in pot and int(np.asarray(pot["tdnp"]).ravel()[0]) == 1
        if self.tdnp:
            ti, td = pack_tdnp(pot)
            self._tints, self._tdbl = ti, td
            if L.tmdo_model_set_tdnp(self.h, _p(ti, ctypes.c_int), ti.size,
                                     _p(td, ctypes.c_double), td.size) != 0:
                raise ValueError("oracle rejected the TDNP nets")
        self.set_etemp(etemp)
        dims = np.zeros(6, dtype=np.int32)
        L.tmdo_model_dims(self.h, _p(dims, ctypes.c_int))
        self.K, self.D, self.M, self.nelt, self.n_in, self.resnet = (int(v) for v in dims)
        self.rmax = float(np.asarray(pot["rmax"]).ravel()[0])
        self.masses = np.asarray(pot["masses"], dtype=np.float64).ravel()

    def set_etemp(self, kelvin: float):
        """Electron temperature (K) of a TDNP potential (fix tensormd/etemp)."""
        self.lib().tmdo_set_etemp(self.h, float(kelvin) / 11604.522060401008)

    def tdnp_totals(self):
        """(entropy, free energy) of the last compute of a TDNP potential."""
        out = np.zeros(2)
        self.lib().tmdo_tdnp_totals(self.h, _p(out, ctypes.c_double))
        return float(out[0]), float(out[1])

    def __del__(self):
        try:
            if getattr(self, "h", None):
                self.lib().tmdo_model_free(self.h)
                self.h = None
        except Exception:
            pass

    @staticmethod
    def neighbors(x, box, pbc, cut):
        """Full list (LAMMPS npair_full_bin semantics) with image shifts.

        Returns (off[n+1] int64, ent[npair,4] int32 = (j, sx, sy, sz))."""
        L = Oracle.lib()
        x = np.ascontiguousarray(x, dtype=np.float64)
        n = x.shape[0]
        bx = np.ascontiguousarray(box, dtype=np.float64)
        pb = np.ascontiguousarray(pbc, dtype=np.int32)
        cnt = np.zeros(max(n, 1), dtype=np.int32)
        tot = L.tmdo_neighbors(n, _p(x, ctypes.c_double), _p(bx, ctypes.c_double),
                               _p(pb, ctypes.c_int), cut, _p(cnt, ctypes.c_int), None, 0)
        ent = np.zeros((max(tot, 1), 4), dtype=np.int32)
        tot2 = L.tmdo_neighbors(n, _p(x, ctypes.c_double), _p(bx, ctypes.c_double),
                                _p(pb, ctypes.c_int), cut, _p(cnt, ctypes.c_int),
                                _p(ent, ctypes.c_int), tot)
        assert tot2 == tot
        off = np.zeros(n + 1, dtype=np.int64)
        off[1:] = np.cumsum(cnt[:n])
        return off, ent[:tot]

    def compute(self, x, elem, box, pbc, nlist=None, skin=0.0, scale=1.0,
                want_G=False, want_dEdG=False, nlocal=None):
        """Return dict(energy, eatom, f, virial, vatom[, G, dEdG]).

        nlocal (ghost-aware evaluation, as a LAMMPS rank): only atoms
        0..nlocal-1 are evaluated (their rows, energies); the others are
        partners only and receive forces and per-atom virial halves."""
        L = self.lib()
        x = np.ascontiguousarray(x, dtype=np.float64)
        n = x.shape[0]
        el = np.ascontiguousarray(elem, dtype=np.int32)
        bx = np.ascontiguousarray(box, dtype=np.float64)
        pb = np.ascontiguousarray(pbc, dtype=np.int32)
        if nlist is None:
            nlist = self.neighbors(x, bx, pb, self.rmax + skin)
        off, ent = nlist
        off = np.ascontiguousarray(off, dtype=np.int64)
        ent = np.ascontiguousarray(ent, dtype=np.int32)
        if nlocal is not None and nlocal < n:
            # ghosts keep no rows: the local rows are the first off[nlocal] entries
            ent = np.ascontiguousarray(ent[:off[nlocal]])
            off = np.concatenate([off[:nlocal + 1], np.full(n - nlocal, off[nlocal])])
        if ent.size == 0:
            ent = np.zeros((1, 4), dtype=np.int32)
        eatom = np.zeros(n)
        f = np.zeros((n, 3))
        vir = np.zeros(6)
        vatom = np.zeros((n, 6))
        G = np.zeros((n, self.n_in)) if want_G else None
        dG = np.zeros((n, self.n_in)) if want_dEdG else None
        e = L.tmdo_compute(self.h, n, _p(x, ctypes.c_double), _p(el, ctypes.c_int),
                           _p(bx, ctypes.c_double), _p(pb, ctypes.c_int),
                           _p(off, ctypes.c_long), _p(ent, ctypes.c_int), scale,
                           eatom.ctypes.data, f.ctypes.data, vir.ctypes.data,
                           vatom.ctypes.data, G.ctypes.data if G is not None else None,
                           dG.ctypes.data if dG is not None else None)
        if nlocal is not None and nlocal < n:
            # an atom without a row still has the energy of an isolated atom
            e -= float(eatom[nlocal:].sum())
            eatom[nlocal:] = 0.0
            if G is not None:
                G = G[:nlocal]
            if dG is not None:
                dG = dG[:nlocal]
        out = dict(energy=e, eatom=eatom, f=f, virial=vir, vatom=vatom)
        if G is not None:
            out["G"] = G
        if dG is not None:
            out["dEdG"] = dG
        return out

    def nve(self, x, v, elem, box, pbc, dt, nsteps, skin=1.0):
        """Velocity Verlet in metal units; returns (x, v, f, thermo[n+1, 2])."""
        L = self.lib()
        x = np.array(x, dtype=np.float64, order="C")
        v = np.array(v, dtype=np.float64, order="C")
        n = x.shape[0]
        el = np.ascontiguousarray(elem, dtype=np.int32)
        bx = np.ascontiguousarray(box, dtype=np.float64)
        pb = np.ascontiguousarray(pbc, dtype=np.int32)
        ms = np.ascontiguousarray(self.masses, dtype=np.float64)
        f = np.zeros((n, 3))
        th = np.zeros((nsteps + 1, 2))
        rc = L.tmdo_nve(self.h, n, _p(x, ctypes.c_double), _p(v, ctypes.c_double),
                        _p(el, ctypes.c_int), _p(ms, ctypes.c_double),
                        _p(bx, ctypes.c_double), _p(pb, ctypes.c_int), dt, nsteps, skin,
                        _p(f, ctypes.c_double), th.ctypes.data)
        if rc != 0:
            raise RuntimeError("oracle nve failed")
        return x, v, f, th

    def nvt(self, x, v, elem, box, pbc, dt, nsteps, t_start, t_stop, t_damp, skin=1.0):
        """fix nvt (Nose-Hoover chain of 3, fresh thermostat); returns
        (x, v, f, thermo[n+1, 3] = pe, ke, chain energy)."""
        L = self.lib()
        x = np.array(x, dtype=np.float64, order="C")
        v = np.array(v, dtype=np.float64, order="C")
        n = x.shape[0]
        el = np.ascontiguousarray(elem, dtype=np.int32)
        bx = np.ascontiguousarray(box, dtype=np.float64)
        pb = np.ascontiguousarray(pbc, dtype=np.int32)
        ms = np.ascontiguousarray(self.masses, dtype=np.float64)
        f = np.zeros((n, 3))
        th = np.zeros((nsteps + 1, 3))
        rc = L.tmdo_nvt(self.h, n, _p(x, ctypes.c_double), _p(v, ctypes.c_double),
                        _p(el, ctypes.c_int), _p(ms, ctypes.c_double),
                        _p(bx, ctypes.c_double), _p(pb, ctypes.c_int), dt, nsteps, skin,
                        t_start, t_stop, t_damp, _p(f, ctypes.c_double), th.ctypes.data)
        if rc != 0:
            raise RuntimeError("oracle nvt failed")
        return x, v, f, th

    def fire(self, x, elem, box, pbc, dt, ftol, maxiter, skin=1.0):
        """min_style fire at LAMMPS's defaults (eulerimplicit, halfstepback),
        stopped when max_i |F_i| < ftol or after maxiter iterations; returns
        (x, f, energy, iterations)."""
        L = self.lib()
        x = np.array(x, dtype=np.float64, order="C")
        n = x.shape[0]
        el = np.ascontiguousarray(elem, dtype=np.int32)
        bx = np.ascontiguousarray(box, dtype=np.float64)
        pb = np.ascontiguousarray(pbc, dtype=np.int32)
        ms = np.ascontiguousarray(self.masses, dtype=np.float64)
        f = np.zeros((n, 3))
        pe = np.zeros(1)
        it = L.tmdo_fire(self.h, n, _p(x, ctypes.c_double), _p(el, ctypes.c_int),
                         _p(ms, ctypes.c_double), _p(bx, ctypes.c_double),
                         _p(pb, ctypes.c_int), dt, ftol, int(maxiter), skin,
                         _p(f, ctypes.c_double), _p(pe, ctypes.c_double))
        return x, f, float(pe[0]), int(it)


if __name__ == "__main__":  # pragma: no cover
    build_oracle(force=True)
    print(LIB_PATH)
