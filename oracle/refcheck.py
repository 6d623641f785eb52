"""Second checker: the reference's own CPU contraction kernels
(src/ML-TENSORMD/tensor_ops.cpp via oracle/_ref/libtmdref.so, built by
oracle/build_ref.py) fed with per-pair inputs built here in FP64.  Test
infrastructure only.

The per-pair inputs follow the reference's setup_tensors_device
(kernel.cu:721-817): u = (x_j - x_i) / r, R = r, mask = 1 inside the cutoff,
neighbors grouped by element block (eltij_pos, tensormd.cpp:165-176) into
padded slots c; M the monomials of u in the order of kernel.cu:1197-1232; H
and dH/dr the Gaussian SF basis times the cosine cutoff (descriptor.cpp:119-138,
cutoff.cpp:20-37).  T is the multiplicity tensor of tensormd.cpp:202-233.
"""
from __future__ import annotations

import ctypes

import numpy as np

from build_ref import LIB, build


def load():
    """The reference kernels, or None when neither the library nor the
    reference tree is available."""
    p = build()
    if p is None or not p.exists():
        return None
    lib = ctypes.CDLL(str(p))
    f = lib.tmdr_pair_forces
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int] * 7 + [ctypes.c_void_p] * 12
    return lib


def monomials(u):
    x, y, z = u[..., 0], u[..., 1], u[..., 2]
    one = np.ones_like(x)
    return np.stack([one, x, y, z, x * x, x * y, x * z, y * y, y * z, z * z,
                     x * x * x, x * x * y, x * x * z, x * y * y, x * y * z, x * z * z,
                     y * y * y, y * y * z, y * z * z, z * z * z], -1)


def t_tensor(max_moment, tsym=False):
    D = {0: 1, 1: 4, 2: 10, 3: 20}[max_moment]
    T = np.zeros((max_moment + 1, D))
    T[0, 0] = 1.0
    if max_moment > 0:
        T[1, 1:4] = 1.0
    if max_moment > 1:
        T[2, 4:10] = [1, 2, 2, 1, 2, 1]
        if tsym:
            T[2, 0] = -1.0 / 3.0
    if max_moment > 2:
        T[3, 10:20] = [1, 3, 3, 3, 6, 3, 1, 3, 3, 1]
        if tsym:
            T[3, 1:4] = -3.0 / 5.0
    return T


def block_index(nelt):
    e = np.zeros((nelt, nelt), dtype=np.int64)
    for i in range(nelt):
        k = 1
        for j in range(nelt):
            if i == j:
                e[i, j] = 0
            else:
                e[i, j] = k
                k += 1
    return e


def gaussian_sf(pot, r):
    """H[..., k], dH/dr[..., k] of the analytic Gaussian basis (method 3) with
    the cosine cutoff (fctype 0)."""
    rc = float(np.asarray(pot["rmax"]).ravel()[0])
    eta = np.asarray(pot["descriptor::eta"], dtype=np.float64)
    om = np.asarray(pot["descriptor::omega"], dtype=np.float64)
    d = r[..., None] - om
    f = np.exp(-eta * d * d / (rc * rc))
    df = -2.0 * eta * d / (rc * rc) * f
    fc = 0.5 * (np.cos(np.pi * r / rc) + 1.0)[..., None]
    dfc = (-0.5 * np.pi / rc * np.sin(np.pi * r / rc))[..., None]
    return fc * f, dfc * f + fc * df


def pair_forces(lib, pot, x, elem, box, nlist, G, dEdG):
    """Reference-kernel P, S and forces for the atoms x (elem 0-based), the
    full neighbor list nlist = (off, ent[j, sx, sy, sz]) and the MLP's G and
    raw dE/dG rows [n][B*K*M]."""
    n = len(x)
    nelt = int(np.asarray(pot["nelt"]).ravel()[0])
    mm = int(np.asarray(pot["max_moment"]).ravel()[0])
    rc = float(np.asarray(pot["rmax"]).ravel()[0])
    K = len(np.asarray(pot["descriptor::eta"]))
    D = {0: 1, 1: 4, 2: 10, 3: 20}[mm]
    M = mm + 1
    tsym = int(np.asarray(pot.get("is_T_symmetric", 0)).ravel()[0]) == 1
    eb = block_index(nelt)
    off, ent = nlist
    a_vec = np.array([box[3], 0, 0]), np.array([box[6], box[4], 0]), np.array([box[7], box[8], box[5]])
    pairs = []  # (i, b, j, dvec)
    for i in range(n):
        for s in range(off[i], off[i + 1]):
            j, sx, sy, sz = ent[s]
            dv = x[j] + sx * a_vec[0] + sy * a_vec[1] + sz * a_vec[2] - x[i]
            r2 = float(dv @ dv)
            if r2 < rc * rc and r2 > 1e-10:
                pairs.append((i, eb[elem[i], elem[j]], j, dv))
    cnt = np.zeros((n, nelt), dtype=np.int64)
    for i, b, _, _ in pairs:
        cnt[i, b] += 1
    C = max(1, int(cnt.max()))
    slot = np.zeros((n, nelt), dtype=np.int64)
    dvec = np.zeros((n, nelt, C, 3))
    mask = np.zeros((n, nelt, C), dtype=np.int32)
    partner = -np.ones((n, nelt, C), dtype=np.int64)
    for i, b, j, dv in pairs:
        c = slot[i, b]
        slot[i, b] += 1
        dvec[i, b, c] = dv
        mask[i, b, c] = 1
        partner[i, b, c] = j
    R = np.linalg.norm(dvec, axis=-1)
    Rs = np.where(mask > 0, R, 1.0)
    u = dvec / Rs[..., None] * mask[..., None]
    Mm = monomials(u)[..., :D] * mask[..., None]
    H, dH = gaussian_sf(pot, Rs)
    H *= mask[..., None]
    dH *= mask[..., None]
    T = t_tensor(mm, tsym)
    Gr = np.ascontiguousarray(np.asarray(G, dtype=np.float64).reshape(n, nelt, K, M))
    dG = np.ascontiguousarray(np.asarray(dEdG, dtype=np.float64).reshape(n, nelt, K, M))
    P = np.zeros((n, nelt, K, D))
    S = np.zeros((n, nelt, K, D))
    F = np.zeros((n, nelt, C, 3))
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (Mm, H, dH, u, Rs)]
    mask = np.ascontiguousarray(mask)
    T = np.ascontiguousarray(T)
    rc_ = lib.tmdr_pair_forces(n, nelt, C, K, D, M, mm, *(a.ctypes.data for a in arrs),
                               mask.ctypes.data, T.ctypes.data, Gr.ctypes.data, dG.ctypes.data,
                               P.ctypes.data, S.ctypes.data, F.ctypes.data)
    assert rc_ == 0
    f = np.zeros((n, 3))
    for i in range(n):
        for b in range(nelt):
            for c in range(C):
                if mask[i, b, c]:
                    f[i] += F[i, b, c]
                    f[partner[i, b, c]] -= F[i, b, c]
    return dict(P=P, S=S, F=F, f=f, T=T)


def invariants(P, T):
    """G = T P^2 with G0 = sign(P0) sqrt(.) (kernel.cu:1028-1061)."""
    G = np.einsum("md,nbkd->nbkm", T, P * P)
    G[..., 0] = np.sign(P[..., 0]) * np.sqrt(G[..., 0])
    return G
