"""Seeded synthetic filament suspensions (the benchmark inputs).

Each filament is straight: one random unit quaternion, normalised from four
N(0,1) draws as Bead::initialBeadRandom does (Bead.hpp:94-98), is shared by all
of its beads; bead n sits at C + (n*DL - Nw*DL/2) t with t the quaternion's
tangent, the placement of Filament::initialFilamentSetupIsoRandCentred
(Filament.cpp:47-66). Centres C are uniform in the periodic box and a proposal
is rejected while any of its beads lies closer than `min_sep` (minimum image)
to an accepted bead or to a periodic image of its own beads, the test of
Filament::checkOverlapWithPeriodic (Filament.cpp:126-153) with the separation
the benchmark configurations state (2.2a) instead of the reference's 2(a+a).

The random stream is numpy's PCG64 seeded with `seed`; the reference's
Armadillo RNG is not reproduced.
"""
import ctypes

import numpy as np

from .abi import FsHostState, P_double, P_int, box_lengths


def quat_tangent(q):
    """assignTangentVec (UnitQuaternion.hpp:341-351) for an (n, 4) array."""
    s, x, y, z = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    q22 = 2 * y * y
    q33 = 2 * z * z
    return np.stack([(1 - q22 - q33), 2 * (x * y + s * z), 2 * (x * z - s * y)], axis=1)


class _HostState:
    def __init__(self, arrays, fil_start, nfil, np_):
        self.arrays = arrays
        self.fil_start = fil_start
        st = FsHostState()
        st.nfil = nfil
        st.np = np_
        st.fil_start = fil_start.ctypes.data_as(P_int)
        for k, v in arrays.items():
            setattr(st, k, v.ctypes.data_as(P_double) if v is not None else None)
        self.struct = st


class Suspension:
    """A filament suspension in the fs_host_state layout (numpy, host)."""

    STATE3 = ("X", "Xs", "Xt", "U", "Us", "Ut", "F", "TAU")
    STATE4 = ("q", "qs", "qt")
    LAMS = ("lam", "lam1", "lam2")

    def __init__(self, fil_start, X, q, kap=1.0, c=1.0):
        self.fil_start = np.ascontiguousarray(fil_start, dtype=np.int32)
        self.nfil = len(self.fil_start) - 1
        self.np = int(self.fil_start[-1])
        self.nlink = self.np - self.nfil
        X = np.ascontiguousarray(X, dtype=np.float64).reshape(self.np, 3)
        q = np.ascontiguousarray(q, dtype=np.float64).reshape(self.np, 4)
        self.arrays = {}
        for k in ("X", "Xs", "Xt"):
            self.arrays[k] = X.copy()
        for k in ("U", "Us", "Ut", "F", "TAU"):
            self.arrays[k] = np.zeros((self.np, 3))
        for k in self.STATE4:
            self.arrays[k] = q.copy()
        for k in self.LAMS:
            self.arrays[k] = np.zeros((self.nlink, 3))
        self.arrays["kap"] = np.broadcast_to(np.asarray(kap, dtype=np.float64), (self.nfil,)).copy()
        self.arrays["c"] = np.broadcast_to(np.asarray(c, dtype=np.float64), (self.nfil,)).copy()

    def __getattr__(self, k):
        arrays = self.__dict__.get("arrays")
        if arrays is not None and k in arrays:
            return arrays[k]
        raise AttributeError(k)

    @property
    def fil_id(self):
        return np.repeat(np.arange(self.nfil, dtype=np.int32), np.diff(self.fil_start))

    @property
    def seg_id(self):
        return (np.arange(self.np) - np.repeat(self.fil_start[:-1], np.diff(self.fil_start))).astype(np.int32)

    def host_state(self):
        return _HostState(self.arrays, self.fil_start, self.nfil, self.np)

    def empty_like_state(self):
        arrays = {k: np.zeros_like(v) for k, v in self.arrays.items()}
        return _HostState(arrays, self.fil_start, self.nfil, self.np)

    def copy(self):
        out = Suspension.__new__(Suspension)
        out.fil_start = self.fil_start.copy()
        out.nfil, out.np, out.nlink = self.nfil, self.np, self.nlink
        out.arrays = {k: v.copy() for k, v in self.arrays.items()}
        return out

    def set_arrays(self, arrays):
        for k, v in arrays.items():
            self.arrays[k][...] = v


def random_suspension(p, nfil, nw, seed, min_sep=None, kap=1.0, c=1.0, max_tries=2000):
    """Rejection-placed straight filaments in the periodic box of params p."""
    rng = np.random.Generator(np.random.PCG64(seed))
    L = np.array(box_lengths(p))
    dl = p.dl
    if min_sep is None:
        min_sep = 2.2 * p.a
    M = np.maximum((L / min_sep).astype(int), 1)
    cell = L / M
    cap = 8
    grid = -np.ones((M[0], M[1], M[2], cap), dtype=np.int64)
    fill = np.zeros((M[0], M[1], M[2]), dtype=np.int64)
    X = np.zeros((nfil * nw, 3))
    Q = np.zeros((nfil * nw, 4))
    offs = np.array([(i, j, k) for i in (-1, 0, 1) for j in (-1, 0, 1) for k in (-1, 0, 1)])
    n_idx = np.arange(nw)
    placed = 0
    for f in range(nfil):
        for _ in range(max_tries):
            q = rng.standard_normal(4)
            q = q / np.sqrt(np.sum(q * q))
            centre = rng.random(3) * L
            t = quat_tangent(q[None, :])[0]
            pos = centre[None, :] + (n_idx[:, None] * dl - nw * dl / 2.0) * t[None, :]
            # own periodic images
            d = pos[:, None, :] - pos[None, :, :]
            dmi = d - L * np.floor(d / L + 0.5)
            wrapped = np.any(np.abs(dmi - d) > 1e-9, axis=2)
            r2 = np.sum(dmi * dmi, axis=2)
            if np.any(wrapped & (r2 < min_sep * min_sep)):
                continue
            if placed:
                wpos = pos - L * np.floor(pos / L)
                ci = np.minimum((wpos / cell).astype(int), M - 1)
                nb = (ci[:, None, :] + offs[None, :, :]) % M
                cand = grid[nb[..., 0], nb[..., 1], nb[..., 2]].reshape(nw, -1)
                ok = True
                if np.any(cand >= 0):
                    cidx = np.where(cand >= 0, cand, 0)
                    dd = pos[:, None, :] - X[cidx]
                    dd = dd - L * np.floor(dd / L + 0.5)
                    rr = np.sum(dd * dd, axis=2)
                    if np.any((cand >= 0) & (rr < min_sep * min_sep)):
                        ok = False
                if not ok:
                    continue
            wpos = pos - L * np.floor(pos / L)
            ci = np.minimum((wpos / cell).astype(int), M - 1)
            for b in range(nw):
                cx, cy, cz = ci[b]
                k = fill[cx, cy, cz]
                if k >= cap:
                    raise RuntimeError("placement grid cell overflow")
                grid[cx, cy, cz, k] = placed + b
                fill[cx, cy, cz] = k + 1
            X[placed:placed + nw] = pos
            Q[placed:placed + nw] = q[None, :]
            placed += nw
            break
        else:
            raise RuntimeError("could not place filament %d after %d tries" % (f, max_tries))
    fil_start = np.arange(nfil + 1, dtype=np.int32) * nw
    return Suspension(fil_start, X, Q, kap=kap, c=c)


def random_forces(np_, seed):
    """Per-bead forces and torques, i.i.d. N(0,1) per component."""
    rng = np.random.Generator(np.random.PCG64(seed))
    F = rng.standard_normal((np_, 3))
    T = rng.standard_normal((np_, 3))
    return F, T


def fcm_positions(p, X):
    """Fcm::assign_filament_data position rule: Y = fmod(X, L) (FCMfunctions.cpp:902-904)."""
    L = np.array(box_lengths(p))
    return np.fmod(X, L)
