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

The generator runs as host code in libfilsim_gpu (fs_suspension_random):
xoshiro256** seeded through splitmix64, Box-Muller normals. The reference's
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


def random_suspension(p, nfil, nw, seed, min_sep=None, kap=1.0, c=1.0, max_tries=1000000):
    """Rejection-placed straight filaments in the periodic box of params p
    (fs_suspension_random, host code of libfilsim_gpu)."""
    import ctypes
    from .abi import lib, check
    if min_sep is None:
        min_sep = 2.2 * p.a
    X = np.zeros((nfil * nw, 3))
    Q = np.zeros((nfil * nw, 4))
    check(lib().fs_suspension_random(ctypes.byref(p), nfil, nw, seed, min_sep, max_tries,
                                     X.ctypes.data_as(ctypes.c_void_p), Q.ctypes.data_as(ctypes.c_void_p)),
          "fs_suspension_random")
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


def swim_parameters(fil_start, p, K0, Sp4, alpha, beta, phase=0.0, kap=None):
    """Per-filament swimming-drive rows (Alpha, Beta, Phase, Wavenumber,
    AngFrequency) for fs_set_swimming, with the Filament constructor's
    Wavenumber = 2 K0 pi / (Nw dL) and AngFrequency = KAP Sp4 / (4 pi mu (Nw dL)^4)
    (Filament.hpp:135-144); alpha, beta, phase and kap are scalars or per filament
    (kap defaults to 1, the bending modulus the constructor sees)."""
    fil_start = np.asarray(fil_start)
    nfil = fil_start.size - 1
    nw = np.diff(fil_start).astype(np.float64)
    kap = np.ones(nfil) if kap is None else np.broadcast_to(np.asarray(kap, dtype=np.float64), (nfil,))
    length = nw * p.dl
    out = np.zeros((nfil, 5))
    out[:, 0] = alpha
    out[:, 1] = beta
    out[:, 2] = phase
    out[:, 3] = 2 * K0 * np.pi / length
    out[:, 4] = kap * Sp4 / (4 * np.pi * p.mu * length ** 4.)
    return out
