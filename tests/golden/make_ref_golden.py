"""Writes tests/golden/ref_pin.npz: inputs and outputs of the REFERENCE'S OWN
FCM mobility solve (Fcm::mobility_solve, FCMfunctions.cpp:175-464) and
collision barrier (LinkedList::link + apply_collision_barrier,
CollisionBarrierFilament.cpp:24-433), built from the FilSim sources by
oracle/refshim (one process; MPI and FFTW 2.1.5 replaced by the stand-ins
there). The GPU tests compare the library with these without needing the
FilSim tree.

    python tests/golden/make_ref_golden.py      (after `make -C oracle/refshim`)
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from filsim_b200.abi import make_params  # noqa: E402
from filsim_b200.configs import params_for  # noqa: E402
from filsim_b200.suspension import fcm_positions, random_forces  # noqa: E402
from oracle import oracle_py  # noqa: E402


def barrier_case(seed, nfil=40, nw=6, npts=32, jitter=0.35):
    """Filaments packed closer than the barrier range, some beads outside the box."""
    p = params_for(npts)
    X, Q = oracle_py.suspension_random(p, nfil, nw, seed, min_sep=1.2)
    X = X + jitter * np.random.default_rng(seed).standard_normal(X.shape)
    X[::7] += np.array([1.0, -1.0, 0.5]) * (npts * p.dx)
    return p, X, np.arange(nfil + 1, dtype=np.int32) * nw


def main():
    out = {}
    # 64^3, 32 filaments x 15 beads, F, T ~ N(0, 1): the mobility_64 workload
    p = params_for(64)
    X, Q = oracle_py.suspension_random(p, 32, 15, 1000)
    F, T = random_forces(X.shape[0], 1007)
    Y = fcm_positions(p, X)
    V, W = oracle_py.ref_fcm_mobility("fcm_64_ngd12", Y, F, T)
    out.update(m64_Y=Y, m64_F=F, m64_T=T, m64_V=V, m64_W=W)
    # the reference's default stencil on a non-cubic grid: ngd 20, dx = sigma_dip / 1.5
    p = make_params((48, 32, 64), ngd=20)
    X, Q = oracle_py.suspension_random(p, 8, 4, 42, min_sep=1.5)
    X[::3] -= np.array([48, 32, 64]) * p.dx
    F, T = random_forces(X.shape[0], 43)
    Y = fcm_positions(p, X)
    V, W = oracle_py.ref_fcm_mobility("fcm_48x32x64_ngd20", Y, F, T)
    out.update(n20_Y=Y, n20_F=F, n20_T=T, n20_V=V, n20_W=W)
    # dense barrier cases: nt = 5, and nt = 0 below initialFrictionSteps = 1
    for key, seed, nt, lib in (("b11", 11, 5, "barrier_32"), ("b13", 13, 0, "barrier_32_friction1")):
        p, X, fil_start = barrier_case(seed)
        Y = fcm_positions(p, X)
        F0 = np.random.default_rng(seed).standard_normal((X.shape[0], 3))
        F, head, lst, md = oracle_py.ref_barrier(lib, fil_start, X, Y, F0, nt)
        out.update({key + "_X": X, key + "_F0": F0, key + "_fil_start": fil_start, key + "_F": F,
                    key + "_head": head, key + "_list": lst, key + "_min_dist2": np.array(md),
                    key + "_nt": np.array(nt)})
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_pin.npz"), **out)


if __name__ == "__main__":
    main()
