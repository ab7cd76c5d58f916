"""Regenerates the golden fixtures of this directory from the CPU oracle.

    python tests/golden/make_golden.py

The reference itself (MPI + FFTW 2.1.5 + Armadillo) cannot be built in this
environment and publishes no vectors, so these fixtures hold the oracle's
outputs on seeded inputs; the CPU tests check the oracle still reproduces them
and the GPU tests compare the kernels against them.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from filsim_b200.configs import make_mobility_case, params_for, sediment_params  # noqa: E402
from filsim_b200.suspension import random_suspension, fcm_positions  # noqa: E402
from oracle import oracle_py as O  # noqa: E402


def dense_barrier_case(seed=11, nfil=40, nw=6, npts=32, jitter=0.35):
    p = params_for(npts)
    s = random_suspension(p, nfil, nw, seed, min_sep=1.2)
    rng = np.random.default_rng(seed)
    X = s.X + jitter * rng.standard_normal(s.X.shape)
    X[::7] += np.array([1.0, -1.0, 0.5]) * (npts * p.dx)
    return p, s, X


def main():
    O.build()
    # FCM mobility, 64^3, 480 beads
    p, s, Y, F, T = make_mobility_case(64, 32, 15, seed=1000)
    V, W = O.fcm_mobility(p, Y, F, T)
    np.savez_compressed(os.path.join(HERE, "mobility_64.npz"), Y=Y, F=F, T=T, V=V, W=W)
    # collision barrier on a dense suspension
    p, s, X = dense_barrier_case()
    F0 = np.random.default_rng(11).standard_normal((s.np, 3))
    head, lst, mp = O.cells_link(p, X)
    r = O.collision_barrier(p, fcm_positions(p, X), F0, s.fil_id, s.seg_id, head, lst, mp, 5, max_pairs=1 << 16)
    np.savez_compressed(os.path.join(HERE, "barrier_dense.npz"), X=X, F0=F0, fil_id=s.fil_id, seg_id=s.seg_id,
                        head=head, list=lst, pairs=r["pairs"], F=r["F"], min_dist2=r["min_dist2"])
    # implicit BDF2 steps of a small sedimenting suspension
    p = sediment_params(32, tol=1e-10, broyden_maxiter=100)
    s = random_suspension(p, 6, 8, seed=31)
    sysw = O.System(p, s)
    its, _ = sysw.run_steps(1, 10)
    out = sysw.download()
    np.savez_compressed(os.path.join(HERE, "steps_small.npz"), X0=s.X, q0=s.q, X=out["X"], q=out["q"],
                        lam=out["lam"], iters=its)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
