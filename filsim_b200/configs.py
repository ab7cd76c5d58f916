"""The benchmark workloads: parameters and seeded synthetic inputs.

mobility_64:   64^3 grid, 32 filaments x 15 beads, F, T ~ N(0,1), one FP64 FCM call
mobility_256:  256^3 grid, 1024 filaments x 30 beads, F, T ~ N(0,1), FP64 and FP32 calls
sediment_512:  512^3 grid, 4096 filaments x 32 beads, gravity (0,0,-1) per bead,
               K_B = K_T = 1, BDF2, dt = 0.05, Broyden tolerance 1e-6, barrier below 2.2a
All share a = 1, mu = 1, dx = a/1.86, sigma = a/sqrt(pi), sigma_dip = a/(36 pi)^(1/6),
12-point Gaussian support per axis.
"""
from .abi import make_params
from .suspension import random_suspension, random_forces, fcm_positions

DX = 1.0 / 1.86

WORKLOADS = {
    "mobility_64": dict(npts=64, nfil=32, nw=15, seed=1000, kind="mobility"),
    "mobility_256": dict(npts=256, nfil=1024, nw=30, seed=1001, kind="mobility"),
    "sediment_512": dict(npts=512, nfil=4096, nw=32, seed=1002, kind="steps"),
}


def params_for(npts, **kw):
    base = dict(ngd=12, a=1.0, dx=DX, tol=1e-6, dt=0.05, impl_euler_steps=1, initial_friction_steps=0,
                broyden_maxiter=300)
    base.update(kw)
    return make_params(npts, **base)


def sediment_params(npts, **kw):
    kw.setdefault("gravity", (0.0, 0.0, -1.0))
    return params_for(npts, **kw)


def make_mobility_case(npts, nfil, nw, seed, **kw):
    p = params_for(npts, **kw)
    s = random_suspension(p, nfil, nw, seed)
    F, T = random_forces(s.np, seed + 7)
    Y = fcm_positions(p, s.X)
    return p, s, Y, F, T


def make_sediment_case(npts, nfil, nw, seed, kap=1.0, c=1.0, **kw):
    p = sediment_params(npts, **kw)
    s = random_suspension(p, nfil, nw, seed, kap=kap, c=c)
    return p, s
