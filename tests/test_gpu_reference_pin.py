"""The GPU library against the reference's own code: tests/golden/ref_pin.npz
holds inputs and outputs of the reference's FCM mobility solve
(FCMfunctions.cpp:175-464) and collision barrier
(CollisionBarrierFilament.cpp:24-433), compiled from the FilSim sources as one
process (oracle/refshim; tests/golden/make_ref_golden.py wrote the file).

- FCM, FP64: U, Omega within 1e-10 of the reference's (64^3 / 480 beads with
  ngd 12; 48 x 32 x 64 with the reference's own stencil, ngd 20 and
  dx = sigma_dip / 1.5, beads outside the box included); FP32 within 1e-5.
- Barrier: head/list, forces and minimum distance bit for bit (nt = 5, and
  nt = 0 below initialFrictionSteps = 1)."""
import os

import numpy as np
import pytest
import torch

from filsim_b200 import abi
from filsim_b200.abi import make_params
from filsim_b200.configs import params_for
from filsim_b200.fcm import Context, Fcm, LinkedList
from filsim_b200.suspension import Suspension, fcm_positions

pytestmark = pytest.mark.gpu

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_pin.npz"))


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max()


def solve(p, Y, F, T, prec):
    ctx = Context(p, max_beads=Y.shape[0])
    ctx.set_precision(prec)
    fcm = Fcm(ctx, Y.shape[0])
    fcm.set(Y, F, T)
    fcm.mobility_solve()
    ctx.synchronize()
    out = fcm.V.cpu().numpy(), fcm.W.cpu().numpy()
    ctx.close()
    return out


@pytest.mark.parametrize("key,params", [("m64", lambda: params_for(64)),
                                        ("n20", lambda: make_params((48, 32, 64), ngd=20))])
def test_gpu_mobility_matches_the_reference_code(gpu_lib, key, params):
    p = params()
    Y, F, T = GOLD[key + "_Y"], GOLD[key + "_F"], GOLD[key + "_T"]
    V0, W0 = GOLD[key + "_V"], GOLD[key + "_W"]
    V, W = solve(p, Y, F, T, abi.FS_PREC_FP64)
    assert rel(V, V0) < 1e-10 and rel(W, W0) < 1e-10
    V32, W32 = solve(p, Y, F, T, abi.FS_PREC_FP32)
    assert rel(V32, V0) < 1e-5 and rel(W32, W0) < 1e-5


@pytest.mark.parametrize("key", ["b11", "b13"])
def test_gpu_barrier_matches_the_reference_code_bit_for_bit(gpu_lib, key):
    p = params_for(32)
    nt = int(GOLD[key + "_nt"])
    if nt == 0:
        p.initial_friction_steps = 1
    X, F0, fil_start = GOLD[key + "_X"], GOLD[key + "_F0"], GOLD[key + "_fil_start"]
    s = Suspension(fil_start, X, np.tile([1.0, 0, 0, 0], (X.shape[0], 1)))
    ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
    ll = LinkedList(ctx)
    ll.link(X)
    head, lst, _ = ll.lists()
    Y = torch.as_tensor(fcm_positions(p, X), device="cuda")
    F = torch.as_tensor(F0.copy(), device="cuda")
    md = ll.apply_collision_barrier(Y, F, nt, s.fil_id, s.seg_id)
    ctx.close()
    assert np.array_equal(head, GOLD[key + "_head"])
    assert np.array_equal(lst, GOLD[key + "_list"])
    assert np.array_equal(F.cpu().numpy(), GOLD[key + "_F"])
    assert md == float(GOLD[key + "_min_dist2"])
