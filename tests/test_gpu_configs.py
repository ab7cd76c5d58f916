"""Parity at the benchmark configurations' own sizes, where index arithmetic that
small cases never reach is exercised: 256^3 and 512^3 grids (byte offsets past
2^31), 110^3 collision cells, 131,072 beads, and a trajectory at the 512^3
suspension's bead density.

- 256^3, 1024 x 30 beads, F, T ~ N(0, 1) (the mixed-precision comparison
  workload): FP64 U, Omega within 1e-10 of the oracle (FCMfunctions.cpp:175-464),
  FP32 within 1e-5 of FP64.
- 512^3, the 4096 x 32 sedimentation suspension: one FP64 solve within 1e-10 of
  the oracle, FP32 within 1e-5 of FP64.
- 512^3 collision cells (110^3) with jittered positions: head/list, pair list,
  forces and minimum distance bit for bit (CollisionBarrierFilament.cpp:24-433).
- 128 x 64 x 64 with 16 x 32 beads (one bead per 1024 grid points, the 512^3
  suspension's density): 50 implicit steps at the benchmark tolerance 1e-6 with
  equal Broyden iteration counts per step and positions within 1e-8 of the box
  (main.cpp:284-754).
"""
import numpy as np
import pytest
import torch

from filsim_b200 import abi
from filsim_b200.configs import make_mobility_case, make_sediment_case, sediment_params
from filsim_b200.fcm import Context, Fcm, LinkedList, Simulation
from filsim_b200.suspension import fcm_positions, random_forces, random_suspension

pytestmark = pytest.mark.gpu

FP64_REL = 1e-10
FP32_REL = 1e-5


def rel_err(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max()


def gpu_solves(p, Y, F, T):
    """FP64 and FP32 mobility solves of the same inputs in one context."""
    ctx = Context(p, max_beads=Y.shape[0])
    fcm = Fcm(ctx, Y.shape[0])
    fcm.set(Y, F, T)
    out = {}
    for name, prec in (("fp64", abi.FS_PREC_FP64), ("fp32", abi.FS_PREC_FP32)):
        ctx.set_precision(prec)
        fcm.mobility_solve()
        ctx.synchronize()
        out[name] = (fcm.V.cpu().numpy(), fcm.W.cpu().numpy())
    ctx.close()
    torch.cuda.empty_cache()
    return out


def check_solves(out, V0, W0):
    V, W = out["fp64"]
    assert rel_err(V, V0) < FP64_REL
    assert rel_err(W, W0) < FP64_REL
    V32, W32 = out["fp32"]
    assert rel_err(V32, V) < FP32_REL
    assert rel_err(W32, W) < FP32_REL


def test_mobility_256_cube_30720_beads(oracle, gpu_lib):
    p, s, Y, F, T = make_mobility_case(256, 1024, 30, seed=1001)
    V0, W0 = oracle.fcm_mobility(p, Y, F, T)
    check_solves(gpu_solves(p, Y, F, T), V0, W0)


def test_mobility_512_cube_sedimentation_suspension(oracle, gpu_lib):
    p, s = make_sediment_case(512, 4096, 32, seed=1002)
    Y = fcm_positions(p, s.X)
    F, T = random_forces(s.np, 1009)
    F[:, 2] -= 1.0  # the gravity each bead carries
    out = gpu_solves(p, Y, F, T)
    V0, W0 = oracle.fcm_mobility(p, Y, F, T)
    check_solves(out, V0, W0)


def test_cells_and_barrier_512_cube_bit_exact(oracle, gpu_lib):
    p, s = make_sediment_case(512, 4096, 32, seed=1002)
    X = s.X + 0.45 * np.random.default_rng(17).standard_normal(s.X.shape)
    nt = 5
    F0 = np.random.default_rng(18).standard_normal((s.np, 3))
    head0, lst0, mp0 = oracle.cells_link(p, X)
    assert head0.size == 110 ** 3
    Y = fcm_positions(p, X)
    ref = oracle.collision_barrier(p, Y, F0, s.fil_id, s.seg_id, head0, lst0, mp0, nt, max_pairs=1 << 21)
    assert ref["npairs"] > 1000
    ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
    ll = LinkedList(ctx)
    ll.link(X)
    head, lst, mp = ll.lists()
    Yd = torch.as_tensor(Y, device="cuda")
    Fd = torch.as_tensor(F0.copy(), device="cuda")
    md = ll.apply_collision_barrier(Yd, Fd, nt, s.fil_id, s.seg_id)
    pairs, n = ll.pairs(Yd, nt, s.fil_id, s.seg_id, max_pairs=1 << 21)
    ctx.close()
    assert np.array_equal(head, head0)
    assert np.array_equal(lst, lst0)
    assert np.array_equal(mp, mp0)
    assert n == ref["npairs"]
    assert np.array_equal(pairs, ref["pairs"])
    assert np.array_equal(Fd.cpu().numpy(), ref["F"])
    assert md == ref["min_dist2"]


def test_trajectory_at_the_512_cube_bead_density(oracle, gpu_lib):
    shape = (128, 64, 64)
    p = sediment_params(shape, broyden_maxiter=200)
    s = random_suspension(p, 16, 32, seed=41, kap=1.0, c=1.0)
    assert abs(s.np / np.prod(shape) - 1 / 1024) < 1e-12
    nsteps = 50
    sysw = oracle.System(p, s)
    its0, st0 = sysw.run_steps(1, nsteps)
    ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
    sim = Simulation(ctx, s)
    its1, st1 = sim.run_steps(1, nsteps)
    g = sim.download()
    o = sysw.download()
    ctx.close()
    assert st0 == 0 and st1 == abi.FS_OK
    assert np.array_equal(np.asarray(its1), np.asarray(its0))
    L = shape[0] * p.dx
    assert np.abs(g["X"] - o["X"]).max() / L < 1e-8
    assert np.abs(g["q"] - o["q"]).max() < 1e-8
