"""Precision escalation (fs_set_precision_escalation): an FP32 step still not
converged after k Broyden iterations runs the rest with the FP64 chain; captured
steps do it with a second loop node whose body is the FP64 chain, bitwise the
host-driven steps; a k no step reaches changes nothing; FP64 contexts ignore it."""
import numpy as np
import pytest

from filsim_b200 import abi
from filsim_b200.configs import make_sediment_case
from filsim_b200.fcm import Context, Simulation

pytestmark = pytest.mark.gpu


def run(escalate, graph, prec=abi.FS_PREC_FP32, nsteps=20, seed=13):
    p, s = make_sediment_case(64, 16, 8, seed)
    ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
    ctx.set_precision(prec)
    abi.check(abi.lib().fs_set_graph_mode(ctx.h, 1 if graph else 0), "fs_set_graph_mode")
    abi.check(abi.lib().fs_set_precision_escalation(ctx.h, escalate), "fs_set_precision_escalation")
    sim = Simulation(ctx, s)
    its, st = sim.run_steps(1, nsteps)
    d = sim.diag()
    out = sim.download()
    ctx.close()
    return its, st, d, out


def test_escalation_host_and_graph(gpu_lib):
    its_h, st_h, d_h, out_h = run(2, graph=False)
    its_g, st_g, d_g, out_g = run(2, graph=True)
    assert st_h == abi.FS_OK and st_g == abi.FS_OK
    assert np.array_equal(its_h, its_g)
    assert d_h.escalated_iters == d_g.escalated_iters
    # every step past two iterations ran the rest in FP64
    assert d_h.escalated_iters == int(np.maximum(its_h - 2, 0).sum()) > 0
    for k in ("X", "q", "lam", "U"):
        assert np.array_equal(out_h[k], out_g[k]), k


def test_unreached_escalation_changes_nothing(gpu_lib):
    its_0, _, d_0, out_0 = run(0, graph=True)
    its_1, _, d_1, out_1 = run(10000, graph=True)
    assert np.array_equal(its_0, its_1)
    assert d_0.escalated_iters == 0 and d_1.escalated_iters == 0
    for k in ("X", "q", "lam", "U"):
        assert np.array_equal(out_0[k], out_1[k]), k


def test_escalation_converges_like_fp64(gpu_lib):
    """Escalating after one iteration, the FP32 steps take the FP64 chain for all but
    their first iteration: the trajectory stays within the FP32 chain's error of the
    FP64 one."""
    its_e, st_e, d_e, out_e = run(1, graph=True)
    its_64, st_64, _, out_64 = run(0, graph=True, prec=abi.FS_PREC_FP64)
    assert st_e == abi.FS_OK and st_64 == abi.FS_OK
    assert d_e.escalated_iters > 0
    dx = 1.0 / 1.86
    assert np.abs(out_e["X"] - out_64["X"]).max() / dx < 1e-5


def test_fp64_and_invalid(gpu_lib):
    _, _, d, _ = run(2, graph=False, prec=abi.FS_PREC_FP64, nsteps=14)
    assert d.escalated_iters == 0
    p, s = make_sediment_case(32, 4, 6, 3)
    ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
    assert abi.lib().fs_set_precision_escalation(ctx.h, -1) == abi.FS_ERR_INVALID_ARG
    ctx.close()
