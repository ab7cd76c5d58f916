"""Velocity predictor (fs_set_velocity_predictor): host-driven and captured steps
give bitwise the same trajectory, alone and with the Broyden memory; weight 0 is
the reference's iteration; without two converged states the update is zero; the
steps still converge to the tolerance; uploads keep or drop the velocity history;
the ensemble path; argument checks."""
import math

import numpy as np
import pytest

from filsim_b200 import abi
from filsim_b200.configs import make_sediment_case
from filsim_b200.ensemble import Ensemble
from filsim_b200.fcm import Context, Simulation

pytestmark = pytest.mark.gpu

KEYS = ("X", "q", "lam", "U")
MEMORY = (8, 3, 4, 12)


def make(prec=abi.FS_PREC_FP32, graph=True, weight=0.5, memory=None, seed=31, nfil=24):
    p, s = make_sediment_case(64, nfil, 8, seed)
    ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
    ctx.set_precision(prec)
    abi.check(abi.lib().fs_set_graph_mode(ctx.h, 1 if graph else 0), "fs_set_graph_mode")
    if weight is not None:
        ctx.set_velocity_predictor(weight)
    if memory is not None:
        ctx.set_broyden_memory(*memory)
    return ctx, s


def run(nsteps=24, **kw):
    ctx, s = make(**kw)
    sim = Simulation(ctx, s)
    its, st = sim.run_steps(1, nsteps)
    out = sim.download()
    ctx.close()
    return its, st, out


def same(a, b):
    return all(np.array_equal(a[k], b[k]) for k in KEYS)


@pytest.mark.parametrize("weight,memory", [(0.5, None), (1.0, None), (0.5, MEMORY)])
def test_host_and_graph(gpu_lib, weight, memory):
    its_h, st_h, out_h = run(graph=False, weight=weight, memory=memory)
    its_g, st_g, out_g = run(graph=True, weight=weight, memory=memory)
    assert st_h == abi.FS_OK and st_g == abi.FS_OK
    assert np.array_equal(its_h, its_g)
    assert same(out_h, out_g)


def test_zero_weight_and_first_steps(gpu_lib):
    its_0, _, out_0 = run(weight=None)
    ctx, s = make(weight=0.5)
    ctx.set_velocity_predictor(0.0)
    sim = Simulation(ctx, s)
    its_1, _ = sim.run_steps(1, 24)
    out_1 = sim.download()
    ctx.close()
    assert np.array_equal(its_0, its_1) and same(out_0, out_1)
    # steps 1 and 2 have fewer than two converged states before them: zero update
    its_a, _, out_a = run(nsteps=2, weight=None)
    its_b, _, out_b = run(nsteps=2, weight=0.5)
    assert np.array_equal(its_a, its_b) and same(out_a, out_b)
    its_c, _, _ = run(nsteps=24, weight=0.5)
    assert not np.array_equal(its_c, its_0)


def test_converges_to_the_same_solution(gpu_lib):
    its_0, st_0, out_0 = run(prec=abi.FS_PREC_FP64, weight=None, nsteps=30)
    its_p, st_p, out_p = run(prec=abi.FS_PREC_FP64, weight=0.5, memory=MEMORY, nsteps=30)
    assert st_0 == abi.FS_OK and st_p == abi.FS_OK
    dx = 1.0 / 1.86
    assert np.abs(out_p["X"] - out_0["X"]).max() / dx < 1e-4


def test_upload_keeps_or_drops(gpu_lib):
    ctx, s = make(memory=MEMORY)
    sim = Simulation(ctx, s.copy())
    its_c = np.concatenate([sim.run_steps(1, 16)[0], sim.run_steps(17, 8)[0]])
    out_c = sim.download()
    ctx.close()
    ctx, s2 = make(memory=MEMORY)
    sim = Simulation(ctx, s2.copy())
    its_a, _ = sim.run_steps(1, 16)
    mid = s2.copy()
    sim.download_into(mid)
    sim.upload(mid)
    its_b, _ = sim.run_steps(17, 8)
    assert np.array_equal(np.concatenate([its_a, its_b]), its_c)
    assert same(sim.download(), out_c)
    sim0 = Simulation(ctx, s.copy())  # other positions: the velocity history goes
    its_o, _ = sim0.run_steps(1, 20)
    out_o = sim0.download()
    ctx.close()
    its_f, _, out_f = run(nsteps=20, memory=MEMORY)
    assert np.array_equal(its_o, its_f) and same(out_o, out_f)


def test_ensemble(gpu_lib):
    boxes = []
    for i, (npts, nfil) in enumerate([(32, 3), (48, 6), (64, 10)]):
        p, s = make_sediment_case(npts, nfil, 8, 700 + i)
        boxes.append((npts, p, s, 1.0))
    ens = Ensemble(boxes, precision=abi.FS_PREC_FP32, memory=MEMORY, predictor=0.5)
    ens.startup(13)
    its, _, _, st = ens.run(14, 5)
    outs = [sim.download() for sim in ens.sims]
    ens.close()
    assert st == abi.FS_OK
    for b, (npts, p, s, kb) in enumerate(boxes):
        ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
        ctx.set_precision(abi.FS_PREC_FP32)
        ctx.set_broyden_memory(*MEMORY)
        ctx.set_velocity_predictor(0.5)
        sim = Simulation(ctx, s)
        ref_its, _ = sim.run_steps(1, 18)
        ref = sim.download()
        ctx.close()
        assert list(its[:, b]) == list(ref_its[13:]), b
        assert same(outs[b], ref), b


def test_invalid(gpu_lib):
    ctx, _ = make(weight=None)
    f = abi.lib().fs_set_velocity_predictor
    for w in (-0.1, 2.5, math.nan, math.inf):
        assert f(ctx.h, w) == abi.FS_ERR_INVALID_ARG, w
    assert f(ctx.h, 2.0) == abi.FS_OK
    ctx.close()
