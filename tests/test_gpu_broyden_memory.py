"""Broyden memory across steps (fs_set_broyden_memory): host-driven and captured
steps give bitwise the same trajectory; all-zero settings are the reference's
iteration; the steps still converge to the tolerance; an upload that repeats the
state keeps the carried state and one that changes it drops it; the restart and
the ensemble path; argument checks."""
import numpy as np
import pytest

from filsim_b200 import abi
from filsim_b200.configs import make_sediment_case
from filsim_b200.ensemble import Ensemble
from filsim_b200.fcm import Context, Simulation

pytestmark = pytest.mark.gpu

KEYS = ("X", "q", "lam", "U")
POLICY = (8, 3, 4, 12)  # keep_columns, carry_columns, threshold, restart_after


def make(prec=abi.FS_PREC_FP32, graph=True, memory=POLICY, seed=21, nfil=24):
    p, s = make_sediment_case(64, nfil, 8, seed)
    ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
    ctx.set_precision(prec)
    abi.check(abi.lib().fs_set_graph_mode(ctx.h, 1 if graph else 0), "fs_set_graph_mode")
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


@pytest.mark.parametrize("memory", [POLICY, (16, 0, 1000, 0), (0, 4, 0, 6)])
def test_host_and_graph(gpu_lib, memory):
    its_h, st_h, out_h = run(graph=False, memory=memory)
    its_g, st_g, out_g = run(graph=True, memory=memory)
    assert st_h == abi.FS_OK and st_g == abi.FS_OK
    assert np.array_equal(its_h, its_g)
    assert same(out_h, out_g)


def test_off_is_the_reference_iteration(gpu_lib):
    its_0, _, out_0 = run(memory=None)
    ctx, s = make(memory=POLICY)
    ctx.set_broyden_memory(0, 0, 0, 0)
    sim = Simulation(ctx, s)
    its_1, _ = sim.run_steps(1, 24)
    out_1 = sim.download()
    ctx.close()
    assert np.array_equal(its_0, its_1)
    assert same(out_0, out_1)


def test_converges_to_the_same_solution(gpu_lib):
    """Every step ends within the tolerance from either start of its iteration:
    FP64, the memory's trajectory (another path: other iteration counts) stays
    within the tolerance's reach of the reference iteration's."""
    its_0, st_0, out_0 = run(prec=abi.FS_PREC_FP64, memory=None, nsteps=30)
    its_m, st_m, out_m = run(prec=abi.FS_PREC_FP64, memory=POLICY, nsteps=30)
    assert st_0 == abi.FS_OK and st_m == abi.FS_OK
    dx = 1.0 / 1.86
    assert np.abs(out_m["X"] - out_0["X"]).max() / dx < 1e-4
    assert not np.array_equal(its_m, its_0)


def test_upload_keeps_or_drops(gpu_lib):
    # continuous run
    ctx, s = make()
    sim = Simulation(ctx, s.copy())
    its_c = np.concatenate([sim.run_steps(1, 16)[0], sim.run_steps(17, 8)[0]])
    out_c = sim.download()
    ctx.close()
    # the same, with the state downloaded and uploaded again between steps 16 and 17
    ctx, s2 = make()
    sim = Simulation(ctx, s2.copy())
    its_a, _ = sim.run_steps(1, 16)
    mid = s2.copy()
    sim.download_into(mid)
    sim.upload(mid)
    its_b, _ = sim.run_steps(17, 8)
    assert np.array_equal(np.concatenate([its_a, its_b]), its_c)
    assert same(sim.download(), out_c)
    # another state of the same layout: the carried state goes, as in a fresh context
    other = s.copy()
    sim0 = Simulation(ctx, other)
    its_o, _ = sim0.run_steps(1, 20)
    out_o = sim0.download()
    ctx.close()
    its_f, _, out_f = run(nsteps=20)
    assert np.array_equal(its_o, its_f)
    assert same(out_o, out_f)


def test_restart(gpu_lib):
    """restart_after 1: every step on carried state that needs a second iteration
    rebuilds J0 there and starts its history afresh."""
    memory = (32, 0, 1000, 1)
    its_h, st_h, out_h = run(graph=False, memory=memory)
    its_g, st_g, out_g = run(graph=True, memory=memory)
    assert st_h == abi.FS_OK and st_g == abi.FS_OK
    assert np.array_equal(its_h, its_g) and same(out_h, out_g)
    its_0, _, _ = run(memory=None)
    assert not np.array_equal(its_h, its_0)


def test_ensemble_with_memory(gpu_lib):
    boxes = []
    for i, (npts, nfil) in enumerate([(32, 3), (48, 6), (64, 10)]):
        p, s = make_sediment_case(npts, nfil, 8, 600 + i)
        boxes.append((npts, p, s, 1.0))
    ens = Ensemble(boxes, precision=abi.FS_PREC_FP32, memory=POLICY)
    ens.startup(13)
    its, _, _, st = ens.run(14, 5)
    outs = [sim.download() for sim in ens.sims]
    ens.close()
    assert st == abi.FS_OK
    for b, (npts, p, s, kb) in enumerate(boxes):
        ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
        ctx.set_precision(abi.FS_PREC_FP32)
        ctx.set_broyden_memory(*POLICY)
        sim = Simulation(ctx, s)
        ref_its, _ = sim.run_steps(1, 18)
        ref = sim.download()
        ctx.close()
        assert list(its[:, b]) == list(ref_its[13:]), b
        assert same(outs[b], ref), b


def test_invalid(gpu_lib):
    ctx, _ = make(memory=None)
    f = abi.lib().fs_set_broyden_memory
    for args in ((-1, 0, 0, 0), (0, -1, 0, 0), (4, 0, -1, 0), (4, 0, 0, -1), (65, 0, 0, 0), (0, 65, 0, 0)):
        assert f(ctx.h, *args) == abi.FS_ERR_INVALID_ARG, args
    assert f(ctx.h, 64, 64, 8, 20) == abi.FS_OK
    ctx.close()
