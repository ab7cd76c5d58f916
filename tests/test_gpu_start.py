"""Start order 2 (fs_start.cu, fs_set_start_order): the first bead of each
filament starts from 3X - 3Xt + Xtt once the context holds the positions two
steps back, and from the reference's 2X - Xt (Bead.hpp:202-216) without that
history; tension extrapolation 1 (fs_set_tension_extrapolation): the next
step's tensions 2 lam - lam1 instead of the reference's quadratic. Steps
converge to the reference start's solution within the tolerance, in fewer
Broyden iterations; captured steps are bitwise the host-driven ones; an upload
of other positions drops the history."""
import numpy as np
import pytest

from filsim_b200 import abi
from filsim_b200.configs import make_sediment_case, sediment_params
from filsim_b200.fcm import Context, Simulation

pytestmark = pytest.mark.gpu

NFIL, NW = 24, 16


def prepared(order, seed=5, prec=abi.FS_PREC_FP64, tension=2, **kw):
    p, s = make_sediment_case(64, NFIL, NW, seed, **kw)
    ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
    ctx.set_precision(prec)
    ctx.set_start_order(order)
    ctx.set_tension_extrapolation(tension)
    return ctx, Simulation(ctx, s)


def first_beads(sim):
    return sim.susp.fil_start[:-1]


def test_start_formula_and_history(gpu_lib):
    ctx, sim = prepared(2)
    b0 = first_beads(sim)
    # a fresh context has no history: the reference's start, also on its second step
    a = sim.download()
    sim.initial_guess()
    g = sim.download()
    assert np.array_equal(g["Xs"][b0], (2 * a["X"] - a["Xt"])[b0])
    s1 = sim.susp.copy()
    sim.download_into(s1)
    sim.upload(s1)
    X = []
    for nt in range(1, 7):
        it, st = sim.step_implicit(nt)
        assert st == abi.FS_OK
        X.append(sim.download()["X"].copy())
    sim.initial_guess()
    g = sim.download()
    assert np.array_equal(g["X"], X[-1])
    assert np.array_equal(g["Xs"][b0], ((3 * X[-1] - 3 * X[-2]) + X[-3])[b0])
    # an upload of the same X, Xt keeps the history; other positions drop it
    s = sim.susp.copy()
    sim.download_into(s)
    sim.upload(s)
    sim.initial_guess()
    assert np.array_equal(sim.download()["Xs"][b0], ((3 * X[-1] - 3 * X[-2]) + X[-3])[b0])
    s.arrays["X"][:] += 1e-3
    sim.upload(s)
    sim.initial_guess()
    g = sim.download()
    assert np.array_equal(g["Xs"][b0], (2 * g["X"] - g["Xt"])[b0])
    # one step later the history holds the uploaded Xt, not a step's: still 2X - Xt
    sim.upload(s)
    sim.step_implicit(7)
    sim.initial_guess()
    g = sim.download()
    assert np.array_equal(g["Xs"][b0], (2 * g["X"] - g["Xt"])[b0])
    # two steps: second order again
    x7 = g["X"].copy()
    sim.step_implicit(8)
    x8 = sim.download()["X"].copy()
    sim.step_implicit(9)
    sim.initial_guess()
    g = sim.download()
    assert np.array_equal(g["Xs"][b0], ((3 * g["X"] - 3 * x8) + x7)[b0])
    # order 1 on the same context: the reference's start
    ctx.set_start_order(1)
    sim.initial_guess()
    g = sim.download()
    assert np.array_equal(g["Xs"][b0], (2 * g["X"] - g["Xt"])[b0])
    ctx.close()


STARTS = [(1, 2), (2, 2), (2, 1)]  # (start order, tension extrapolation); (1, 2) is the reference's


def test_same_solution_fewer_iterations(gpu_lib):
    """At TOL 1e-12 every start converges to the same trajectory (positions within
    1e-8 of dx after 16 steps); at TOL 1e-6 the second-order start needs fewer
    Broyden iterations over the steady steps than the reference's, and adding the
    linear tension extrapolation no more than the second-order start alone."""
    out = {}
    for key in STARTS:
        ctx, sim = prepared(key[0], tension=key[1], tol=1e-12)
        its, st = sim.run_steps(1, 16)
        assert st == abi.FS_OK
        out[key] = (its, sim.download())
        ctx.close()
    dx = sediment_params(64).dx
    for key in STARTS[1:]:
        assert np.abs(out[STARTS[0]][1]["X"] - out[key][1]["X"]).max() / dx < 1e-8, key
        assert np.abs(out[STARTS[0]][1]["q"] - out[key][1]["q"]).max() < 1e-8, key
    its = {}
    for key in STARTS:
        ctx, sim = prepared(key[0], tension=key[1])
        i, st = sim.run_steps(1, 40)
        assert st == abi.FS_OK
        its[key] = i
        ctx.close()
    for key in STARTS:
        print("iterations, steps 13-40, start", key, its[key][12:].tolist())
    assert its[(2, 2)][12:].sum() < its[(1, 2)][12:].sum()
    assert its[(2, 1)][12:].sum() <= its[(2, 2)][12:].sum()


def test_linear_tension_extrapolation(gpu_lib):
    """Tension order 1: after lambda_extrap_step, Filament::step sets the next
    tensions to 2 lam - lam1 (lam1, lam2 the last two converged); order 2 keeps the
    reference's 3 lam - 3 lam1 + lam2."""
    ctx, sim = prepared(1, tension=1)
    ex = ctx.params.lambda_extrap_step
    its, st = sim.run_steps(1, ex + 3)
    g = sim.download()
    assert np.array_equal(g["lam"], 2 * g["lam1"] - g["lam2"])
    ctx.set_tension_extrapolation(2)
    prev = g
    sim.step_implicit(ex + 4)
    g = sim.download()
    assert np.array_equal(g["lam2"], prev["lam1"])
    quad = (3 * g["lam1"] - 3 * g["lam2"]) + prev["lam2"]  # the kernel may fuse a multiply-add
    assert np.abs(g["lam"] - quad).max() <= 1e-14 * np.abs(quad).max()
    ctx.close()


@pytest.mark.parametrize("prec,tension", [(abi.FS_PREC_FP64, 2), (abi.FS_PREC_FP32, 2), (abi.FS_PREC_FP32, 1)])
def test_graph_steps_are_host_steps(gpu_lib, prec, tension):
    out = []
    for graph in (0, 1):
        ctx, sim = prepared(2, prec=prec, tension=tension)
        ctx.call("fs_set_graph_mode", graph)
        its, st = sim.run_steps(1, 20)
        assert st == abi.FS_OK
        out.append((its, sim.download()))
        ctx.close()
    assert np.array_equal(out[0][0], out[1][0])
    for k in ("X", "q", "lam", "U"):
        assert np.array_equal(out[0][1][k], out[1][1][k]), k


def test_invalid_order(gpu_lib):
    ctx, sim = prepared(1)
    for bad in (0, 3, -1):
        assert abi.lib().fs_set_start_order(ctx.h, bad) == abi.FS_ERR_INVALID_ARG
        assert abi.lib().fs_set_tension_extrapolation(ctx.h, bad) == abi.FS_ERR_INVALID_ARG
    ctx.close()
