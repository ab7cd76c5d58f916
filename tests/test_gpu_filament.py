"""Filament mechanics, Jacobian, Broyden and the implicit step on the GPU
against the oracle (Filament.hpp, MobilityConstraints.cpp,
FilamentJacobianSolver.hpp, main.cpp:284-754)."""
import numpy as np
import pytest
import torch

from filsim_b200 import abi
from filsim_b200.configs import make_sediment_case, sediment_params
from filsim_b200.fcm import Context, Simulation
from filsim_b200.suspension import random_suspension

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def evolved_pair(oracle, p, s, nsteps):
    """Oracle run for nsteps so the state has non-trivial U, q, lambda; returns
    the oracle system and a suspension holding the same state."""
    sysw = oracle.System(p, s)
    sysw.run_steps(1, nsteps)
    arrays = sysw.download()
    s2 = s.copy()
    s2.set_arrays(arrays)
    return sysw, s2


@pytest.fixture(scope="module")
def small(gpu_lib):
    p, s = make_sediment_case(32, 6, 8, seed=21, kap=np.linspace(0.5, 2.0, 6), c=1.0)
    return p, s


def test_forces_and_jacobian_match(oracle, small):
    p, s = small
    sysw, s2 = evolved_pair(oracle, p, s, 3)
    ctx = Context(p, max_beads=s2.np, max_filaments=s2.nfil)
    sim = Simulation(ctx, s2)
    nt = 4
    sysw.initial_guess()
    sysw.filament_forces(nt)
    sim.initial_guess()
    sim.filament_forces(nt)
    g = sim.download()
    o = sysw.download()
    for k in ("Xs", "Us", "qs", "F", "TAU"):
        assert rel(g[k], o[k]) < 1e-12, k
    Y = sim.device_array("Y", (s2.np, 3)).cpu().numpy()
    assert rel(Y, sysw.array("Y", (s2.np, 3))) < 1e-12
    sysw.build_jacobian(nt)
    sim.build_jacobian(nt)
    for f in range(s2.nfil):
        assert rel(sim.jinv(f), sysw.jinv(f)) < 1e-10


def test_error_check_apply_update_step(oracle, small):
    p, s = small
    sysw, s2 = evolved_pair(oracle, p, s, 2)
    ctx = Context(p, max_beads=s2.np, max_filaments=s2.nfil)
    sim = Simulation(ctx, s2)
    nt = 3
    for w in (sysw, sim):
        w.initial_guess()
        w.filament_forces(nt)
        w.build_jacobian(nt)
    rng = np.random.default_rng(5)
    V = 1e-2 * rng.standard_normal((s2.np, 3))
    W = 1e-2 * rng.standard_normal((s2.np, 3))
    e0, c0 = sysw.error_check(V, W, nt)
    e1, c1 = sim.error_check(V, W, nt)
    assert c0 == c1
    # Err = Xs - 4/3 X + 1/3 Xt - 2/3 dt V cancels positions of size L (17 here)
    # down to ~1e-3: a rounding difference of the GPU's contracted arithmetic
    # (~1e-16 L) shows as ~1e-12 of max |Err|
    assert rel(e1.cpu().numpy(), e0) < 1e-11
    # history columns then the bad-Broyden apply
    n6 = 6 * s2.np
    C = rng.standard_normal((2, n6))
    D = rng.standard_normal((2, n6)) / np.sqrt(n6)
    for i in range(2):
        sysw.set_cols(C[i], D[i], i)
        sim.set_cols(C[i], D[i], i)
    x0 = sysw.jsolve(e0, 2)
    x1 = sim.broyden_apply(e0, 2).cpu().numpy()
    assert rel(x1, x0) < 1e-10
    sysw.update(1e-3 * x0)
    sim.update(1e-3 * x0)
    sysw.step(nt)
    sim.step(nt)
    g = sim.download()
    o = sysw.download()
    for k in ("X", "Xt", "U", "Ut", "q", "qt", "lam", "lam1", "lam2"):
        assert rel(g[k], o[k]) < 1e-12, k


def test_implicit_steps_trajectory(oracle, gpu_lib):
    """100 implicit steps (start-up and steady BDF2 regimes) with a tight
    tolerance: positions agree to 1e-8 of the box, quaternions to 1e-8."""
    p = sediment_params(32, tol=1e-12, broyden_maxiter=100)
    s = random_suspension(p, 6, 8, seed=31, kap=1.0, c=1.0)
    sysw = oracle.System(p, s)
    its0, st0 = sysw.run_steps(1, 100)
    ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
    sim = Simulation(ctx, s)
    its1, st1 = sim.run_steps(1, 100)
    g = sim.download()
    o = sysw.download()
    L = np.array([32 * p.dx] * 3)
    assert np.abs(g["X"] - o["X"]).max() / L[0] < 1e-8
    assert np.abs(g["q"] - o["q"]).max() < 1e-8
    assert np.abs(np.asarray(its1) - np.asarray(its0)).max() <= 1


def test_implicit_steps_iteration_counts(oracle, gpu_lib):
    """At the benchmark tolerance 1e-6 the Broyden iteration counts agree."""
    p = sediment_params(32)
    s = random_suspension(p, 6, 8, seed=32, kap=1.0, c=1.0)
    sysw = oracle.System(p, s)
    its0, _ = sysw.run_steps(1, 6)
    ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
    sim = Simulation(ctx, s)
    its1, _ = sim.run_steps(1, 6)
    assert np.array_equal(its0, its1)
    assert its0.sum() > 0
    d = sim.diag()
    assert d.total_iters == its1.sum()
    assert d.nonfinite == 0
