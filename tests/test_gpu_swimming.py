"""Swimming drive (time-dependent strain twist of applyElasticTorques,
Filament.hpp:297-326) and spring links (spring_link_functions.cpp:24-45) on
the GPU against the oracle."""
import ctypes

import numpy as np
import pytest

from filsim_b200 import abi
from filsim_b200.configs import make_sediment_case, sediment_params
from filsim_b200.fcm import Context, Simulation
from filsim_b200.suspension import random_suspension, swim_parameters

pytestmark = pytest.mark.gpu

LINKS = np.array([[0, 9], [9, 20], [3, 23], [40, 1]])
SPRING_K, SPRING_L0 = 0.2, 3.0


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def drive(p, s, sperm_decay=False):
    swim = swim_parameters(s.fil_start, p, K0=1.0, Sp4=12.0,
                           alpha=np.linspace(0.0, 1.2, s.nfil), beta=np.linspace(1.0, 0.2, s.nfil),
                           phase=np.linspace(-1.0, 2.0, s.nfil), kap=s.kap)
    return swim, 8.25, sperm_decay


def setup_both(oracle, p, s, swim=True, springs=True, sperm_decay=False):
    sysw = oracle.System(p, s)
    ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
    sim = Simulation(ctx, s)
    if swim:
        sw, curv, sd = drive(p, s, sperm_decay)
        sysw.set_swimming(sw, curv, sd)
        sim.set_swimming(sw, curv, sd)
    if springs:
        sysw.set_spring_links(LINKS, SPRING_K, SPRING_L0)
        sim.set_spring_links(LINKS, SPRING_K, SPRING_L0)
    return sysw, ctx, sim


@pytest.mark.parametrize("sperm_decay", [False, True])
def test_forces_and_jacobian_with_drive_and_springs(oracle, gpu_lib, sperm_decay):
    p, s = make_sediment_case(32, 6, 8, seed=71, kap=np.linspace(0.5, 2.0, 6), c=1.0)
    sysw0 = oracle.System(p, s)
    sysw0.run_steps(1, 3)  # non-trivial U, q, lambda
    s2 = s.copy()
    s2.set_arrays(sysw0.download())
    sysw, ctx, sim = setup_both(oracle, p, s2, sperm_decay=sperm_decay)
    nt = 4
    for w in (sysw, sim):
        w.initial_guess()
        w.filament_forces(nt)
    g, o = sim.download(), sysw.download()
    for k in ("Xs", "F", "TAU"):
        assert rel(g[k], o[k]) < 1e-12, k
    sysw.build_jacobian(nt)
    sim.build_jacobian(nt)
    for f in range(s2.nfil):
        assert rel(sim.jinv(f), sysw.jinv(f)) < 1e-10
    ctx.close()


def test_drive_off_is_the_plain_path_bitwise(oracle, gpu_lib):
    """A drive with Alpha = Beta = 0, or no drive, gives the plain forces bitwise."""
    p, s = make_sediment_case(32, 4, 8, seed=72)
    ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
    sim = Simulation(ctx, s)
    sim.initial_guess()
    sim.filament_forces(5)
    ref = sim.download()
    sw = swim_parameters(s.fil_start, p, K0=1.0, Sp4=12.0, alpha=0.0, beta=0.0, phase=0.3)
    sim.set_swimming(sw, 8.25, False)
    sim.filament_forces(5)
    got = sim.download()
    for k in ("F", "TAU"):
        assert np.array_equal(got[k], ref[k]), k
    sim.set_swimming(None)
    sim.filament_forces(5)
    for k in ("F", "TAU"):
        assert np.array_equal(sim.download()[k], ref[k]), k
    ctx.close()


def test_swimming_trajectory(oracle, gpu_lib):
    """40 implicit steps with a swimming drive and spring links (start-up and
    BDF2 regimes, tight tolerance): positions and quaternions agree with the
    oracle and the iteration counts match; graph mode falls back to host-driven
    steps for a drive whose forces depend on nt."""
    p = sediment_params(32, tol=1e-12, broyden_maxiter=100)
    s = random_suspension(p, 6, 8, seed=73, kap=1.0, c=1.0)
    sysw, ctx, sim = setup_both(oracle, p, s)
    ctx.call("fs_set_graph_mode", 1)
    its0, st0 = sysw.run_steps(1, 40)
    its1, st1 = sim.run_steps(1, 40)
    assert st0 == st1 == abi.FS_OK
    g, o = sim.download(), sysw.download()
    L = 32 * p.dx
    assert np.abs(g["X"] - o["X"]).max() / L < 1e-8
    assert np.abs(g["q"] - o["q"]).max() < 1e-8
    assert np.abs(np.asarray(its1) - np.asarray(its0)).max() <= 1
    # the drive moved the filaments differently from the undriven run
    ref = oracle.System(p, s)
    ref.run_steps(1, 40)
    assert np.abs(ref.download()["q"] - o["q"]).max() > 1e-6
    ctx.close()


def test_spring_links_in_captured_steps(gpu_lib):
    """Spring links take part in graph-captured steps: the same steady steps run
    as graphs and host-driven are bitwise equal."""
    p, s = make_sediment_case(32, 6, 8, seed=74)
    out = []
    for graph in (0, 1):
        ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
        sim = Simulation(ctx, s)
        sim.set_spring_links(LINKS, SPRING_K, SPRING_L0)
        ctx.call("fs_set_graph_mode", graph)
        its, st = sim.run_steps(1, 20)
        out.append((its, sim.download()))
        ctx.close()
    assert np.array_equal(out[0][0], out[1][0])
    for k in ("X", "q", "lam"):
        assert np.array_equal(out[0][1][k], out[1][1][k]), k


def test_invalid_arguments(gpu_lib):
    p, s = make_sediment_case(32, 2, 8, seed=75)
    ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
    sim = Simulation(ctx, s)
    L = abi.lib()
    for bad in ([[0, 0]], [[0, s.np]], [[-1, 3]]):
        arr = np.ascontiguousarray(bad, dtype=np.int32)
        st = L.fs_set_spring_links(ctx.h, 1, arr.ctypes.data_as(ctypes.c_void_p), 1.0, 1.0)
        assert st == abi.FS_ERR_INVALID_ARG
    sw = np.full((s.nfil, 5), np.nan)
    assert L.fs_set_swimming(ctx.h, sw.ctypes.data_as(ctypes.c_void_p), 1.0, 0) == abi.FS_ERR_INVALID_ARG
    ctx.close()
