"""The alternative drivers' pieces on the GPU against the oracle: the barrier
pair filters (CollisionBarrierFilament.cpp:441-945) and the gait-reset step
(main_gaitreset.cpp:302-830)."""
import numpy as np
import pytest

from filsim_b200 import abi
from filsim_b200.configs import sediment_params
from filsim_b200.fcm import Context, Simulation
from filsim_b200.suspension import random_suspension

pytestmark = pytest.mark.gpu


def dense_case(seed):
    p = sediment_params(32, tol=1e-10, broyden_maxiter=100)
    s = random_suspension(p, 10, 8, seed=seed, min_sep=2.0)
    return p, s


@pytest.mark.parametrize("mode", [abi.FS_BARRIER_NOT_SWIMMER, abi.FS_BARRIER_NOT_TEST_PARTICLES,
                                  abi.FS_BARRIER_OFF])
def test_barrier_modes_match_oracle(oracle, gpu_lib, mode):
    p, s = dense_case(101)
    sysw = oracle.System(p, s)
    sysw.set_barrier_mode(mode)
    its0, _ = sysw.run_steps(1, 6)
    ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
    sim = Simulation(ctx, s)
    sim.set_barrier_mode(mode)
    its1, _ = sim.run_steps(1, 6)
    g, o = sim.download(), sysw.download()
    assert np.abs(g["X"] - o["X"]).max() < 1e-8
    assert np.abs(g["q"] - o["q"]).max() < 1e-8
    assert np.abs(np.asarray(its1) - np.asarray(its0)).max() <= 1
    ctx.close()


def test_gait_reset_matches_oracle(oracle, gpu_lib):
    p, s = dense_case(102)
    sysw = oracle.System(p, s)
    sysw.run_steps(1, 13)  # past the start-up regimes
    s13 = s.copy()
    s13.set_arrays(sysw.download())
    ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
    sim = Simulation(ctx, s13)
    for nt in range(14, 18):
        its0, vwf0, st0 = sysw.step_gait_reset(nt)
        its1, vwf1, st1 = sim.step_gait_reset(nt)
        assert st0 == st1 == abi.FS_OK
        assert np.abs(its1 - its0).max() <= 1, nt
        scale = np.abs(vwf0).max(axis=(0, 1))
        assert (np.abs(vwf1 - vwf0).max(axis=(0, 1)) <= 1e-7 * np.maximum(scale, 1e-3)).all(), nt
    g, o = sim.download(), sysw.download()
    assert np.abs(g["X"] - o["X"]).max() < 1e-8
    assert np.abs(g["lam"] - o["lam"]).max() < 1e-6 * max(1.0, np.abs(o["lam"]).max())
    ctx.close()
