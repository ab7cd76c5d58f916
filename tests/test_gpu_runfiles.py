"""A GPU run resumed from the reference's checkpoint files (.par + .bak,
continue_from_checkpoint, file_functions.cpp:226-318) follows the
uninterrupted run."""
import numpy as np
import pytest

from filsim_b200 import runfiles
from filsim_b200.configs import sediment_params
from filsim_b200.fcm import Context, Simulation
from filsim_b200.suspension import random_suspension

pytestmark = pytest.mark.gpu


def test_resume_from_checkpoint(gpu_lib, tmp_path):
    p = sediment_params(32, tol=1e-12, broyden_maxiter=100)
    s = random_suspension(p, 6, 8, seed=82, kap=np.linspace(0.5, 2.0, 6), c=1.0)
    ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
    sim = Simulation(ctx, s)
    sim.run_steps(1, 10)
    s10 = s.copy()
    sim.download_into(s10)
    runfiles.write_parameters(tmp_path / "run.par", s10, runfiles.run_info(p=p))
    runfiles.save_backup(tmp_path / "run.bak", s10, 10)
    runfiles.save_data_column_names(tmp_path / "run.dat", s10)
    runfiles.save_data(tmp_path / "run.dat", s10, 10)
    sim.run_steps(11, 5)
    full = sim.download()
    ctx.close()

    r, nt_next = runfiles.continue_from_checkpoint(tmp_path / "run", kap=s.kap, c=s.c)
    assert nt_next == 11
    ctx2 = Context(p, max_beads=r.np, max_filaments=r.nfil)
    sim2 = Simulation(ctx2, r)
    its, st = sim2.run_steps(nt_next, 5)
    got = sim2.download()
    ctx2.close()
    assert np.abs(got["X"] - full["X"]).max() < 1e-9
    assert np.abs(got["q"] - full["q"]).max() < 1e-9
    # the .dat row holds the checkpointed positions
    row = (tmp_path / "run.dat").read_text().split("\n")[1].split(" ")
    vals = np.array([float(x) for x in row[1:-1]]).reshape(s.np, 7)
    assert np.abs(vals[:, :3] - s10.Xs).max() < 1e-13


def test_checkpoint_fields_are_the_whole_state(gpu_lib):
    """Stepping from uploads of only the checkpointed fields (X, Xt, q, qt, U, Ut,
    lam, lam1, lam2; Xs, Us, qs, F, TAU left NULL) gives the trajectory of full
    uploads bitwise: every step recomputes the rest."""
    p = sediment_params(32)
    s = random_suspension(p, 6, 8, seed=83)
    keep = ("X", "Xt", "q", "qt", "U", "Ut", "lam", "lam1", "lam2", "kap", "c")
    out = []
    for fields in (None, keep):
        ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
        sim = Simulation(ctx, s)
        sim.run_steps(1, 14)
        host = s.copy()
        sim.download_into(host)
        if fields:
            host.arrays = {k: v for k, v in host.arrays.items() if k in fields}
        for nt in range(15, 19):
            sim.upload(host)
            sim.step_implicit(nt)
            sim.download_into(host)
        out.append(host.arrays)
        ctx.close()
    for k in ("X", "Xt", "q", "qt", "U", "Ut", "lam", "lam1", "lam2"):
        assert np.array_equal(out[0][k], out[1][k]), k
