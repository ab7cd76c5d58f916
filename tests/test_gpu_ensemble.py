"""Ensembles (fs_batch_*): one graph launch per ensemble step must give every box
exactly the trajectory and iteration counts of stepping it alone."""
import numpy as np
import pytest

from filsim_b200 import abi
from filsim_b200.configs import sediment_params
from filsim_b200.ensemble import Ensemble
from filsim_b200.fcm import Context, Simulation
from filsim_b200.suspension import random_suspension

pytestmark = pytest.mark.gpu


def small_boxes():
    out = []
    for i, (npts, nfil) in enumerate([(32, 3), (48, 6), (64, 10), (48, 4), (64, 12)]):
        p = sediment_params(npts, broyden_maxiter=100)
        s = random_suspension(p, nfil, 8, seed=500 + i, kap=float(0.3 + i))
        out.append((npts, p, s, 0.3 + i))
    return out


@pytest.mark.parametrize("prec,esc", [(abi.FS_PREC_FP32, 0), (abi.FS_PREC_FP64, 0), (abi.FS_PREC_FP32, 2)])
def test_batch_matches_boxes_alone(gpu_lib, prec, esc):
    """esc 2: each box's captured step escalates to FP64 after two iterations
    (fs_set_precision_escalation), inside the ensemble graph as alone."""
    boxes = small_boxes()
    ens = Ensemble(boxes, precision=prec, escalate=esc)
    ens.startup(13)
    its, ms, total, st = ens.run(14, 4)
    outs = [sim.download() for sim in ens.sims]
    ens.close()
    assert st == abi.FS_OK
    assert (ms > 0).all() and total > 0
    for b, (npts, p, s, kb) in enumerate(boxes):
        ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
        ctx.set_precision(prec)
        ctx.set_precision_escalation(esc)
        sim = Simulation(ctx, s)
        ref_its, _ = sim.run_steps(1, 17)
        ref = sim.download()
        ctx.close()
        assert list(its[:, b]) == list(ref_its[13:]), b
        for k in ref:
            assert np.array_equal(outs[b][k], ref[k]), (b, k)
