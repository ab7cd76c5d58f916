"""Graph-captured steps (fs_graph.cu): in the steady regime each step is one CUDA
graph with the Broyden loop on the device; the trajectory and the iteration
counts must be bitwise those of the host-driven step."""
import numpy as np
import pytest

from filsim_b200 import abi
from filsim_b200.configs import make_sediment_case
from filsim_b200.fcm import Context, Simulation

pytestmark = pytest.mark.gpu


def run(npts, nfil, nw, prec, graph, nsteps=20, seed=21):
    p, s = make_sediment_case(npts, nfil, nw, seed)
    ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
    ctx.set_precision(prec)
    abi.check(abi.lib().fs_set_graph_mode(ctx.h, 1 if graph else 0), "fs_set_graph_mode")
    sim = Simulation(ctx, s)
    l0 = abi.lib().fs_kernel_launches()
    its, st = sim.run_steps(1, nsteps)
    launches = abi.lib().fs_kernel_launches() - l0
    d = sim.diag()
    out = sim.download()
    ctx.close()
    return list(its), st, out, d, launches


@pytest.mark.parametrize("npts,nfil,nw,prec", [(64, 16, 8, abi.FS_PREC_FP64), (32, 4, 6, abi.FS_PREC_FP32),
                                               (128, 48, 8, abi.FS_PREC_FP32)])
def test_graph_steps_match_host_steps(gpu_lib, npts, nfil, nw, prec):
    its_h, st_h, out_h, d_h, l_h = run(npts, nfil, nw, prec, graph=False)
    its_g, st_g, out_g, d_g, l_g = run(npts, nfil, nw, prec, graph=True)
    assert st_h == abi.FS_OK and st_g == abi.FS_OK
    assert its_g == its_h
    for k in out_h:
        assert np.array_equal(out_g[k], out_h[k]), k
    assert d_g.total_iters == d_h.total_iters
    assert d_g.mobility_solves == d_h.mobility_solves
    # the counter counts graph-launched kernels too; a graph step adds the loop's
    # head/tail and bookkeeping kernels and the (empty) history dots of iteration 0
    assert l_h <= l_g <= l_h + 8 * (4 + 3 * max(its_g))


def test_graph_single_steps_and_mode_switch(gpu_lib):
    p, s = make_sediment_case(64, 16, 8, 5)
    ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
    sim = Simulation(ctx, s)
    sim.run_steps(1, 13)
    abi.check(abi.lib().fs_set_graph_mode(ctx.h, 1), "fs_set_graph_mode")
    a = [sim.step_implicit(14 + k)[0] for k in range(3)]
    abi.check(abi.lib().fs_set_graph_mode(ctx.h, 0), "fs_set_graph_mode")
    b = [sim.step_implicit(17 + k)[0] for k in range(2)]
    out = sim.download()
    ctx.close()
    ctx2 = Context(p, max_beads=s.np, max_filaments=s.nfil)
    sim2 = Simulation(ctx2, s)
    its, _ = sim2.run_steps(1, 18)
    out2 = sim2.download()
    ctx2.close()
    assert a + b == list(its[13:])
    for k in out:
        assert np.array_equal(out[k], out2[k]), k
