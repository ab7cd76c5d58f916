"""Learned Broyden warm start inside the implicit step (fs_mlp.cu, fs_capi.cu).

- the recorded targets are the update from the extrapolated guess to the
  converged state: starting from guess + target, the step needs at most one
  Broyden iteration;
- a start worse than the plain one is put back per filament: with every
  filament put back the trajectory is bitwise the plain solver's;
- a network trained by the library on plain-solver data predicts part of the
  held-out filament translation correction and the warm-started steps converge.
"""
import ctypes

import numpy as np
import pytest
import torch

from filsim_b200 import abi
from filsim_b200.configs import make_sediment_case
from filsim_b200.fcm import Context, Simulation
from filsim_b200.learn import WarmStartModel, generate, record, set_warm_start

pytestmark = pytest.mark.gpu

NW, NFIL, WARM = 8, 16, 14


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def prepared(seed=11, precision=abi.FS_PREC_FP64):
    p, s = make_sediment_case(64, NFIL, NW, seed)
    ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
    ctx.set_precision(precision)
    model = WarmStartModel(ctx, NW, hidden=128, batch_capacity=128, seed=1)
    sim = Simulation(ctx, s)
    its, st = sim.run_steps(1, WARM)
    assert st == abi.FS_OK
    return ctx, model, sim


def snapshot(sim):
    s = sim.susp.copy()
    sim.download_into(s)
    return s


def test_features_match_definition(gpu_lib):
    ctx, model, sim = prepared()
    s = snapshot(sim)
    sim.upload(s)  # same X, Xt: the two-step history survives
    f = torch.empty((NFIL, model.n_features), dtype=torch.float32, device="cuda")
    ctx.call("fs_learn_features", _ptr(f))
    f = f.cpu().numpy()
    a = s.arrays
    dt = ctx.params.dt
    for fi in (0, NFIL - 1):
        b = slice(fi * NW, (fi + 1) * NW)
        X, Xt, q, U, Ut = a["X"][b], a["Xt"][b], a["q"][b], a["U"][b], a["Ut"][b]
        per_bead = f[fi, :19 * NW].reshape(NW, 19)
        np.testing.assert_allclose(per_bead[:, 0:3], X - X.mean(0), rtol=1e-5, atol=1e-5)
        np.testing.assert_allclose(per_bead[:, 3:7], q, rtol=1e-6, atol=1e-7)
        np.testing.assert_allclose(per_bead[:, 7:10], (X - Xt) / dt, rtol=1e-5, atol=1e-9)
        np.testing.assert_allclose(per_bead[:, 10:13], U / dt, rtol=1e-5, atol=1e-12)
        np.testing.assert_allclose(per_bead[:, 13:16], Ut / dt, rtol=1e-5, atol=1e-12)
        assert np.abs(per_bead[:, 16:19]).max() > 0  # acceleration from the kept history
        lk = slice(fi * (NW - 1), (fi + 1) * (NW - 1))
        per_link = f[fi, 19 * NW:19 * NW + 9 * (NW - 1)].reshape(NW - 1, 9)
        np.testing.assert_allclose(per_link[:, 0:3], a["lam"][lk], rtol=1e-5, atol=1e-9)
        np.testing.assert_allclose(per_link[:, 3:6], a["lam1"][lk], rtol=1e-5, atol=1e-9)
        np.testing.assert_allclose(per_link[:, 6:9], a["lam2"][lk], rtol=1e-5, atol=1e-9)
        assert f[fi, -1] == pytest.approx(np.log(a["kap"][fi]), abs=1e-6)
    ctx.close()


def test_targets_are_guess_to_converged_update(gpu_lib):
    ctx, model, sim = prepared()
    s0 = snapshot(sim)
    f, t, its = record(sim, model, WARM + 1, 1)
    assert its[0] > 1
    conv = sim.download()
    sim.upload(s0)
    pred = torch.zeros((NFIL, model.n_targets), dtype=torch.float32, device="cuda")
    pred[:, :6 * NW] = t[:, :6 * NW]
    set_warm_start(ctx, 1)
    ctx.call("fs_learn_override", _ptr(pred))
    it, st = sim.step_implicit(WARM + 1)
    d = sim.diag()
    assert st == abi.FS_OK and it <= 1
    assert d.learned_filaments == NFIL and d.fallback_filaments == 0
    out = sim.download()
    assert np.abs(out["X"] - conv["X"]).max() < 1e-8
    ctx.close()


def test_all_fallback_reproduces_plain_trajectory(gpu_lib):
    ctx, model, sim = prepared()
    s0 = snapshot(sim)
    its_plain, st = sim.run_steps(WARM + 1, 3)
    plain = sim.download()
    sim.upload(s0)
    set_warm_start(ctx, 1)
    bad = torch.full((NFIL, model.n_targets), 1e-2, dtype=torch.float32, device="cuda")
    its = []
    for k in range(3):
        ctx.call("fs_learn_override", _ptr(bad))
        it, st = sim.step_implicit(WARM + 1 + k)
        its.append(it)
        d = sim.diag()
        assert d.fallback_filaments == NFIL and d.learned_filaments == 0
    out = sim.download()
    assert list(its) == list(its_plain)
    for k in plain:
        assert np.array_equal(out[k], plain[k]), k
    ctx.close()


def test_partial_fallback(gpu_lib):
    ctx, model, sim = prepared()
    s0 = snapshot(sim)
    f, t, its = record(sim, model, WARM + 1, 1)
    sim.upload(s0)
    # exact starts except one filament given the correction with the wrong sign
    # (twice the plain start's error): that filament goes back (the flow couples
    # filaments, so close neighbours may go back too)
    pred = torch.zeros((NFIL, model.n_targets), dtype=torch.float32, device="cuda")
    pred[:, :6 * NW] = t[:, :6 * NW]
    pred[1, :6 * NW] = -t[1, :6 * NW]
    set_warm_start(ctx, 1)
    ctx.call("fs_learn_override", _ptr(pred))
    it, st = sim.step_implicit(WARM + 1)
    d = sim.diag()
    assert st == abi.FS_OK
    assert d.fallback_filaments >= 1 and d.learned_filaments >= NFIL // 2
    assert d.learned_filaments + d.fallback_filaments == NFIL
    ctx.close()


def test_trained_network_gain(gpu_lib):
    """Trained on 12 seeded plain-solver runs (K_B log-uniform in [0.1, 10]), evaluated on
    a held-out seed: the prediction removes part of the filament translation
    correction X0 and the warm-started steps converge to the same tolerance."""
    def make_case(seed, kb):
        return make_sediment_case(128, 64, NW, seed=seed, kap=kb)

    p, s = make_case(300, 1.0)
    ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
    model = WarmStartModel(ctx, NW, hidden=256, batch_capacity=1024, seed=0)
    feats, tgts, _ = generate(make_case, list(range(200, 212)), 13, 6, model=model)
    model.fit_normalization(feats, tgts)
    model.fit(feats, tgts, epochs=40, batch=512, lr=1e-3, lr_final=5e-5)
    ctx.set_precision(abi.FS_PREC_FP32)
    sim = Simulation(ctx, make_case(999, 1.0)[1])
    set_warm_start(ctx, 0)
    sim.run_steps(1, 13)
    s0 = snapshot(sim)
    fh, th, its_plain = record(sim, model, 14, 4)
    ph = model.forward(fh)
    x0_err = (ph[:, :3] - th[:, :3]).pow(2).mean().sqrt().item()
    x0_rms = th[:, :3].pow(2).mean().sqrt().item()
    assert x0_err < 0.9 * x0_rms
    # the same six steps from the same state: plain start, then the learned start
    # with its fallback checked against a carried plain residual (refreshed every 8
    # learned steps), so that it costs one solve on all steps but the first
    nsteps = 6
    sim.upload(s0)
    set_warm_start(ctx, 0)
    its_plain, st = sim.run_steps(14, nsteps)
    solves_plain = sim.diag().mobility_solves
    assert st == abi.FS_OK
    sim.upload(s0)
    set_warm_start(ctx, 1)
    abi.check(abi.lib().fs_warm_start_bound(ctx.h, 8), "fs_warm_start_bound")
    its, st = sim.run_steps(14, nsteps)
    d = sim.diag()
    assert st == abi.FS_OK
    assert d.learned_filaments > d.fallback_filaments
    print("held-out X0 correction rms %.3e, residual after prediction %.3e; iterations plain %s learned %s; "
          "mobility solves plain %d learned %d" % (x0_rms, x0_err, list(its_plain), list(its), solves_plain,
                                                   d.mobility_solves))
    assert sum(its) < sum(its_plain)
    assert d.mobility_solves < solves_plain
    ctx.close()


def test_cost_gate(gpu_lib):
    """fs_warm_start_gate: each step takes the start with the lower running mean of
    mobility solves per step and probes the other one (first after period steps, then
    at doubling intervals while the choice holds); the learned start must save the
    margin (fs_warm_start_gate_margin); with the gate off the learned start runs on
    every step."""
    ctx, model, sim = prepared()
    s0 = snapshot(sim)
    set_warm_start(ctx, 1)

    def stats():
        steps = np.zeros(2, np.int64)
        solves = np.zeros(2, np.float64)
        ctx.call("fs_warm_start_gate_stats", ctypes.c_void_p(steps.ctypes.data),
                 ctypes.c_void_p(solves.ctypes.data))
        return steps, solves

    margin = 1.0
    ctx.call("fs_warm_start_gate_margin", ctypes.c_double(margin))
    ctx.call("fs_warm_start_gate", 3)
    its, st = sim.run_steps(WARM + 1, 12)
    assert st == abi.FS_OK
    steps, solves = stats()
    assert steps.sum() == 12
    assert steps.min() >= 2                       # both starts measured and re-probed
    major = int(np.argmax(steps))
    # the learned start runs most only when it saves the margin
    if major == 1:
        assert solves[1] + margin <= solves[0] + 1e-9
    assert abi.lib().fs_warm_start_gate_margin(ctx.h, ctypes.c_double(-1.0)) == abi.FS_ERR_INVALID_ARG
    assert abi.lib().fs_warm_start_gate_margin(ctx.h, ctypes.c_double(float("nan"))) == abi.FS_ERR_INVALID_ARG
    # gate off: the learned start on every step
    sim.upload(s0)
    ctx.call("fs_warm_start_gate", 0)
    its, st = sim.run_steps(WARM + 1, 4)
    d = sim.diag()  # counts of this call
    assert st == abi.FS_OK
    assert d.learned_filaments + d.fallback_filaments == 4 * NFIL
    ctx.close()


@pytest.mark.parametrize("start_order", [1, 2])
def test_gated_plain_steps_run_as_graphs_bitwise(gpu_lib, start_order):
    """Under the cost gate, the steps given the plain start run as captured step
    graphs when graph mode is on: the trajectory, the iteration counts and the
    gate's choices are bitwise those of the host-driven run, with the reference's
    start and with the second-order start (whose history the graph keeps)."""
    out = []
    for graph in (0, 1):
        ctx, model, sim = prepared()
        ctx.set_start_order(start_order)
        set_warm_start(ctx, 1)
        ctx.call("fs_warm_start_gate", 3)
        ctx.call("fs_set_graph_mode", graph)
        its, st = sim.run_steps(WARM + 1, 12)
        assert st == abi.FS_OK
        steps = np.zeros(2, np.int64)
        solves = np.zeros(2, np.float64)
        ctx.call("fs_warm_start_gate_stats", ctypes.c_void_p(steps.ctypes.data),
                 ctypes.c_void_p(solves.ctypes.data))
        out.append((its, snapshot(sim), steps, solves))
        ctx.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][2], out[1][2]) and np.array_equal(out[0][3], out[1][3])
    for k in ("X", "q", "lam", "U"):
        assert np.array_equal(out[0][1].arrays[k], out[1][1].arrays[k]), k
    assert out[1][2][0] >= 1  # some steps took the plain start (as graphs)
