"""Cell linked list and collision barrier on the GPU against the oracle
(CollisionBarrierFilament.cpp:24-433). Lists, pair lists, forces and the
minimum distance are compared bit for bit."""
import numpy as np
import pytest
import torch

from filsim_b200.configs import params_for
from filsim_b200.fcm import Context, LinkedList
from filsim_b200.suspension import random_suspension, fcm_positions

pytestmark = pytest.mark.gpu


def dense_case(seed, nfil=40, nw=6, npts=32, jitter=0.35):
    """Filaments packed closer than the barrier range, unwrapped positions."""
    p = params_for(npts)
    s = random_suspension(p, nfil, nw, seed, min_sep=1.2)
    rng = np.random.default_rng(seed)
    X = s.X + jitter * rng.standard_normal(s.X.shape)
    X[::7] += np.array([1.0, -1.0, 0.5]) * (npts * p.dx)  # some beads outside the box
    return p, s, X


def run_gpu(p, s, X, nt, F0):
    ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
    ll = LinkedList(ctx)
    ll.link(X)
    head, lst, mp = ll.lists()
    Y = torch.as_tensor(fcm_positions(p, X), device="cuda")
    F = torch.as_tensor(F0.copy(), device="cuda")
    md = ll.apply_collision_barrier(Y, F, nt, s.fil_id, s.seg_id)
    pairs, n = ll.pairs(Y, nt, s.fil_id, s.seg_id)
    return head, lst, mp, F.cpu().numpy(), md, pairs, n


@pytest.mark.parametrize("seed,nt", [(11, 5), (12, 5), (13, 0)])
def test_barrier_bit_exact(oracle, gpu_lib, seed, nt):
    p, s, X = dense_case(seed)
    if nt == 0:
        p.initial_friction_steps = 1  # nt < initialFrictionSteps: adjacent beads interact too
    F0 = np.random.default_rng(seed).standard_normal((s.np, 3))
    head0, lst0, mp0 = oracle.cells_link(p, X)
    Y = fcm_positions(p, X)
    ref = oracle.collision_barrier(p, Y, F0, s.fil_id, s.seg_id, head0, lst0, mp0, nt, max_pairs=1 << 16)
    assert ref["npairs"] > 20  # the case really exercises the barrier
    head, lst, mp, F, md, pairs, n = run_gpu(p, s, X, nt, F0)
    assert np.array_equal(head, head0)
    assert np.array_equal(lst, lst0)
    assert np.array_equal(mp, mp0)
    assert n == ref["npairs"]
    assert np.array_equal(pairs, ref["pairs"])
    assert np.array_equal(F, ref["F"])
    assert md == ref["min_dist2"]


def test_barrier_no_pairs(oracle, gpu_lib):
    p = params_for(32)
    s = random_suspension(p, 10, 4, 5)
    F0 = np.zeros((s.np, 3))
    head, lst, mp, F, md, pairs, n = run_gpu(p, s, s.X, 3, F0)
    head0, lst0, mp0 = oracle.cells_link(p, s.X)
    ref = oracle.collision_barrier(p, fcm_positions(p, s.X), F0, s.fil_id, s.seg_id, head0, lst0, mp0, 3)
    assert n == 0 and ref["npairs"] == 0
    assert np.array_equal(F, F0)
    assert md == ref["min_dist2"]


def test_link_bit_exact_benchmark_suspension(oracle, gpu_lib):
    p = params_for(64)
    s = random_suspension(p, 32, 15, 1000)
    ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
    ll = LinkedList(ctx)
    ll.link(s.X)
    head, lst, _ = ll.lists()
    head0, lst0, _ = oracle.cells_link(p, s.X)
    assert np.array_equal(head, head0) and np.array_equal(lst, lst0)


def test_full_cell_and_crowded_bead_report_capacity(gpu_lib):
    """The visiting-order key keeps list positions in 12 bits and a bead's events
    in a 64-entry list: a cell of 4096 or more beads makes fs_cells_link return
    FS_ERR_CAPACITY, and a bead with more than 64 interactions makes
    fs_collision_barrier return it."""
    from filsim_b200.abi import FsError, FS_ERR_CAPACITY
    p = params_for(32)
    L = 32 * p.dx
    p.cell_width = 0.99 * L  # one cell for the whole box
    n = 4100
    X = np.random.default_rng(5).uniform(0, L, (n, 3))
    ctx = Context(p, max_beads=n, max_filaments=n)
    with pytest.raises(FsError) as e:
        LinkedList(ctx).link(X)
    assert e.value.status == FS_ERR_CAPACITY
    ctx.close()
    p = params_for(32)
    n = 80
    X = 8.0 + 0.3 * np.random.default_rng(6).standard_normal((n, 3))
    ctx = Context(p, max_beads=n, max_filaments=n)
    ll = LinkedList(ctx)
    ll.link(X)
    Y = torch.as_tensor(X, device="cuda")
    F = torch.zeros_like(Y)
    with pytest.raises(FsError) as e:
        ll.apply_collision_barrier(Y, F, 5, np.arange(n), np.zeros(n))
    assert e.value.status == FS_ERR_CAPACITY
    ctx.close()
