"""fs_collision_barrier_noalloc: the collision barrier for callers that cannot
allocate device memory (a host program with its own fixed memory pool, or a
step loop that must not pay cudaMalloc's synchronisation). Its working memory
is one static device array, so this test checks that two calls in a row each
give exactly the forces and minimum distance of the context-based
fs_cells_link + fs_collision_barrier, i.e. that a call leaves nothing behind
that the next one reads. The file name sorts last so a run that stops at the
first failure has run every other test first."""
import ctypes

import numpy as np
import pytest
import torch

from filsim_b200 import abi
from filsim_b200.configs import params_for
from filsim_b200.fcm import Context, LinkedList
from filsim_b200.suspension import fcm_positions, random_suspension

pytestmark = pytest.mark.gpu


def dense_case(seed, nfil, nw=6, npts=32, jitter=0.35):
    p = params_for(npts)
    s = random_suspension(p, nfil, nw, seed, min_sep=1.2)
    X = s.X + jitter * np.random.default_rng(seed).standard_normal(s.X.shape)
    X[::7] += np.array([1.0, -1.0, 0.5]) * (npts * p.dx)
    return p, s, X


def with_context(p, s, X, F0, nt):
    ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
    ll = LinkedList(ctx)
    ll.link(X)
    Y = torch.as_tensor(fcm_positions(p, X), device="cuda")
    F = torch.as_tensor(F0.copy(), device="cuda")
    md = ll.apply_collision_barrier(Y, F, nt, s.fil_id, s.seg_id)
    out = F.cpu().numpy(), md
    ctx.close()
    return out


def noalloc_call(p, X, Y, F0, fil_id, seg_id, nt, stream=None, want_min=True):
    """One call through the C-ABI; returns (status, F after the call, min_dist2 or None)."""
    Xd = torch.as_tensor(X, device="cuda")
    Yd = torch.as_tensor(Y, device="cuda")
    F = torch.as_tensor(F0.copy(), device="cuda")
    fid = torch.as_tensor(fil_id, dtype=torch.int32, device="cuda")
    sid = torch.as_tensor(seg_id, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    md = ctypes.c_double()
    vp = lambda t: ctypes.c_void_p(t.data_ptr())
    st = abi.lib().fs_collision_barrier_noalloc(ctypes.byref(p), vp(Xd), vp(Yd), vp(F), X.shape[0], nt, vp(fid),
                                                vp(sid), ctypes.c_void_p(stream) if stream else None,
                                                ctypes.byref(md) if want_min else None)
    torch.cuda.synchronize()
    return st, F.cpu().numpy(), (md.value if want_min else None)


def without_allocation(p, s, X, F0, nt):
    st, F, md = noalloc_call(p, X, fcm_positions(p, X), F0, s.fil_id, s.seg_id, nt)
    abi.check(st, "fs_collision_barrier_noalloc")
    return F, md


def test_two_calls_match_the_context_path():
    cases = [dense_case(11, 40), dense_case(12, 25, nw=8)]  # the second call has fewer beads and other cells
    for p, s, X in cases:
        F0 = np.random.default_rng(s.np).standard_normal((s.np, 3))
        F_ref, md_ref = with_context(p, s, X, F0, nt=5)
        F_na, md_na = without_allocation(p, s, X, F0, nt=5)
        assert not np.array_equal(F_ref, F0)  # the barrier acted
        assert np.array_equal(F_na, F_ref)
        assert md_na == md_ref


MAX_BEADS = 65536  # FS_NOALLOC_MAX_BEADS


def test_too_many_beads_is_rejected():
    """A call above the stated limit returns FS_ERR_INVALID_ARG. The buffers are
    full size, so even a call that wrongly went ahead would stay in bounds."""
    p = params_for(32)
    n = MAX_BEADS + 1
    X = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    F = torch.zeros_like(X)
    ids = torch.zeros(n, dtype=torch.int32, device="cuda")
    vp = lambda t: ctypes.c_void_p(t.data_ptr())
    st = abi.lib().fs_collision_barrier_noalloc(ctypes.byref(p), vp(X), vp(X), vp(F), n, 0, vp(ids), vp(ids),
                                                None, None)
    assert st == 1  # FS_ERR_INVALID_ARG


def test_side_stream_and_no_minimum_output():
    """A call on a caller's own stream, without asking for the minimum distance,
    gives the context path's forces."""
    p, s, X = dense_case(13, 30)
    F0 = np.random.default_rng(3).standard_normal((s.np, 3))
    F_ref, _ = with_context(p, s, X, F0, nt=5)
    side = torch.cuda.Stream()
    st, F_na, _ = noalloc_call(p, X, fcm_positions(p, X), F0, s.fil_id, s.seg_id, 5, stream=side.cuda_stream,
                               want_min=False)
    assert st == abi.FS_OK
    assert np.array_equal(F_na, F_ref)


MAX_CELLS = 262144  # FS_NOALLOC_MAX_CELLS


@pytest.mark.parametrize("width", [0.2, 0.0, -1.0, float("nan"), float("inf")])
def test_cell_width_outside_the_limits_is_rejected(width):
    """A cell width that makes more than the stated number of cells, or that is
    not a finite positive number, returns FS_ERR_INVALID_ARG before any launch."""
    p = params_for(32)
    p.cell_width = width
    if width == 0.2:
        assert int(32 * p.dx / width) ** 3 > MAX_CELLS
    n = 8
    X = np.random.default_rng(1).uniform(0, 32 * p.dx, (n, 3))
    F0 = np.zeros((n, 3))
    st, F, _ = noalloc_call(p, X, X, F0, np.arange(n), np.zeros(n), 5)
    assert st == abi.FS_ERR_INVALID_ARG
    assert np.array_equal(F, F0)


def test_full_cell_reports_capacity_and_leaves_forces():
    """One cell holding 4096 beads or more does not fit the visiting-order key:
    FS_ERR_CAPACITY, with F_inout unchanged."""
    p = params_for(32)
    L = 32 * p.dx
    p.cell_width = 0.99 * L  # one cell for the whole box
    n = 4100
    rng = np.random.default_rng(5)
    X = rng.uniform(0, L, (n, 3))
    F0 = rng.standard_normal((n, 3))
    st, F, _ = noalloc_call(p, X, X, F0, np.arange(n), np.zeros(n), 5)
    assert st == abi.FS_ERR_CAPACITY
    assert np.array_equal(F, F0)


def test_crowded_bead_reports_capacity():
    """A bead with more than 64 barrier interactions returns FS_ERR_CAPACITY."""
    p = params_for(32)
    n = 80
    rng = np.random.default_rng(6)
    X = 8.0 + 0.3 * rng.standard_normal((n, 3))  # every pair well inside 2.2a
    st, _, _ = noalloc_call(p, X, X, np.zeros((n, 3)), np.arange(n), np.zeros(n), 5)
    assert st == abi.FS_ERR_CAPACITY
