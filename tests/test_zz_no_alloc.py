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


def without_allocation(p, s, X, F0, nt):
    Xd = torch.as_tensor(X, device="cuda")
    Y = torch.as_tensor(fcm_positions(p, X), device="cuda")
    F = torch.as_tensor(F0.copy(), device="cuda")
    fid = torch.as_tensor(s.fil_id, dtype=torch.int32, device="cuda")
    sid = torch.as_tensor(s.seg_id, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    md = ctypes.c_double()
    st = abi.lib().fs_collision_barrier_noalloc(ctypes.byref(p), ctypes.c_void_p(Xd.data_ptr()),
                                                ctypes.c_void_p(Y.data_ptr()), ctypes.c_void_p(F.data_ptr()), s.np,
                                                nt, ctypes.c_void_p(fid.data_ptr()), ctypes.c_void_p(sid.data_ptr()),
                                                None, ctypes.byref(md))
    abi.check(st, "fs_collision_barrier_noalloc")
    return F.cpu().numpy(), md.value


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
