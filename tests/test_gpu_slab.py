"""The x-slab decomposition of one box's FCM mobility solve on the GPU: each
rank's spread, transforms, projection and interpolation are the library's
(fs_set_slab, fs_fcm_spread, fs_slab_forward_yz, fs_slab_solve_x,
fs_slab_inverse_yz, fs_fcm_interpolate). One rank, and two or four ranks
emulated by host threads on this one GPU (each with its own context; the exchanges
are host-side tensor copies, so no kernel waits for another), give the
library's one-box FP64 solve to 1e-10."""
import threading

import numpy as np
import pytest
import torch

from filsim_b200 import abi
from filsim_b200.abi import make_params
from filsim_b200.fcm import Context, Fcm
from filsim_b200.slab import SlabFcm

pytestmark = pytest.mark.gpu

DX = 1.0 / 1.86


def case(shape, n, seed, ngd=12):
    p = make_params(shape, ngd=ngd, dx=DX)
    rng = np.random.default_rng(seed)
    L = np.array(shape) * p.dx
    Y = np.fmod(rng.uniform(-0.2, 1.2, (n, 3)) * L, L)
    return p, Y, rng.standard_normal((n, 3)), rng.standard_normal((n, 3))


def one_box(p, Y, F, T):
    ctx = Context(p, max_beads=Y.shape[0])
    fcm = Fcm(ctx, Y.shape[0])
    fcm.set(Y, F, T)
    fcm.mobility_solve()
    ctx.synchronize()
    out = fcm.V.cpu().numpy(), fcm.W.cpu().numpy()
    ctx.close()
    return out


class ThreadExchange:
    """Exchanges between ranks that are threads of this process."""

    def __init__(self, world, rank, shared):
        self.world, self.rank, self.s = world, rank, shared

    def _post_and_take(self, key, value, src):
        self.s["box"][(key, self.rank)] = value
        self.s["barrier"].wait()
        got = self.s["box"][(key, src)]
        self.s["barrier"].wait()
        return got

    def shift(self, send, recv, to_next):
        src = (self.rank - 1) % self.world if to_next else (self.rank + 1) % self.world
        recv.copy_(self._post_and_take(("shift", to_next), send.clone(), src))

    def all_to_all(self, out, inp, out_splits, in_splits):
        self.s["box"][("a2a", self.rank)] = list(torch.split(inp.clone(), in_splits))
        self.s["barrier"].wait()
        parts = [self.s["box"][("a2a", r)][self.rank] for r in range(self.world)]
        self.s["barrier"].wait()
        out.copy_(torch.cat(parts))

    def all_reduce(self, t):
        self.s["box"][("sum", self.rank)] = t.clone()
        self.s["barrier"].wait()
        acc = sum(self.s["box"][("sum", r)] for r in range(self.world))
        self.s["barrier"].wait()
        t.copy_(acc)


@pytest.mark.parametrize("shape,ngd,world", [((64, 32, 48), 12, 1), ((64, 32, 48), 12, 2), ((64, 32, 48), 12, 4),
                                             ((64, 32, 32), 20, 1), ((64, 32, 32), 20, 2)])
def test_slab_solve_matches_the_one_box_solve(gpu_lib, shape, ngd, world):
    p, Y, F, T = case(shape, 60, 7, ngd)
    V0, W0 = one_box(p, Y, F, T)
    shared = {"box": {}, "barrier": threading.Barrier(world)}
    results, errors = {}, []

    def run(rank):
        try:
            torch.cuda.set_device(0)
            slab = SlabFcm(p, world, rank, max_beads=Y.shape[0])
            slab.ex = ThreadExchange(world, rank, shared)
            results[rank] = slab.mobility(Y, F, T)
            slab.close()
        except Exception as e:  # reported below, after the other thread is released
            errors.append(e)
            shared["barrier"].abort()

    threads = [threading.Thread(target=run, args=(r,)) for r in range(world)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for r in range(world):
        V, W = results[r]
        assert np.abs(V - V0).max() / np.abs(V0).max() < 1e-10
        assert np.abs(W - W0).max() / np.abs(W0).max() < 1e-10
