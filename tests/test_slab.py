"""The x-slab decomposition of one box's FCM mobility solve (filsim_b200/slab.py)
on CPU ranks over gloo: the partition into slabs, the halo reduction of the
spread, the transposes between ranks (uneven kz ranges) and the halo gather of
the interpolation, with each rank's own arithmetic done by numpy in the
reference's formulas (FCMfunctions.cpp:549-808). Two and four ranks give the
oracle's one-box velocities to 1e-10 (the decomposition the reference makes
with FFTW-MPI, FCMfunctions.cpp:16-23, 360-406, 460-461)."""
import os
import tempfile

import numpy as np
import pytest
import torch

from filsim_b200.abi import make_params
from filsim_b200.slab import SlabFcm, SlabLayout

DX = 1.0 / 1.86


def case(shape, n, seed):
    p = make_params(shape, ngd=12, dx=DX)
    rng = np.random.default_rng(seed)
    L = np.array(shape) * p.dx
    Y = rng.uniform(-0.2, 1.2, (n, 3)) * L
    Y = np.fmod(Y, L)  # Fcm::assign_filament_data's rule: may stay negative
    F = rng.standard_normal((n, 3))
    T = rng.standard_normal((n, 3))
    return p, Y, F, T


class NumpyPieces:
    """A rank's arithmetic in numpy: the oracle's whole-box spread cut to the
    window, numpy transforms with the reference's conventions, and the
    interpolation of gaussian_setup / particle_velocities / particle_rotations."""

    def __init__(self, p, layout, oracle):
        self.p, self.L, self.oracle = p, layout, oracle
        s = p.sigma ** 2
        self.anorm, self.anorm2 = 1 / np.sqrt(2 * np.pi * s), 2 * s
        sd = p.sigma_dip ** 2
        self.anormdip, self.anormdip2, self.sdsq = 1 / np.sqrt(2 * np.pi * sd), 2 * sd, sd

    def spread(self, Y, F, T):
        L = self.L
        _, _, f, _ = self.oracle.fcm_mobility(self.p, Y, F, T, return_grids=True)
        planes = (L.x0 + np.arange(L.nxs + L.H)) % L.nx
        return torch.from_numpy(np.ascontiguousarray(f[:, planes]))

    def forward_yz(self, f):
        s = np.fft.fft(np.fft.rfft(f.numpy(), axis=3), axis=2).transpose(0, 1, 3, 2)
        return torch.from_numpy(np.ascontiguousarray(np.stack([s.real, s.imag], -1)))

    def _q(self, n, idx):
        i = np.asarray(idx)
        return np.where(i <= n // 2, i, i - n) * (2 * np.pi / (n * self.p.dx))

    def solve_x(self, spec_t):
        L = self.L
        s = np.fft.fft(spec_t[..., 0].numpy() + 1j * spec_t[..., 1].numpy(), axis=3)
        q1 = self._q(L.nx, np.arange(L.nx))[None, None, :]
        q2 = self._q(L.ny, np.arange(L.ny))[None, :, None]
        q3 = ((L.kz0 + np.arange(L.nkz)) * (2 * np.pi / (L.nz * self.p.dx)))[:, None, None]
        norm = 1.0 / ((q2 * q2 + q1 * q1 + 1e-18) + q3 * q3)
        kdotf = (q1 * s[0] + q2 * s[1] + q3 * s[2]) * norm
        total = float(L.nx * L.ny * L.nz)
        u = np.stack([norm * (s[0] - q1 * kdotf), norm * (s[1] - q2 * kdotf), norm * (s[2] - q3 * kdotf)]) / total
        if L.kz0 == 0:
            u[:, 0, 0, 0] = 0
        u = np.fft.ifft(u, axis=3) * L.nx
        spec_t[..., 0] = torch.from_numpy(u.real)
        spec_t[..., 1] = torch.from_numpy(u.imag)

    def inverse_yz(self, spec):
        L = self.L
        s = np.fft.ifft(spec[..., 0].numpy() + 1j * spec[..., 1].numpy(), axis=3) * L.ny
        s[:, :, 0, :] = s[:, :, 0, :].real  # the halfcomplex inverse has no slot for these
        s[:, :, -1, :] = s[:, :, -1, :].real
        u = np.fft.irfft(s.transpose(0, 1, 3, 2), n=L.nz, axis=3) * L.nz
        return torch.from_numpy(np.ascontiguousarray(u))

    def interpolate(self, uw, Y):
        L, p = self.L, self.p
        u = uw.numpy()
        V = np.zeros((Y.shape[0], 3))
        W = np.zeros((Y.shape[0], 3))
        ngdh = p.ngd // 2
        for b in range(Y.shape[0]):
            g, gd, r, ind = [], [], [], []
            for a, n in enumerate((L.nx, L.ny, L.nz)):
                xc = int(Y[b, a] / p.dx)
                xg = xc - ngdh + np.arange(1, p.ngd + 1)
                xx = xg * p.dx - Y[b, a]
                g.append(self.anorm * np.exp(-xx * xx / self.anorm2))
                gd.append(self.anormdip * np.exp(-xx * xx / self.anormdip2))
                r.append(-xx / self.sdsq)
                i = np.mod(xg, n)
                ind.append(np.mod(i - L.x0, L.nx) if a == 0 else i)
            ux = u[:, ind[0]][:, :, ind[1]][:, :, :, ind[2]]
            gg = np.einsum("i,j,k->ijk", g[0], g[1], g[2])
            dd = np.einsum("i,j,k->ijk", gd[0], gd[1], gd[2])
            rx, ry, rz = r[0][:, None, None], r[1][None, :, None], r[2][None, None, :]
            V[b] = (ux * gg).sum(axis=(1, 2, 3)) * p.dx ** 3
            w0 = ((ux[2] * ry - ux[1] * rz) * dd).sum()
            w1 = ((ux[0] * rz - ux[2] * rx) * dd).sum()
            w2 = ((ux[1] * rx - ux[0] * ry) * dd).sum()
            W[b] = -0.5 * np.array([w0, w1, w2]) * p.dx ** 3
        return torch.from_numpy(V), torch.from_numpy(W)


def _rank(rank, world, port, out, shape, n, seed):
    import torch.distributed as dist
    from oracle import oracle_py
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        p, Y, F, T = case(shape, n, seed)
        layout = SlabLayout(p, world, rank)
        slab = SlabFcm(p, world, rank, pieces=NumpyPieces(p, layout, oracle_py))
        V, W = slab.mobility(Y, F, T)
        np.savez(os.path.join(out, "r%d.npz" % rank), V=V, W=W)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,shape,port", [(2, (64, 32, 48), 29611), (4, (128, 32, 32), 29612)])
def test_slabs_over_gloo_ranks_give_the_one_box_solve(oracle, world, shape, port):
    n, seed = 60, 5
    with tempfile.TemporaryDirectory() as out:
        torch.multiprocessing.spawn(_rank, args=(world, port, out, shape, n, seed), nprocs=world, join=True)
        res = [np.load(os.path.join(out, "r%d.npz" % r)) for r in range(world)]
    p, Y, F, T = case(shape, n, seed)
    V0, W0 = oracle.fcm_mobility(p, Y, F, T)
    for r in res:  # every rank holds all velocities
        assert np.abs(r["V"] - V0).max() / np.abs(V0).max() < 1e-10
        assert np.abs(r["W"] - W0).max() / np.abs(W0).max() < 1e-10
    owners = SlabLayout(p, world, 0).owners(Y)
    assert len(set(owners.tolist())) == world  # every rank owned beads


def test_layout_rules():
    p = make_params((64, 32, 32), ngd=12, dx=DX)
    L = SlabLayout(p, 2, 1)
    assert (L.nxs, L.H, L.x0) == (32, 16, 32)
    assert L.kz_bounds == [0, 8, 17]
    with pytest.raises(ValueError):
        SlabLayout(p, 3, 0)  # 64 planes do not split over 3 ranks
    with pytest.raises(ValueError):
        SlabLayout(make_params((64, 32, 32), ngd=20, dx=DX), 4, 0)  # 16-plane slabs cannot hold 32 halo planes
