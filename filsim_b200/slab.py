"""One box's FCM mobility solve split over ranks by x slabs.

The reference runs one box on many MPI ranks: FFTW-MPI splits the grid into x
slabs and transposes it between the passes of its 3-D transform
(FCMfunctions.cpp:16-23, 360-406), and V, W are reduced over ranks (:460-461).
Here every rank holds one GPU and the planes [x0, x0 + nxs) of the box:

1. spread: the rank spreads the beads whose Gaussian stencil starts in its
   planes into a window of nxs + H planes (H >= ngd - 1), its own context in
   slab mode (fs_set_slab); the H planes past its slab go to the next rank,
   which adds them to its first planes (a halo reduction);
2. z and y transforms of the slab (fs_slab_forward_yz);
3. a transpose between ranks (all-to-all): each rank receives, for its range of
   kz, the spectrum of every x;
4. x transforms, the Stokes projection and the inverse x transforms
   (fs_slab_solve_x), and the transpose back;
5. inverse y and z transforms (fs_slab_inverse_yz);
6. interpolation: the rank appends the next rank's first H planes to its slab
   (a halo gather) and interpolates its own beads (fs_fcm_interpolate);
7. each bead has one owner, so a sum over ranks assembles V and W.

The exchanges go through torch.distributed (NCCL between GPUs: point-to-point
sends for the halos, all_to_all_single for the transposes; gloo on CPU for
the tests). The arithmetic of every piece is the library's FP64 path (the
parity path); `LocalPieces` is the interface the orchestration uses, which
the CPU tests implement with numpy to check the decomposition by itself.
"""
import ctypes
import math

import numpy as np
import torch

from .abi import FsParams, check, lib
from .fcm import Context


class SlabLayout:
    """The index arithmetic: slabs, halo, kz ranges, bead owners."""

    def __init__(self, params, world, rank):
        self.nx, self.ny, self.nz = params.npts_x, params.npts_y, params.npts_z
        self.ngd = params.ngd
        self.dx = params.dx
        self.world, self.rank = world, rank
        if self.nx % world:
            raise ValueError("the box's %d x planes do not split over %d ranks" % (self.nx, world))
        self.nxs = self.nx // world
        # halo planes: whole 16-point tiles holding the ngd - 1 planes a stencil reaches past its start
        self.H = 16 * math.ceil((self.ngd - 1) / 16)
        if self.nxs % 16 or self.H > self.nxs:
            raise ValueError("a slab must be whole 16-plane tiles and at least the %d halo planes" % self.H)
        self.x0 = rank * self.nxs
        self.nzh = self.nz // 2 + 1
        self.kz_bounds = [(r * self.nzh) // world for r in range(world + 1)]
        self.kz0 = self.kz_bounds[rank]
        self.nkz = self.kz_bounds[rank + 1] - self.kz0

    def nkz_of(self, r):
        return self.kz_bounds[r + 1] - self.kz_bounds[r]

    def owners(self, Y):
        """Rank owning each bead: the slab holding the x start of its stencil,
        with gaussian_setup's rules (FCMfunctions.cpp:565-571): xc = (int)(Y/dx),
        start = xc - ngd/2 + 1 wrapped into the box."""
        xc = np.trunc(np.asarray(Y)[:, 0] / self.dx).astype(np.int64)
        start = np.mod(xc - self.ngd // 2 + 1, self.nx)
        return start // self.nxs


class Exchange:
    """The exchanges between ranks, over a torch.distributed group (None with
    one rank: every exchange is a local copy)."""

    def __init__(self, world, rank, group=None):
        self.world, self.rank, self.group = world, rank, group

    def _dist(self):
        import torch.distributed as dist
        return dist

    def shift(self, send, recv, to_next):
        """send -> rank + 1 (to_next) or rank - 1, recv <- the other neighbour."""
        if self.world == 1:
            recv.copy_(send)
            return
        dist = self._dist()
        dst = (self.rank + (1 if to_next else -1)) % self.world
        src = (self.rank - (1 if to_next else -1)) % self.world
        ops = [dist.P2POp(dist.isend, send, dst, self.group), dist.P2POp(dist.irecv, recv, src, self.group)]
        for r in dist.batch_isend_irecv(ops):
            r.wait()

    def all_to_all(self, out, inp, out_splits, in_splits):
        if self.world == 1:
            out.copy_(inp)
            return
        self._dist().all_to_all_single(out, inp, out_splits, in_splits, group=self.group)

    def all_reduce(self, t):
        if self.world > 1:
            self._dist().all_reduce(t, group=self.group)


class LocalPieces:
    """The per-rank arithmetic (this class: the library on the rank's GPU, FP64).
    Arrays are torch tensors on the rank's device; complex values are trailing
    (re, im) pairs."""

    def __init__(self, params, layout, max_beads):
        self.layout = layout
        w = FsParams()
        ctypes.memmove(ctypes.byref(w), ctypes.byref(params), ctypes.sizeof(FsParams))
        w.npts_x = layout.nxs + layout.H
        self.ctx = Context(w, max_beads=max(1, max_beads))
        check(lib().fs_set_slab(self.ctx.h, layout.x0, layout.nx), "fs_set_slab")
        self.device = torch.device("cuda", torch.cuda.current_device())

    def _p(self, t):
        return ctypes.c_void_p(t.data_ptr()) if t is not None and t.numel() else None

    def spread(self, Y, F, T):
        L = self.layout
        f = torch.empty((3, L.nxs + L.H, L.ny, L.nz), dtype=torch.float64, device=self.device)
        Yd, Fd, Td = (torch.as_tensor(np.ascontiguousarray(a), device=self.device) for a in (Y, F, T))
        self.ctx.call("fs_fcm_spread", self._p(Yd), self._p(Fd), self._p(Td), int(Yd.shape[0]), self._p(f))
        return f

    def forward_yz(self, f):
        L = self.layout
        spec = torch.empty((3, L.nxs, L.nzh, L.ny, 2), dtype=torch.float64, device=self.device)
        self.ctx.call("fs_slab_forward_yz", self._p(f), L.nxs, self._p(spec))
        return spec

    def solve_x(self, spec_t):
        L = self.layout
        self.ctx.call("fs_slab_solve_x", self._p(spec_t), L.kz0, L.nkz)

    def inverse_yz(self, spec):
        L = self.layout
        u = torch.empty((3, L.nxs, L.ny, L.nz), dtype=torch.float64, device=self.device)
        self.ctx.call("fs_slab_inverse_yz", self._p(spec), L.nxs, self._p(u))
        return u

    def interpolate(self, u_window, Y):
        n = Y.shape[0]
        V = torch.zeros((n, 3), dtype=torch.float64, device=self.device)
        W = torch.zeros_like(V)
        Yd = torch.as_tensor(np.ascontiguousarray(Y), device=self.device)
        self.ctx.call("fs_fcm_interpolate", self._p(u_window), self._p(Yd), n, self._p(V), self._p(W))
        return V, W

    def close(self):
        self.ctx.close()


class SlabFcm:
    """Fcm::mobility_solve of one box over `world` ranks (x slabs). Every rank
    calls mobility() with all beads (host arrays) and gets all V, W back."""

    def __init__(self, params, world=1, rank=0, group=None, max_beads=0, pieces=None):
        self.layout = SlabLayout(params, world, rank)
        self.ex = Exchange(world, rank, group)
        self.pieces = pieces if pieces is not None else LocalPieces(params, self.layout, max_beads)

    def mobility(self, Y, F, T):
        L, P, ex = self.layout, self.pieces, self.ex
        Y, F, T = (np.ascontiguousarray(a, dtype=np.float64) for a in (Y, F, T))
        own = np.nonzero(L.owners(Y) == L.rank)[0]
        # 1. spread into the window; its last H planes belong to the next rank
        fw = P.spread(Y[own], F[own], T[own])
        halo = torch.empty_like(fw[:, : L.H])
        ex.shift(fw[:, L.nxs:].contiguous(), halo, to_next=True)
        f = fw[:, : L.nxs].contiguous()
        f[:, : L.H] += halo
        # 2. z, y transforms; 3. to every rank its kz range of every x
        spec = P.forward_yz(f)
        send = torch.cat([spec[:, :, L.kz_bounds[d]:L.kz_bounds[d + 1]].reshape(-1) for d in range(L.world)])
        in_splits = [3 * L.nxs * L.nkz_of(d) * L.ny * 2 for d in range(L.world)]
        out_splits = [3 * L.nxs * L.nkz * L.ny * 2] * L.world
        recv = torch.empty(sum(out_splits), dtype=spec.dtype, device=spec.device)
        ex.all_to_all(recv, send, out_splits, in_splits)
        spec_t = (recv.view(L.world, 3, L.nxs, L.nkz, L.ny, 2).permute(1, 3, 4, 0, 2, 5)
                  .reshape(3, L.nkz, L.ny, L.nx, 2).contiguous())
        # 4. x transforms and the projection, then back
        P.solve_x(spec_t)
        back = (spec_t.view(3, L.nkz, L.ny, L.world, L.nxs, 2).permute(3, 0, 4, 1, 2, 5).reshape(-1).contiguous())
        recv2 = torch.empty(sum(in_splits), dtype=spec.dtype, device=spec.device)
        ex.all_to_all(recv2, back, in_splits, out_splits)
        parts, off = [], 0
        for d in range(L.world):
            n = in_splits[d]
            parts.append(recv2[off:off + n].view(3, L.nxs, L.nkz_of(d), L.ny, 2))
            off += n
        spec2 = torch.cat(parts, dim=2).contiguous()
        # 5. inverse y, z transforms; 6. the next rank's first H planes appended, interpolation
        u = P.inverse_yz(spec2)
        uh = torch.empty_like(u[:, : L.H])
        ex.shift(u[:, : L.H].contiguous(), uh, to_next=False)
        uw = torch.cat([u, uh], dim=1).contiguous()
        Vo, Wo = P.interpolate(uw, Y[own])
        # 7. one owner per bead: the sum over ranks assembles V and W
        VW = torch.zeros((2, Y.shape[0], 3), dtype=torch.float64, device=Vo.device)
        idx = torch.as_tensor(own, device=Vo.device)
        VW[0, idx] = Vo
        VW[1, idx] = Wo
        ex.all_reduce(VW)
        VW = VW.cpu().numpy()
        return VW[0], VW[1]

    def close(self):
        if hasattr(self.pieces, "close"):
            self.pieces.close()
