"""Host-side mirror of FilSim's hot-path interface over libfilsim_gpu's C-ABI.

Class and method names follow the reference so a main.cpp-shaped driver reads
the same:
  Fcm             struct Fcm (FCMfunctions.hpp:7-59)
  LinkedList      struct LinkedList (CollisionBarrierFilament.hpp:19-57)
  Simulation      the filament suspension with Filament's per-step calls,
                  filamentJsolver (FilamentJacobianSolver.hpp:14-87) and the
                  time loop of main.cpp:284-754

Device buffers are torch CUDA tensors (plumbing only); every computation runs
in the library's kernels. Each wrapper call keeps its argument tensors alive
and synchronises the context before returning, so torch may reuse or read the
memory afterwards. Errors raise FsError with the library's status.
"""
import ctypes

import numpy as np
import torch

from . import abi
from .abi import check, lib


def _dptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _dev(x, dtype=torch.float64):
    if isinstance(x, torch.Tensor):
        return x.to(device="cuda", dtype=dtype).contiguous()
    npdt = np.float64 if dtype == torch.float64 else np.int32
    return torch.as_tensor(np.ascontiguousarray(x, dtype=npdt), device="cuda")


class _DeviceView:
    """__cuda_array_interface__ over a library-owned device array."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 2}


class Context:
    """Owns one fs_ctx (grids, cuFFT plans, cell lists, suspension buffers)."""

    def __init__(self, params, max_beads, max_filaments=None, stream=None):
        self.params = params
        self.max_beads = int(max_beads)
        self.max_filaments = int(max_filaments if max_filaments is not None else max(1, max_beads))
        h = ctypes.c_void_p()
        st = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        check(lib().fs_create(ctypes.byref(params), self.max_beads, self.max_filaments, st, ctypes.byref(h)),
              "fs_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().fs_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self):
        check(lib().fs_synchronize(self.h), "fs_synchronize")

    def call(self, name, *args):
        """Calls fs_<name>(ctx, *args), then synchronises the context."""
        check(getattr(lib(), name)(self.h, *args), name)
        self.synchronize()

    def set_precision(self, prec):
        check(lib().fs_set_precision(self.h, prec), "fs_set_precision")

    def set_start_order(self, order):
        """1: the reference's start (first bead from 2X - Xt); 2: the first bead from
        3X - 3Xt + Xtt once the context holds the positions two steps back."""
        check(lib().fs_set_start_order(self.h, order), "fs_set_start_order")

    def set_tension_extrapolation(self, order):
        """2: the reference's quadratic tension extrapolation after lambda_extrap_step;
        1: linear from lambda_extrap_step on."""
        check(lib().fs_set_tension_extrapolation(self.h, order), "fs_set_tension_extrapolation")

    def set_broyden_memory(self, keep_columns, carry_columns=0, threshold=0, restart_after=0):
        """Broyden memory across steps: after a step of fewer than `threshold`
        iterations J0 and up to keep_columns history columns continue into the next
        step; after a longer one its last carry_columns columns start the next step
        beside a new J0; a step on carried state reaching restart_after iterations
        starts afresh (0: never). keep_columns = carry_columns = 0 turns it off."""
        check(lib().fs_set_broyden_memory(self.h, keep_columns, carry_columns, threshold, restart_after),
              "fs_set_broyden_memory")

    def set_velocity_predictor(self, weight):
        """Before each step's first residual, one Broyden update of the given weight
        from the residual with V, W extrapolated from the last two converged states
        (no solve); 0 turns it off."""
        check(lib().fs_set_velocity_predictor(self.h, float(weight)), "fs_set_velocity_predictor")

    def set_precision_escalation(self, after_iters):
        """FP32 steps still not converged after after_iters Broyden iterations run the
        rest of their iterations with the FP64 chain; 0 turns it off."""
        check(lib().fs_set_precision_escalation(self.h, after_iters), "fs_set_precision_escalation")

    def device_bytes(self):
        n = ctypes.c_size_t()
        check(lib().fs_device_bytes(self.h, ctypes.byref(n)), "fs_device_bytes")
        return n.value

    def profile_enable(self, on=True):
        check(lib().fs_profile_enable(self.h, 1 if on else 0), "fs_profile_enable")

    def profile(self):
        """{stage: (milliseconds, calls)} since the last profile_enable."""
        pr = abi.FsProfile()
        check(lib().fs_profile_get(self.h, ctypes.byref(pr)), "fs_profile_get")
        return {name: (pr.ms[i], pr.calls[i]) for i, name in enumerate(abi.STAGES)}


class Fcm:
    """struct Fcm: Y, F, T in; V, W out (Np x 3, device)."""

    def __init__(self, ctx, np_):
        self.ctx = ctx
        self.np = int(np_)
        z = lambda: torch.zeros((self.np, 3), dtype=torch.float64, device="cuda")
        self.Y, self.F, self.T, self.V, self.W = z(), z(), z(), z(), z()

    def mobility_solve(self):
        """Fcm::mobility_solve (FCMfunctions.cpp:175-464)."""
        self.ctx.call("fs_fcm_mobility", _dptr(self.Y), _dptr(self.F), _dptr(self.T), _dptr(self.V),
                      _dptr(self.W), self.np)

    def friction_mobility_solve(self):
        """Fcm::friction_mobility_solve (FCMfunctions.cpp:865-880)."""
        self.ctx.call("fs_fcm_friction", _dptr(self.F), _dptr(self.T), _dptr(self.V), _dptr(self.W), self.np)

    def spread(self):
        """The force grid f (3, Nx, Ny, Nz, float64) of the current Y, F, T, spread in
        the context's precision."""
        p = self.ctx.params
        f = torch.empty((3, p.npts_x, p.npts_y, p.npts_z), dtype=torch.float64, device="cuda")
        self.ctx.call("fs_fcm_spread", _dptr(self.Y), _dptr(self.F), _dptr(self.T), self.np, _dptr(f))
        return f

    def velocity_grid(self):
        p = self.ctx.params
        n = 3 * p.npts_x * p.npts_y * p.npts_z
        out = np.zeros(n)
        self.ctx.call("fs_fcm_get_grid", out.ctypes.data_as(ctypes.c_void_p), n)
        return out.reshape(3, p.npts_x, p.npts_y, p.npts_z)

    def flow_solve(self, f):
        f = _dev(f)
        u = torch.empty_like(f)
        self.ctx.call("fs_fcm_flow_solve", _dptr(f), _dptr(u))
        return u

    def set(self, Y=None, F=None, T=None):
        for name, val in (("Y", Y), ("F", F), ("T", T)):
            if val is not None:
                getattr(self, name).copy_(_dev(val).reshape(self.np, 3))
        torch.cuda.synchronize()


def mobility_host(ctx, Y, F, T):
    """fs_fcm_mobility_host: host arrays in, host arrays out."""
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    F = np.ascontiguousarray(F, dtype=np.float64)
    T = np.ascontiguousarray(T, dtype=np.float64)
    V = np.zeros_like(Y)
    W = np.zeros_like(Y)
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    ctx.call("fs_fcm_mobility_host", vp(Y), vp(F), vp(T), vp(V), vp(W), Y.shape[0])
    return V, W


class LinkedList:
    """struct LinkedList: cell lists and the collision barrier."""

    def __init__(self, ctx):
        self.ctx = ctx
        M = np.zeros(3, dtype=np.int32)
        check(lib().fs_cells_dims(ctx.h, M.ctypes.data_as(ctypes.c_void_p)), "fs_cells_dims")
        self.M = tuple(int(m) for m in M)
        self.ncell = self.M[0] * self.M[1] * self.M[2]
        self.np = 0

    def link(self, Xs):
        """LinkedList::link (CollisionBarrierFilament.cpp:370-433) from unwrapped positions."""
        Xs = _dev(Xs)
        self.np = Xs.shape[0]
        self.ctx.call("fs_cells_link", _dptr(Xs), self.np)

    def lists(self):
        head = np.zeros(self.ncell, dtype=np.int32)
        lst = np.zeros(max(self.np, 1), dtype=np.int32)
        mp = np.zeros(13 * self.ncell, dtype=np.int32)
        vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        self.ctx.call("fs_cells_get_lists", vp(head), vp(lst), vp(mp))
        return head, lst[: self.np], mp

    def apply_collision_barrier(self, Y, F, nt, fil_id=None, seg_id=None):
        """Adds barrier forces into F (device tensor, modified in place); returns min_dist2."""
        fid = _dev(fil_id, torch.int32) if fil_id is not None else None
        sid = _dev(seg_id, torch.int32) if seg_id is not None else None
        md = ctypes.c_double()
        self.ctx.call("fs_collision_barrier", _dptr(Y), _dptr(F), Y.shape[0], nt, _dptr(fid), _dptr(sid),
                      ctypes.byref(md))
        return md.value

    def pairs(self, Y, nt, fil_id=None, seg_id=None, max_pairs=1 << 20):
        fid = _dev(fil_id, torch.int32) if fil_id is not None else None
        sid = _dev(seg_id, torch.int32) if seg_id is not None else None
        out = np.zeros(2 * max_pairs, dtype=np.int32)
        n = ctypes.c_int()
        self.ctx.call("fs_collision_pairs", _dptr(Y), Y.shape[0], nt, _dptr(fid), _dptr(sid),
                      out.ctypes.data_as(ctypes.c_void_p), max_pairs, ctypes.byref(n))
        return out[: 2 * min(n.value, max_pairs)].reshape(-1, 2), n.value


class Simulation:
    """Device-resident filament suspension with the reference's implicit step."""

    def __init__(self, ctx, susp):
        self.ctx = ctx
        self.susp = susp
        self.upload(susp)

    def upload(self, susp):
        self.susp = susp
        self._hs = susp.host_state()
        self.ctx.call("fs_state_upload", ctypes.byref(self._hs.struct))

    def download(self):
        out = self.susp.empty_like_state()
        self.ctx.call("fs_state_download", ctypes.byref(out.struct))
        return out.arrays

    def download_into(self, susp):
        """Downloads the device state into susp's own arrays (e.g. pinned ones)."""
        hs = susp.host_state()
        self.ctx.call("fs_state_download", ctypes.byref(hs.struct))

    def device_array(self, which, shape):
        """A copy of a library-resident array (Y, V, W, err, ...)."""
        ptr = ctypes.c_void_p()
        check(lib().fs_state_device_ptr(self.ctx.h, which.encode(), ctypes.byref(ptr)), "fs_state_device_ptr")
        self.ctx.synchronize()
        n = int(np.prod(shape))
        return torch.as_tensor(_DeviceView(ptr.value, n), device="cuda").clone().reshape(shape)

    def initial_guess(self):
        self.ctx.call("fs_initial_guess")

    def filament_forces(self, nt):
        self.ctx.call("fs_filament_forces", nt)

    def set_swimming(self, swim, curvature=0.0, sperm_decay=False):
        """Swimming drive: swim = [nfil x 5] (Alpha, Beta, Phase, Wavenumber,
        AngFrequency) per filament, or None to switch it off (fs_set_swimming)."""
        if swim is None:
            self.ctx.call("fs_set_swimming", None, 0.0, 0)
            return
        self._swim = np.ascontiguousarray(swim, dtype=np.float64).reshape(-1, 5)
        if self._swim.shape[0] != self.susp.nfil:
            raise ValueError("swim needs one row per filament")
        self.ctx.call("fs_set_swimming", self._swim.ctypes.data_as(ctypes.c_void_p), float(curvature),
                      int(bool(sperm_decay)))

    def set_barrier_mode(self, mode):
        """Pair filter of the step's collision barrier (abi.FS_BARRIER_*)."""
        self.ctx.call("fs_set_barrier_mode", int(mode))

    def step_gait_reset(self, nt):
        """One gait-reset step (main_gaitreset.cpp:302-830): returns the three
        solves' iterations, filament 0's V, W, F per solve [3, Nw0, 9] and the status."""
        nw0 = int(self.susp.fil_start[1] - self.susp.fil_start[0])
        its = np.zeros(3, dtype=np.int32)
        vwf = np.zeros((3, nw0, 9))
        st = lib().fs_step_gait_reset(self.ctx.h, nt, its.ctypes.data_as(ctypes.c_void_p),
                                      vwf.ctypes.data_as(ctypes.c_void_p))
        if st not in (abi.FS_OK, abi.FS_ERR_NOT_CONVERGED):
            check(st, "fs_step_gait_reset")
        return its, vwf, st

    def set_spring_links(self, beads, k, l0):
        """Spring links: beads = [n x 2] global bead indices, in link order
        (spring_links::apply_spring_link_forces; fs_set_spring_links)."""
        self._springs = np.ascontiguousarray(beads, dtype=np.int32).reshape(-1, 2)
        self.ctx.call("fs_set_spring_links", self._springs.shape[0], self._springs.ctypes.data_as(ctypes.c_void_p),
                      float(k), float(l0))

    def build_jacobian(self, nt):
        self.ctx.call("fs_jacobian_build", nt)

    def jinv(self, f):
        nw = int(self.susp.fil_start[f + 1] - self.susp.fil_start[f])
        out = np.zeros((6 * nw, 6 * nw))
        self.ctx.call("fs_jacobian_get_inverse", f, out.ctypes.data_as(ctypes.c_void_p), 6 * nw)
        return out

    def error_check(self, V, W, nt):
        V, W = _dev(V), _dev(W)
        err = torch.zeros(6 * self.susp.np, dtype=torch.float64, device="cuda")
        chk = ctypes.c_int()
        self.ctx.call("fs_error_check", _dptr(V), _dptr(W), _dptr(err), nt, ctypes.byref(chk))
        return err, bool(chk.value)

    def broyden_apply(self, b, iter_):
        b = _dev(b)
        x = torch.zeros_like(b)
        self.ctx.call("fs_broyden_apply", _dptr(b), _dptr(x), iter_)
        return x

    def set_cols(self, c, d, iter_):
        c, d = _dev(c), _dev(d)
        self.ctx.call("fs_broyden_set_cols", _dptr(c), _dptr(d), iter_)

    def update(self, u):
        u = _dev(u)
        self.ctx.call("fs_state_update", _dptr(u))

    def step(self, nt):
        self.ctx.call("fs_step", nt)

    def step_implicit(self, nt):
        it = ctypes.c_int()
        st = lib().fs_step_implicit(self.ctx.h, nt, ctypes.byref(it))
        if st not in (abi.FS_OK, abi.FS_ERR_NOT_CONVERGED):
            check(st, "fs_step_implicit")
        return it.value, st

    def run_steps(self, nt_start, nsteps):
        its = np.zeros(nsteps, dtype=np.int32)
        st = lib().fs_run_steps(self.ctx.h, nt_start, nsteps, its.ctypes.data_as(ctypes.c_void_p))
        if st not in (abi.FS_OK, abi.FS_ERR_NOT_CONVERGED):
            check(st, "fs_run_steps")
        return its, st

    def diag(self):
        d = abi.FsDiag()
        check(lib().fs_get_diag(self.ctx.h, ctypes.byref(d)), "fs_get_diag")
        return d
