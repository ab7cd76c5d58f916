"""Host-side mirror of FilSim's hot-path interface over libfilsim_gpu's C-ABI.

Class and method names follow the reference so a main.cpp-shaped driver reads
the same:
  Fcm            struct Fcm (FCMfunctions.hpp:7-59)
  LinkedList     struct LinkedList (CollisionBarrierFilament.hpp:19-57)
  FilamentJsolver class filamentJsolver (FilamentJacobianSolver.hpp:14-87)
  Simulation     the filament suspension and the time loop of main.cpp:284-754

Device buffers are torch CUDA tensors (plumbing only); every computation runs
in the library's kernels. Errors raise FsError with the library's status.
"""
import ctypes

import numpy as np
import torch

from . import abi
from .abi import check, lib
from .suspension import Suspension


def _dptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _dev(x, device="cuda"):
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=torch.float64).contiguous()
    return torch.as_tensor(np.ascontiguousarray(x, dtype=np.float64), device=device)


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

    def set_precision(self, prec):
        check(lib().fs_set_precision(self.h, prec), "fs_set_precision")

    def device_bytes(self):
        n = ctypes.c_size_t()
        check(lib().fs_device_bytes(self.h, ctypes.byref(n)), "fs_device_bytes")
        return n.value


class Fcm:
    """struct Fcm: Y, F, T in; V, W out (Np x 3, device)."""

    def __init__(self, ctx, np_):
        self.ctx = ctx
        self.np = int(np_)
        z = lambda: torch.zeros((self.np, 3), dtype=torch.float64, device="cuda")
        self.Y, self.F, self.T, self.V, self.W = z(), z(), z(), z(), z()

    def mobility_solve(self):
        """Fcm::mobility_solve (FCMfunctions.cpp:175-464)."""
        check(lib().fs_fcm_mobility(self.ctx.h, _dptr(self.Y), _dptr(self.F), _dptr(self.T), _dptr(self.V),
                                    _dptr(self.W), self.np), "fs_fcm_mobility")

    def friction_mobility_solve(self):
        """Fcm::friction_mobility_solve (FCMfunctions.cpp:865-880)."""
        check(lib().fs_fcm_friction(self.ctx.h, _dptr(self.F), _dptr(self.T), _dptr(self.V), _dptr(self.W),
                                    self.np), "fs_fcm_friction")

    def spread(self):
        """The force grid f (3, Nx, Ny, Nz) of the current Y, F, T (FP64)."""
        p = self.ctx.params
        f = torch.empty((3, p.npts_x, p.npts_y, p.npts_z), dtype=torch.float64, device="cuda")
        check(lib().fs_fcm_spread(self.ctx.h, _dptr(self.Y), _dptr(self.F), _dptr(self.T), self.np, _dptr(f)),
              "fs_fcm_spread")
        return f

    def velocity_grid(self):
        p = self.ctx.params
        n = 3 * p.npts_x * p.npts_y * p.npts_z
        out = np.zeros(n)
        check(lib().fs_fcm_get_grid(self.ctx.h, out.ctypes.data_as(ctypes.c_void_p), n), "fs_fcm_get_grid")
        return out.reshape(3, p.npts_x, p.npts_y, p.npts_z)

    def flow_solve(self, f):
        f = _dev(f)
        u = torch.empty_like(f)
        check(lib().fs_fcm_flow_solve(self.ctx.h, _dptr(f), _dptr(u)), "fs_fcm_flow_solve")
        return u

    def set(self, Y=None, F=None, T=None):
        for name, val in (("Y", Y), ("F", F), ("T", T)):
            if val is not None:
                getattr(self, name).copy_(_dev(val).reshape(self.np, 3))


def mobility_host(ctx, Y, F, T):
    """fs_fcm_mobility_host: host arrays in, host arrays out."""
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    F = np.ascontiguousarray(F, dtype=np.float64)
    T = np.ascontiguousarray(T, dtype=np.float64)
    V = np.zeros_like(Y)
    W = np.zeros_like(Y)
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    check(lib().fs_fcm_mobility_host(ctx.h, vp(Y), vp(F), vp(T), vp(V), vp(W), Y.shape[0]),
          "fs_fcm_mobility_host")
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
        check(lib().fs_cells_link(self.ctx.h, _dptr(Xs), self.np), "fs_cells_link")

    def lists(self):
        head = np.zeros(self.ncell, dtype=np.int32)
        lst = np.zeros(max(self.np, 1), dtype=np.int32)
        mp = np.zeros(13 * self.ncell, dtype=np.int32)
        vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        check(lib().fs_cells_get_lists(self.ctx.h, vp(head), vp(lst), vp(mp)), "fs_cells_get_lists")
        return head, lst[: self.np], mp

    def apply_collision_barrier(self, Y, F, nt, fil_id=None, seg_id=None):
        """Adds barrier forces into F (device tensor, modified in place); returns min_dist2."""
        fid = torch.as_tensor(fil_id, dtype=torch.int32, device="cuda") if fil_id is not None else None
        sid = torch.as_tensor(seg_id, dtype=torch.int32, device="cuda") if seg_id is not None else None
        md = ctypes.c_double()
        check(lib().fs_collision_barrier(self.ctx.h, _dptr(Y), _dptr(F), Y.shape[0], nt, _dptr(fid), _dptr(sid),
                                         ctypes.byref(md)), "fs_collision_barrier")
        return md.value

    def pairs(self, Y, nt, fil_id=None, seg_id=None, max_pairs=1 << 20):
        fid = torch.as_tensor(fil_id, dtype=torch.int32, device="cuda") if fil_id is not None else None
        sid = torch.as_tensor(seg_id, dtype=torch.int32, device="cuda") if seg_id is not None else None
        out = np.zeros(2 * max_pairs, dtype=np.int32)
        n = ctypes.c_int()
        check(lib().fs_collision_pairs(self.ctx.h, _dptr(Y), Y.shape[0], nt, _dptr(fid), _dptr(sid),
                                       out.ctypes.data_as(ctypes.c_void_p), max_pairs, ctypes.byref(n)),
              "fs_collision_pairs")
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
        check(lib().fs_state_upload(self.ctx.h, ctypes.byref(self._hs.struct)), "fs_state_upload")

    def download(self):
        out = self.susp.empty_like_state()
        check(lib().fs_state_download(self.ctx.h, ctypes.byref(out.struct)), "fs_state_download")
        return out.arrays

    def device_array(self, which, shape):
        ptr = ctypes.c_void_p()
        check(lib().fs_state_device_ptr(self.ctx.h, which.encode(), ctypes.byref(ptr)), "fs_state_device_ptr")
        n = int(np.prod(shape))
        self.ctx.synchronize()
        # device-to-device copy (kind 3) through the CUDA runtime torch links
        t = torch.empty(n, dtype=torch.float64, device="cuda")
        torch.cuda.cudart().cudaMemcpy(t.data_ptr(), ptr.value, n * 8, 3)
        return t.reshape(shape)

    def initial_guess(self):
        check(lib().fs_initial_guess(self.ctx.h), "fs_initial_guess")

    def filament_forces(self, nt):
        check(lib().fs_filament_forces(self.ctx.h, nt), "fs_filament_forces")

    def build_jacobian(self, nt):
        check(lib().fs_jacobian_build(self.ctx.h, nt), "fs_jacobian_build")

    def jinv(self, f):
        nw = int(self.susp.fil_start[f + 1] - self.susp.fil_start[f])
        out = np.zeros((6 * nw, 6 * nw))
        check(lib().fs_jacobian_get_inverse(self.ctx.h, f, out.ctypes.data_as(ctypes.c_void_p), 6 * nw),
              "fs_jacobian_get_inverse")
        return out

    def error_check(self, V, W, nt):
        err = torch.zeros(6 * self.susp.np, dtype=torch.float64, device="cuda")
        chk = ctypes.c_int()
        check(lib().fs_error_check(self.ctx.h, _dptr(_dev(V)), _dptr(_dev(W)), _dptr(err), nt, ctypes.byref(chk)),
              "fs_error_check")
        return err, bool(chk.value)

    def broyden_apply(self, b, iter_):
        b = _dev(b)
        x = torch.zeros_like(b)
        check(lib().fs_broyden_apply(self.ctx.h, _dptr(b), _dptr(x), iter_), "fs_broyden_apply")
        return x

    def set_cols(self, c, d, iter_):
        check(lib().fs_broyden_set_cols(self.ctx.h, _dptr(_dev(c)), _dptr(_dev(d)), iter_), "fs_broyden_set_cols")

    def update(self, u):
        check(lib().fs_state_update(self.ctx.h, _dptr(_dev(u))), "fs_state_update")

    def step(self, nt):
        check(lib().fs_step(self.ctx.h, nt), "fs_step")

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
