"""ctypes bindings of the CPU oracle (oracle/fs_oracle.c).

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, always as the reference the results are compared with.
"""
import ctypes
import os
import subprocess

import numpy as np

from filsim_b200.abi import FsParams, FsHostState, P_double, P_int

_DIR = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_DIR, "_build", "libfs_oracle.so")
_lib = None


_REF_DIR = os.path.join(_DIR, "_ref")
REFERENCE_TREE = "/root/reference"


def build():
    subprocess.run(["make", "-s", "-C", _DIR], check=True)
    # the reference's own FCM and barrier sources, where the FilSim tree is present
    if os.path.isdir(REFERENCE_TREE):
        subprocess.run(["make", "-s", "-C", os.path.join(_DIR, "refshim"), "REF=" + REFERENCE_TREE], check=True)


# ---- the reference pin: the reference's own sources built by oracle/refshim ----
REF_FCM_CASES = {  # library tag -> (grid, ngd, dx rule)
    "fcm_64_ngd12": ((64, 64, 64), 12, "a/1.86"),
    "fcm_32_ngd20": ((32, 32, 32), 20, "sigma_dip/1.5"),
    "fcm_48x32x64_ngd20": ((48, 32, 64), 20, "sigma_dip/1.5"),
}
_ref_libs = {}


def ref_available(tag):
    return os.path.exists(os.path.join(_REF_DIR, "libref_%s.so" % tag))


def _ref_lib(tag):
    if tag not in _ref_libs:
        path = os.path.join(_REF_DIR, "libref_%s.so" % tag)
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = ctypes.CDLL(path)
        vp = ctypes.c_void_p
        L.ref_fcm_config.argtypes = [vp, vp]
        L.ref_fcm_mobility.restype = ctypes.c_int
        L.ref_fcm_mobility.argtypes = [ctypes.c_int, vp, vp, vp, vp, vp]
        if hasattr(L, "ref_barrier"):
            L.ref_barrier.restype = ctypes.c_int
            L.ref_barrier.argtypes = [ctypes.c_int, vp, vp, vp, vp, ctypes.c_int, vp, vp, vp, vp]
        _ref_libs[tag] = L
    return _ref_libs[tag]


def ref_config(tag):
    """(grid, ngd, dx) the reference library was compiled for."""
    L = _ref_lib(tag)
    cfg = np.zeros(4, dtype=np.int32)
    dx = ctypes.c_double()
    L.ref_fcm_config(_ptr(cfg), ctypes.byref(dx))
    return tuple(int(v) for v in cfg[:3]), int(cfg[3]), dx.value


def ref_fcm_mobility(tag, Y, F, T):
    """Fcm::initialise + Fcm::mobility_solve of the reference's own code."""
    L = _ref_lib(tag)
    Y, F, T = _f64(Y), _f64(F), _f64(T)
    V = np.zeros_like(Y)
    W = np.zeros_like(Y)
    st = L.ref_fcm_mobility(Y.shape[0], _ptr(Y), _ptr(F), _ptr(T), _ptr(V), _ptr(W))
    assert st == 0
    return V, W


def ref_barrier(tag, fil_start, Xs, Y, F, nt):
    """LinkedList::initialise, link and apply_collision_barrier of the reference's
    own code; returns (F after, head, list, min_dist2)."""
    L = _ref_lib(tag)
    fil_start = np.ascontiguousarray(fil_start, dtype=np.int32)
    Xs, Y = _f64(Xs), _f64(Y)
    F = _f64(F).copy()
    np_ = int(fil_start[-1])
    head = np.zeros(1 << 20, dtype=np.int32)
    lst = np.zeros(max(np_, 1), dtype=np.int32)
    nc = ctypes.c_int()
    md = ctypes.c_double()
    st = L.ref_barrier(len(fil_start) - 1, _ptr(fil_start), _ptr(Xs), _ptr(Y), _ptr(F), nt, _ptr(head), _ptr(lst),
                       ctypes.byref(nc), ctypes.byref(md))
    assert st == 0, st
    return F, head[: nc.value].copy(), lst[:np_].copy(), md.value


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = ctypes.CDLL(_SO)
        vp = ctypes.c_void_p
        pp = ctypes.POINTER(FsParams)
        L.or_fft_r2c_3d.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.or_fft_c2r_3d.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.or_fcm_mobility.argtypes = [pp, ctypes.c_int, vp, vp, vp, vp, vp, vp, vp]
        L.or_flow_solve.argtypes = [pp, vp, vp]
        L.or_fcm_friction.argtypes = [pp, ctypes.c_int, vp, vp, vp, vp]
        L.or_cells_dims.argtypes = [pp, vp]
        L.or_cells_bulkmap.argtypes = [vp, vp]
        L.or_cells_link.argtypes = [pp, ctypes.c_int, vp, vp, vp]
        L.or_collision_barrier.argtypes = [pp, ctypes.c_int, vp, vp, vp, vp, vp, vp, ctypes.c_int, vp, vp, vp,
                                           ctypes.c_int]
        L.or_system_create.restype = vp
        L.or_system_create.argtypes = [pp, ctypes.POINTER(FsHostState)]
        L.or_system_destroy.argtypes = [vp]
        L.or_system_get.argtypes = [vp, ctypes.POINTER(FsHostState)]
        L.or_system_set.argtypes = [vp, ctypes.POINTER(FsHostState)]
        L.or_system_array.restype = P_double
        L.or_system_array.argtypes = [vp, ctypes.c_char_p]
        for n in ("or_initial_guess",):
            getattr(L, n).argtypes = [vp]
        L.or_set_swimming.argtypes = [vp, vp, ctypes.c_double, ctypes.c_int]
        L.or_set_spring_links.argtypes = [vp, ctypes.c_int, vp, ctypes.c_double, ctypes.c_double]
        L.or_filament_forces.argtypes = [vp, ctypes.c_int]
        L.or_set_barrier_mode.argtypes = [vp, ctypes.c_int]
        L.or_step_gait_reset.restype = ctypes.c_int
        L.or_step_gait_reset.argtypes = [vp, ctypes.c_int, vp, vp]
        L.or_build_jacobian.argtypes = [vp, ctypes.c_int]
        L.or_get_jinv.argtypes = [vp, ctypes.c_int, vp]
        L.or_error_check.argtypes = [vp, vp, vp, vp, ctypes.c_int]
        L.or_jsolve.argtypes = [vp, vp, vp, ctypes.c_int]
        L.or_set_cols.argtypes = [vp, vp, vp, ctypes.c_int]
        L.or_update.argtypes = [vp, vp]
        L.or_step.argtypes = [vp, ctypes.c_int]
        L.or_step_implicit.argtypes = [vp, ctypes.c_int, vp]
        L.or_run_steps.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp]
        L.or_last_min_dist2.restype = ctypes.c_double
        L.or_last_min_dist2.argtypes = [vp]
        L.or_mobility_solves.restype = ctypes.c_longlong
        L.or_mobility_solves.argtypes = [vp]
        L.or_sample_costs.restype = ctypes.c_int
        L.or_sample_costs.argtypes = [vp, ctypes.c_int, vp]
        L.or_stage_costs.restype = ctypes.c_int
        L.or_stage_costs.argtypes = [vp, ctypes.c_int, ctypes.c_uint, ctypes.c_int, vp]
        L.or_suspension_random.restype = ctypes.c_int
        L.or_suspension_random.argtypes = [pp, ctypes.c_int, ctypes.c_int, ctypes.c_ulonglong, ctypes.c_double,
                                           ctypes.c_int, vp, vp]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _f64(a, n=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a


def suspension_random(p, nfil, nw, seed, min_sep=None, max_tries=1000000):
    """Bead positions X and quaternions Q of the seeded generator, restated on
    the CPU (or_suspension.c), so a CPU-only caller builds the same inputs as
    filsim_b200.suspension.random_suspension without the GPU library."""
    if min_sep is None:
        min_sep = 2.2 * p.a
    X = np.zeros((nfil * nw, 3))
    Q = np.zeros((nfil * nw, 4))
    st = lib().or_suspension_random(ctypes.byref(p), nfil, nw, seed, min_sep, max_tries, _ptr(X), _ptr(Q))
    if st != 0:
        raise RuntimeError("or_suspension_random failed: %d" % st)
    return X, Q


def fft_r2c_3d(x):
    x = _f64(x)
    nx, ny, nz = x.shape
    out = np.zeros((nx, ny, nz // 2 + 1), dtype=np.complex128)
    lib().or_fft_r2c_3d(_ptr(x), _ptr(out), nx, ny, nz)
    return out


def fft_c2r_3d(xh, nz):
    xh = np.ascontiguousarray(xh, dtype=np.complex128).copy()
    nx, ny, _ = xh.shape
    out = np.zeros((nx, ny, nz), dtype=np.float64)
    lib().or_fft_c2r_3d(_ptr(xh), _ptr(out), nx, ny, nz)
    return out


def fcm_mobility(p, Y, F, T, return_grids=False):
    Y, F, T = _f64(Y), _f64(F), _f64(T)
    np_ = Y.shape[0]
    V = np.zeros((np_, 3))
    W = np.zeros((np_, 3))
    N = p.npts_x * p.npts_y * p.npts_z
    fg = np.zeros(3 * N) if return_grids else None
    ug = np.zeros(3 * N) if return_grids else None
    st = lib().or_fcm_mobility(ctypes.byref(p), np_, _ptr(Y), _ptr(F), _ptr(T), _ptr(V), _ptr(W), _ptr(fg), _ptr(ug))
    assert st == 0, st
    if return_grids:
        shp = (3, p.npts_x, p.npts_y, p.npts_z)
        return V, W, fg.reshape(shp), ug.reshape(shp)
    return V, W


def flow_solve(p, f):
    f = _f64(f)
    u = np.zeros_like(f)
    st = lib().or_flow_solve(ctypes.byref(p), _ptr(f), _ptr(u))
    assert st == 0
    return u


def fcm_friction(p, F, T):
    F, T = _f64(F), _f64(T)
    V = np.zeros_like(F)
    W = np.zeros_like(T)
    lib().or_fcm_friction(ctypes.byref(p), F.shape[0], _ptr(F), _ptr(T), _ptr(V), _ptr(W))
    return V, W


def cells_dims(p):
    M = np.zeros(3, dtype=np.int32)
    lib().or_cells_dims(ctypes.byref(p), _ptr(M))
    return tuple(int(m) for m in M)


def cells_link(p, Xs):
    Xs = _f64(Xs)
    M = cells_dims(p)
    ncell = M[0] * M[1] * M[2]
    head = np.zeros(ncell, dtype=np.int32)
    lst = np.zeros(Xs.shape[0], dtype=np.int32)
    lib().or_cells_link(ctypes.byref(p), Xs.shape[0], _ptr(Xs), _ptr(head), _ptr(lst))
    mp = np.zeros(13 * ncell, dtype=np.int32)
    lib().or_cells_bulkmap(_ptr(np.array(M, dtype=np.int32)), _ptr(mp))
    return head, lst, mp


def collision_barrier(p, Y, F, fil_id, seg_id, head, lst, mp, nt, max_pairs=0):
    Y = _f64(Y)
    F = _f64(F).copy()
    md = np.zeros(1)
    pairs = np.zeros(2 * max_pairs, dtype=np.int32) if max_pairs else None
    fil_id = np.ascontiguousarray(fil_id, dtype=np.int32)
    seg_id = np.ascontiguousarray(seg_id, dtype=np.int32)
    n = lib().or_collision_barrier(ctypes.byref(p), Y.shape[0], _ptr(fil_id), _ptr(seg_id), _ptr(Y), _ptr(head),
                                   _ptr(lst), _ptr(mp), nt, _ptr(F), _ptr(md), _ptr(pairs), max_pairs)
    out = {"F": F, "min_dist2": float(md[0]), "npairs": int(n)}
    if max_pairs:
        out["pairs"] = pairs[: 2 * min(n, max_pairs)].reshape(-1, 2)
    return out


class System:
    """Oracle filament suspension (host arrays) with the reference's step."""

    FIELDS3 = ("X", "Xs", "Xt", "U", "Us", "Ut", "F", "TAU")
    FIELDS4 = ("q", "qs", "qt")

    def __init__(self, p, susp):
        self.p = p
        self.susp = susp
        hs = susp.host_state()
        self._keep = hs
        self.h = lib().or_system_create(ctypes.byref(p), ctypes.byref(hs.struct))

    def close(self):
        if self.h:
            lib().or_system_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def download(self):
        """Returns a dict of the state arrays."""
        s = self.susp.empty_like_state()
        lib().or_system_get(self.h, ctypes.byref(s.struct))
        return s.arrays

    def upload(self, susp):
        hs = susp.host_state()
        lib().or_system_set(self.h, ctypes.byref(hs.struct))

    def array(self, which, shape):
        ptr = lib().or_system_array(self.h, which.encode())
        n = int(np.prod(shape))
        return np.ctypeslib.as_array(ptr, shape=(n,)).reshape(shape).copy()

    def initial_guess(self):
        lib().or_initial_guess(self.h)

    def set_swimming(self, swim, curvature=0.0, sperm_decay=False):
        """swim: [nfil x 5] (alpha, beta, phase, wavenumber, angular frequency), or None."""
        if swim is None:
            lib().or_set_swimming(self.h, None, 0.0, 0)
            return
        self._swim = _f64(swim).reshape(-1, 5)
        lib().or_set_swimming(self.h, _ptr(self._swim), float(curvature), int(bool(sperm_decay)))

    def set_spring_links(self, beads, k, l0):
        """beads: [n x 2] global bead indices of the linked pairs, in link order."""
        self._springs = np.ascontiguousarray(beads, dtype=np.int32).reshape(-1, 2)
        lib().or_set_spring_links(self.h, self._springs.shape[0], _ptr(self._springs), float(k), float(l0))

    def filament_forces(self, nt):
        lib().or_filament_forces(self.h, nt)

    def set_barrier_mode(self, mode):
        lib().or_set_barrier_mode(self.h, int(mode))

    def step_gait_reset(self, nt):
        """Returns (iterations [3], V W F of filament 0 per solve [3, Nw0, 9], status)."""
        nw0 = int(self.susp.fil_start[1] - self.susp.fil_start[0])
        its = np.zeros(3, dtype=np.int32)
        vwf = np.zeros((3, nw0, 9))
        st = lib().or_step_gait_reset(self.h, nt, _ptr(its), _ptr(vwf))
        return its, vwf, st

    def build_jacobian(self, nt):
        lib().or_build_jacobian(self.h, nt)

    def jinv(self, f):
        nw = int(self.susp.fil_start[f + 1] - self.susp.fil_start[f])
        out = np.zeros((6 * nw, 6 * nw))
        lib().or_get_jinv(self.h, f, _ptr(out))
        return out

    def error_check(self, V, W, nt):
        V, W = _f64(V), _f64(W)
        err = np.zeros(6 * self.susp.np)
        chk = lib().or_error_check(self.h, _ptr(V), _ptr(W), _ptr(err), nt)
        return err, bool(chk)

    def jsolve(self, b, iter_):
        b = _f64(b)
        x = np.zeros_like(b)
        lib().or_jsolve(self.h, _ptr(b), _ptr(x), iter_)
        return x

    def set_cols(self, c, d, iter_):
        lib().or_set_cols(self.h, _ptr(_f64(c)), _ptr(_f64(d)), iter_)

    def update(self, u):
        lib().or_update(self.h, _ptr(_f64(u)))

    def step(self, nt):
        lib().or_step(self.h, nt)

    def step_implicit(self, nt):
        it = np.zeros(1, dtype=np.int32)
        st = lib().or_step_implicit(self.h, nt, _ptr(it))
        return int(it[0]), st

    def run_steps(self, nt_start, nsteps):
        its = np.zeros(nsteps, dtype=np.int32)
        st = lib().or_run_steps(self.h, nt_start, nsteps, _ptr(its))
        return its, st

    def min_dist2(self):
        return lib().or_last_min_dist2(self.h)

    STAGE_NAMES = ("spread", "fft_fwd", "project", "fft_inv", "interp", "jacobian", "iteration_other", "barrier")

    def stage_costs(self, stages, stride=1, warm=False):
        """Wall seconds of the named stages (STAGE_NAMES) of one iteration, each
        on every stride-th work unit and scaled back (stride 1: full size);
        returns (dict of the stages run, threads)."""
        parts = np.zeros(9)
        mask = 0
        for name in stages:
            mask |= 1 << self.STAGE_NAMES.index(name)
        nth = lib().or_stage_costs(self.h, stride, mask, int(bool(warm)), _ptr(parts))
        if nth < 0:
            raise MemoryError("or_stage_costs: workspace allocation failed")
        return {n: float(parts[i]) for i, n in enumerate(self.STAGE_NAMES) if mask & (1 << i)}, int(nth)

    def sample_costs(self, stride):
        """Stage wall seconds of one iteration, sampled on 1/stride of the work
        units and scaled back; returns (dict, threads)."""
        parts = np.zeros(9)
        nth = lib().or_sample_costs(self.h, stride, _ptr(parts))
        return dict(zip(self.STAGE_NAMES, parts[:8].tolist())), int(nth)
