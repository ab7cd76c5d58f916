"""ctypes mirror of include/filsim_gpu.h and the loader of libfilsim_gpu.so.

The structures here are plain data; importing this module does not load the
CUDA library. ``lib()`` loads it on first use and raises if it is missing: there
is no CPU fallback.
"""
import ctypes
import math
import os

c_int = ctypes.c_int
c_double = ctypes.c_double
c_void_p = ctypes.c_void_p
c_size_t = ctypes.c_size_t
c_longlong = ctypes.c_longlong
P_int = ctypes.POINTER(c_int)
P_double = ctypes.POINTER(c_double)

PI = 3.14159265358979323846264338327950288

FS_OK = 0
STATUS_NAMES = {
    0: "FS_OK", 1: "FS_ERR_INVALID_ARG", 2: "FS_ERR_NO_DEVICE", 3: "FS_ERR_CUDA", 4: "FS_ERR_CUFFT",
    5: "FS_ERR_OOM", 6: "FS_ERR_NOT_CONVERGED", 7: "FS_ERR_NONFINITE", 8: "FS_ERR_CAPACITY", 9: "FS_ERR_STATE",
    10: "FS_ERR_IO",
}
FS_ERR_INVALID_ARG = 1
FS_ERR_NO_DEVICE = 2
FS_ERR_CUDA = 3
FS_ERR_CUFFT = 4
FS_ERR_OOM = 5
FS_ERR_NOT_CONVERGED = 6
FS_ERR_NONFINITE = 7
FS_ERR_CAPACITY = 8
FS_ERR_STATE = 9
FS_ERR_IO = 10
FS_BARRIER_ALL, FS_BARRIER_NOT_SWIMMER, FS_BARRIER_NOT_TEST_PARTICLES, FS_BARRIER_OFF = 0, 1, 2, 3
FS_PREC_FP64 = 0
FS_PREC_FP32 = 1


class FsParams(ctypes.Structure):
    """fs_params: runtime replacement of config.hpp / multi_filament_header.hpp:32-81."""
    _fields_ = [
        ("npts_x", c_int), ("npts_y", c_int), ("npts_z", c_int), ("ngd", c_int),
        ("a", c_double), ("ah", c_double), ("mu", c_double), ("dx", c_double),
        ("sigma", c_double), ("sigma_dip", c_double), ("dl", c_double), ("dt", c_double),
        ("gravity", c_double * 3), ("strain_twist", c_double * 3), ("tol", c_double),
        ("broyden_maxiter", c_int), ("impl_euler_steps", c_int), ("initial_friction_steps", c_int),
        ("precision", c_int),
        ("barrier_fs_over_2a", c_double), ("barrier_distance_cap", c_double), ("cell_width", c_double),
        ("lambda_extrap_step", c_int), ("reserved0", c_int),
    ]


class FsDiag(ctypes.Structure):
    _fields_ = [
        ("last_nt", c_int), ("last_iters", c_int), ("total_iters", c_longlong), ("mobility_solves", c_longlong),
        ("not_converged_steps", c_int), ("nonfinite", c_int), ("explosion", c_int), ("reserved", c_int),
        ("min_dist2", c_double), ("last_max_abs_err", c_double),
        ("learned_filaments", c_longlong), ("fallback_filaments", c_longlong), ("escalated_iters", c_longlong),
    ]


STAGES = ["spread", "fft_fwd", "project", "fft_inv", "interp", "link", "barrier", "forces", "jacobian",
          "error_check", "broyden", "update", "friction", "learn",
          # single kernels inside the stages above
          "k_spread", "k_fft_z_fwd", "k_fft_y_fwd", "k_fft_y_inv", "k_fft_z_inv", "k_interp"]
FS_STAGE_COUNT = 32


class FsProfile(ctypes.Structure):
    _fields_ = [("ms", c_double * FS_STAGE_COUNT), ("calls", c_longlong * FS_STAGE_COUNT)]


class FsHostState(ctypes.Structure):
    _fields_ = [
        ("nfil", c_int), ("np", c_int), ("fil_start", P_int),
        ("X", P_double), ("Xs", P_double), ("Xt", P_double),
        ("U", P_double), ("Us", P_double), ("Ut", P_double),
        ("q", P_double), ("qs", P_double), ("qt", P_double),
        ("F", P_double), ("TAU", P_double),
        ("lam", P_double), ("lam1", P_double), ("lam2", P_double),
        ("kap", P_double), ("c", P_double),
    ]


class FsRunInfo(ctypes.Structure):
    """fs_run_info: the columns of the reference's .par file."""
    _fields_ = [
        ("simulation_name", ctypes.c_char * 128), ("simulation_tag", ctypes.c_char * 128),
        ("a", c_double), ("ah", c_double), ("dl", c_double), ("sp4", c_double), ("kap", c_double),
        ("c", c_double), ("mu", c_double), ("curvature", c_double), ("k0", c_double),
        ("time_steps", c_double), ("steps_per_period", c_double), ("tol", c_double),
        ("broyden_maxiter", c_int), ("box", c_double * 3), ("plot_steps", c_int),
        ("strain_twist", c_double * 3),
        ("kap_network_filaments", c_double), ("bnumber", c_double), ("steps_per_settling_time", c_double),
        ("dt", c_double), ("initial_friction_steps", c_int), ("enable_spring_links", c_int),
        ("cn_num_swimming_filaments", c_double), ("cn_num_nodes", c_double), ("cn_connection_radius", c_double),
        ("cn_min_node_spacing", c_double), ("cn_spacing_away_from_node", c_double),
        ("network_spring_constant", c_double), ("network_spring_natural_length", c_double),
    ]


def make_params(npts, ngd=12, a=1.0, dx=None, **kw):
    """Parameters with the reference's derived defaults (multi_filament_header.hpp:47-60).

    dx defaults to sigma_dip/1.5 as in the reference; the benchmark
    configurations pass dx = a/1.86 explicitly.
    """
    if isinstance(npts, int):
        npts = (npts, npts, npts)
    p = FsParams()
    p.npts_x, p.npts_y, p.npts_z = npts
    p.ngd = ngd
    p.a = a
    p.ah = kw.pop("ah", a)
    p.mu = kw.pop("mu", 1.0)
    p.sigma_dip = kw.pop("sigma_dip", a / (36.0 * PI) ** (1.0 / 6.0))
    p.sigma = kw.pop("sigma", a / math.sqrt(PI))
    p.dx = dx if dx is not None else p.sigma_dip / 1.5
    p.dl = kw.pop("dl", 2.2 * a)
    p.dt = kw.pop("dt", 0.05)
    g = kw.pop("gravity", (0.0, 0.0, 0.0))
    st = kw.pop("strain_twist", (0.0, 0.0, 0.0))
    for i in range(3):
        p.gravity[i] = g[i]
        p.strain_twist[i] = st[i]
    p.tol = kw.pop("tol", 1e-6)
    p.broyden_maxiter = kw.pop("broyden_maxiter", 300)
    p.impl_euler_steps = kw.pop("impl_euler_steps", 1)
    p.initial_friction_steps = kw.pop("initial_friction_steps", 0)
    p.precision = kw.pop("precision", FS_PREC_FP64)
    p.barrier_fs_over_2a = kw.pop("barrier_fs_over_2a", 15 * PI)
    p.barrier_distance_cap = kw.pop("barrier_distance_cap", 2.0)
    p.cell_width = kw.pop("cell_width", 2.5 * a)
    p.lambda_extrap_step = kw.pop("lambda_extrap_step", 12)
    if kw:
        raise TypeError("unknown parameters: %s" % sorted(kw))
    return p


def box_lengths(p):
    return (p.npts_x * p.dx, p.npts_y * p.dx, p.npts_z * p.dx)


_PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG_DIR, "_lib", "libfilsim_gpu.so")
_lib = None


class FsError(RuntimeError):
    def __init__(self, status, where):
        self.status = status
        super().__init__("%s failed: %s (%d)" % (where, STATUS_NAMES.get(status, "?"), status))


def _declare(L):
    sig = {
        "fs_abi_version": (c_int, []),
        "fs_status_string": (ctypes.c_char_p, [c_int]),
        "fs_params_default": (None, [ctypes.POINTER(FsParams), c_int, c_int, c_int]),
        "fs_create": (c_int, [ctypes.POINTER(FsParams), c_int, c_int, c_void_p, ctypes.POINTER(c_void_p)]),
        "fs_destroy": (c_int, [c_void_p]),
        "fs_get_params": (c_int, [c_void_p, ctypes.POINTER(FsParams)]),
        "fs_set_precision": (c_int, [c_void_p, c_int]),
        "fs_synchronize": (c_int, [c_void_p]),
        "fs_device_bytes": (c_int, [c_void_p, ctypes.POINTER(c_size_t)]),
        "fs_fcm_mobility": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int]),
        "fs_fcm_mobility_host": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int]),
        "fs_fcm_friction": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int]),
        "fs_fcm_get_grid": (c_int, [c_void_p, c_void_p, c_size_t]),
        "fs_fcm_spread": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
        "fs_fcm_flow_solve": (c_int, [c_void_p, c_void_p, c_void_p]),
        "fs_cells_dims": (c_int, [c_void_p, c_void_p]),
        "fs_cells_link": (c_int, [c_void_p, c_void_p, c_int]),
        "fs_cells_get_lists": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
        "fs_collision_barrier": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p, c_void_p]),
        "fs_collision_pairs": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
        "fs_state_upload": (c_int, [c_void_p, ctypes.POINTER(FsHostState)]),
        "fs_state_download": (c_int, [c_void_p, ctypes.POINTER(FsHostState)]),
        "fs_state_device_ptr": (c_int, [c_void_p, ctypes.c_char_p, ctypes.POINTER(c_void_p)]),
        "fs_initial_guess": (c_int, [c_void_p]),
        "fs_filament_forces": (c_int, [c_void_p, c_int]),
        "fs_set_swimming": (c_int, [c_void_p, c_void_p, c_double, c_int]),
        "fs_set_spring_links": (c_int, [c_void_p, c_int, c_void_p, c_double, c_double]),
        "fs_set_barrier_mode": (c_int, [c_void_p, c_int]),
        "fs_step_gait_reset": (c_int, [c_void_p, c_int, c_void_p, c_void_p]),
        "fs_jacobian_build": (c_int, [c_void_p, c_int]),
        "fs_jacobian_get_inverse": (c_int, [c_void_p, c_int, c_void_p, c_int]),
        "fs_error_check": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
        "fs_broyden_apply": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
        "fs_broyden_set_cols": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
        "fs_state_update": (c_int, [c_void_p, c_void_p]),
        "fs_step": (c_int, [c_void_p, c_int]),
        "fs_step_implicit": (c_int, [c_void_p, c_int, c_void_p]),
        "fs_run_steps": (c_int, [c_void_p, c_int, c_int, c_void_p]),
        "fs_get_diag": (c_int, [c_void_p, ctypes.POINTER(FsDiag)]),
        "fs_suspension_random": (c_int, [ctypes.POINTER(FsParams), c_int, c_int, ctypes.c_ulonglong, c_double,
                                         c_int, c_void_p, c_void_p]),
        "fs_kernel_launches": (ctypes.c_ulonglong, []),
        "fs_collision_barrier_noalloc": (c_int, [ctypes.POINTER(FsParams), c_void_p, c_void_p, c_void_p, c_int, c_int,
                                                 c_void_p, c_void_p, c_void_p, c_void_p]),
        "fs_profile_enable": (c_int, [c_void_p, c_int]),
        "fs_profile_get": (c_int, [c_void_p, ctypes.POINTER(FsProfile)]),
        "fs_mlp_create": (c_int, [c_void_p, c_int, c_int, c_int, ctypes.c_ulonglong]),
        "fs_mlp_dims": (c_int, [c_void_p, c_void_p]),
        "fs_mlp_set_normalization": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
        "fs_mlp_get_params": (c_int, [c_void_p, c_void_p, c_size_t]),
        "fs_mlp_set_params": (c_int, [c_void_p, c_void_p, c_size_t]),
        "fs_mlp_forward": (c_int, [c_void_p, c_void_p, c_int, c_void_p]),
        "fs_mlp_gradients": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_size_t, c_void_p]),
        "fs_mlp_train_step": (c_int, [c_void_p, c_void_p, c_void_p, c_int, ctypes.c_float, c_void_p]),
        "fs_learn_features": (c_int, [c_void_p, c_void_p]),
        "fs_learn_record": (c_int, [c_void_p, c_int]),
        "fs_learn_targets": (c_int, [c_void_p, c_void_p]),
        "fs_set_warm_start": (c_int, [c_void_p, c_int]),
        "fs_warm_start_gate": (c_int, [c_void_p, c_int]),
        "fs_set_start_order": (c_int, [c_void_p, c_int]),
        "fs_set_tension_extrapolation": (c_int, [c_void_p, c_int]),
        "fs_set_precision_escalation": (c_int, [c_void_p, c_int]),
        "fs_set_broyden_memory": (c_int, [c_void_p, c_int, c_int, c_int, c_int]),
        "fs_set_velocity_predictor": (c_int, [c_void_p, c_double]),
        "fs_warm_start_gate_margin": (c_int, [c_void_p, c_double]),
        "fs_warm_start_bound": (c_int, [c_void_p, c_int]),
        "fs_set_slab": (c_int, [c_void_p, c_int, c_int]),
        "fs_fcm_interpolate": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p]),
        "fs_slab_forward_yz": (c_int, [c_void_p, c_void_p, c_int, c_void_p]),
        "fs_slab_solve_x": (c_int, [c_void_p, c_void_p, c_int, c_int]),
        "fs_slab_inverse_yz": (c_int, [c_void_p, c_void_p, c_int, c_void_p]),
        "fs_warm_start_gate_stats": (c_int, [c_void_p, c_void_p, c_void_p]),
        "fs_set_graph_mode": (c_int, [c_void_p, c_int]),
        "fs_autotune": (c_int, [c_void_p, c_int, c_void_p, c_void_p]),
        "fs_set_tuning": (c_int, [c_void_p, c_void_p]),
        "fs_batch_create": (c_int, [c_void_p, c_int, ctypes.POINTER(c_void_p)]),
        "fs_batch_destroy": (c_int, [c_void_p]),
        "fs_batch_run": (c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p, c_void_p]),
        "fs_learn_override": (c_int, [c_void_p, c_void_p]),
        "fs_gemm_bf16": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int, c_int]),
        "fs_par_write": (c_int, [ctypes.c_char_p, ctypes.POINTER(FsRunInfo), ctypes.POINTER(FsHostState)]),
        "fs_par_read_layout": (c_int, [ctypes.c_char_p, ctypes.POINTER(c_int), ctypes.POINTER(c_int), c_void_p,
                                       c_int]),
        "fs_backup_write": (c_int, [ctypes.c_char_p, ctypes.POINTER(FsHostState), c_int]),
        "fs_backup_read": (c_int, [ctypes.c_char_p, ctypes.POINTER(FsHostState), ctypes.POINTER(c_int)]),
        "fs_data_write_header": (c_int, [ctypes.c_char_p, ctypes.POINTER(FsHostState)]),
        "fs_data_append": (c_int, [ctypes.c_char_p, ctypes.POINTER(FsHostState), c_int]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    return L


# every symbol include/filsim_gpu.h declares
EXPORTED_SYMBOLS = None


def header_symbols(header_path=None):
    """Function names declared in include/filsim_gpu.h (parsed, not hard-coded)."""
    import re
    if header_path is None:
        header_path = os.path.join(os.path.dirname(_PKG_DIR), "include", "filsim_gpu.h")
    text = open(header_path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fs_[a-z0-9_]+)\s*\(", text)))


def lib():
    """Load libfilsim_gpu.so (built in-tree by __graft_entry__.build())."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libfilsim_gpu.so not built at %s: run __graft_entry__.build()" % LIB_PATH)
        _lib = _declare(ctypes.CDLL(LIB_PATH))
    return _lib


def check(status, where):
    if status != FS_OK:
        raise FsError(status, where)
    return status
