"""FCM mobility on the GPU against the CPU oracle (FCMfunctions.cpp:175-880).

Tolerances: FP64 mode U/Omega within 1e-10 of the oracle relative to the
largest component; FP32 mode within 1e-5 of FP64.
"""
import numpy as np
import pytest
import torch

from filsim_b200 import abi
from filsim_b200.configs import make_mobility_case, params_for
from filsim_b200.fcm import Context, Fcm, mobility_host

pytestmark = pytest.mark.gpu

FP64_REL = 1e-10
FP32_REL = 1e-5


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return np.abs(a - b).max() / np.abs(b).max()


def gpu_mobility(p, Y, F, T, prec=abi.FS_PREC_FP64):
    ctx = Context(p, max_beads=max(1, Y.shape[0]))
    ctx.set_precision(prec)
    fcm = Fcm(ctx, Y.shape[0])
    fcm.set(Y, F, T)
    fcm.mobility_solve()
    ctx.synchronize()
    out = fcm.V.cpu().numpy(), fcm.W.cpu().numpy()
    ctx.close()
    return out


@pytest.fixture(scope="module")
def case64(gpu_lib):
    return make_mobility_case(64, 32, 15, seed=1000)


def test_mobility_64_fp64_matches_oracle(oracle, case64):
    p, s, Y, F, T = case64
    V0, W0 = oracle.fcm_mobility(p, Y, F, T)
    V, W = gpu_mobility(p, Y, F, T)
    assert rel_err(V, V0) < FP64_REL
    assert rel_err(W, W0) < FP64_REL


def test_mobility_golden_fixture(case64):
    g = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden", "mobility_64.npz"))
    p = params_for(64)
    V, W = gpu_mobility(p, g["Y"], g["F"], g["T"])
    assert rel_err(V, g["V"]) < FP64_REL
    assert rel_err(W, g["W"]) < FP64_REL


def test_spread_grid_matches_oracle(oracle):
    p, s, Y, F, T = make_mobility_case(32, 6, 5, seed=7)
    _, _, f0, _ = oracle.fcm_mobility(p, Y, F, T, return_grids=True)
    ctx = Context(p, max_beads=Y.shape[0])
    fcm = Fcm(ctx, Y.shape[0])
    fcm.set(Y, F, T)
    f = fcm.spread().cpu().numpy()
    assert np.abs(f - f0).max() / np.abs(f0).max() < 1e-13


FP32_SPREAD_REL = 1e-6


@pytest.mark.parametrize("shape,nb,seed,chunk,cols", [
    ((32, 32, 32), 40, 21, 32, 4),
    ((16, 32, 48), 30, 22, 32, 2),  # a 16-point axis: one bin, stencils wrap inside the tile
    ((48, 32, 16), 60, 23, 64, 8),
    ((32, 32, 32), 1500, 24, 32, 8),  # ~1500 candidates per tile: many staging chunks
    ((64, 32, 32), 1500, 25, 64, 2),
    ((64, 32, 32), 1500, 25, 64, 4),
])
def test_fp32_spread_grid_matches_oracle(oracle, shape, nb, seed, chunk, cols):
    """The FP32 chain's spread (k_spread_records32 + k_spread32: Kahan sums on packed
    pairs) against the oracle's FP64 force grid, positions drawn over 1.5 box lengths
    (negative and past the far face included), F, T ~ N(0,1), for both staging chunks
    and the three warp column blocks (2 x 16 x 8, 4 x 16 x 4, 8 x 16 x 2); a repeat is
    bitwise equal."""
    import ctypes
    from filsim_b200.abi import check, lib
    p = params_for(shape[0])
    p.npts_x, p.npts_y, p.npts_z = shape
    rng = np.random.default_rng(seed)
    L = np.array(shape) * p.dx
    Y = rng.uniform(-0.25, 1.25, (nb, 3)) * L
    F = rng.standard_normal((nb, 3))
    T = rng.standard_normal((nb, 3))
    _, _, f0, _ = oracle.fcm_mobility(p, Y, F, T, return_grids=True)
    ctx = Context(p, max_beads=nb)
    ctx.set_precision(abi.FS_PREC_FP32)
    tune = np.array([chunk, 8, 0, cols], np.int32)
    check(lib().fs_set_tuning(ctx.h, tune.ctypes.data_as(ctypes.c_void_p)), "fs_set_tuning")
    fcm = Fcm(ctx, nb)
    fcm.set(Y, F, T)
    f = fcm.spread().cpu().numpy()
    f2 = fcm.spread().cpu().numpy()
    ctx.close()
    assert rel_err(f, f0) < FP32_SPREAD_REL
    assert np.array_equal(f, f2)


def test_velocity_grid_matches_oracle(oracle):
    p, s, Y, F, T = make_mobility_case(32, 6, 5, seed=8)
    _, _, _, u0 = oracle.fcm_mobility(p, Y, F, T, return_grids=True)
    ctx = Context(p, max_beads=Y.shape[0])
    fcm = Fcm(ctx, Y.shape[0])
    fcm.set(Y, F, T)
    fcm.mobility_solve()
    u = fcm.velocity_grid()
    assert np.abs(u - u0).max() / np.abs(u0).max() < 1e-11


def test_sinusoidal_forcing_known_answer():
    """FCMfunctions.cpp:252-275: fz = sin(2 pi x / Nx) gives uz = fz / k^2 (mu = 1)."""
    p = params_for(32)
    N = 32
    f = np.zeros((3, N, N, N))
    f[2] = np.sin(2 * np.pi * np.arange(N) / N)[:, None, None]
    ctx = Context(p, max_beads=1)
    fcm = Fcm(ctx, 1)
    u = fcm.flow_solve(f).cpu().numpy()
    k = 2 * np.pi / (N * p.dx)
    assert np.abs(u[2] - f[2] / k ** 2).max() < 1e-12
    assert np.abs(u[:2]).max() < 1e-12


def numpy_flow_solve(p, f):
    """flow_solve (FCMfunctions.cpp:648-736) in numpy FP64: unnormalised transforms,
    norm = 1/(|q|^2 + 1e-18), u = norm (f - q (q.f) norm) / N, k = 0 zeroed, the
    Nyquist index taking +k; irfftn drops the imaginary parts of the kz = 0 and
    kz = Nz/2 coefficients as the reference's real inverse transform does."""
    nx, ny, nz = f.shape[1:]
    fh = np.fft.rfftn(f, axes=(1, 2, 3))

    def wn(n):
        i = np.arange(n)
        return np.where(i <= n // 2, i, i - n) * 2 * np.pi / (n * p.dx)

    q1 = wn(nx)[:, None, None]
    q2 = wn(ny)[None, :, None]
    q3 = (np.arange(nz // 2 + 1) * 2 * np.pi / (nz * p.dx))[None, None, :]
    qq = q2 * q2 + q1 * q1 + 1e-18
    norm = 1.0 / (qq + q3 * q3)
    kdotf = (q1 * fh[0] + q2 * fh[1] + q3 * fh[2]) * norm
    total = nx * ny * nz
    u = np.stack([norm * (fh[0] - q1 * kdotf), norm * (fh[1] - q2 * kdotf), norm * (fh[2] - q3 * kdotf)]) / total
    u[:, 0, 0, 0] = 0
    return np.fft.irfftn(u, s=(nx, ny, nz), axes=(1, 2, 3)) * total


def flow_input(kind, dims, seed):
    """White noise, or fields whose spectrum lies only in the kz = 0, kz = Nz/2 or
    kx = Nx/2 planes (the modes the real inverse transform treats specially)."""
    nx, ny, nz = dims
    rng = np.random.default_rng(seed)
    if kind == "noise":
        return rng.standard_normal((3, nx, ny, nz))
    if kind == "kz0":
        return np.repeat(rng.standard_normal((3, nx, ny, 1)), nz, axis=3)
    if kind == "kzN":
        return rng.standard_normal((3, nx, ny, 1)) * ((-1.0) ** np.arange(nz))[None, None, None, :]
    if kind == "kxN":
        return rng.standard_normal((3, 1, ny, nz)) * ((-1.0) ** np.arange(nx))[None, :, None, None]
    raise ValueError(kind)


def warp_fft_lengths_ok(dims):
    """Line lengths of the FP32 warp transform: 2^p up to 512 (z from 64) or 96, 192, 384."""
    ok = lambda n, lo: n >= lo and ((n & (n - 1)) == 0 and n <= 512 or n in (96, 192, 384))
    return ok(dims[0], 32) and ok(dims[1], 32) and ok(dims[2], 64)


@pytest.mark.parametrize("dims", [(64, 64, 64), (32, 128, 64), (128, 32, 256), (32, 32, 32),
                                  (512, 32, 64), (256, 64, 128), (64, 512, 64), (32, 64, 512),
                                  (96, 96, 96), (384, 32, 96), (32, 192, 384), (192, 96, 64), (64, 384, 192),
                                  (48, 48, 48)])
@pytest.mark.parametrize("kind", ["noise", "kz0", "kzN", "kxN"])
def test_flow_solve_fp64_and_fp32_against_numpy(dims, kind):
    """Grids whose line lengths are 2^p (z from 64) or 3 * 2^p >= 96 run the FP32
    five-pass transform (fs_fft.cu; its kernels show in the profile); 32^3 and 48^3
    run cuFFT. FP64 within 1e-12, FP32 within 1e-5 of the largest velocity
    component."""
    p = params_for(dims)
    f = flow_input(kind, dims, seed=sum(dims) + len(kind))
    ref = numpy_flow_solve(p, f)
    ctx = Context(p, max_beads=1)
    fcm = Fcm(ctx, 1)
    u64 = fcm.flow_solve(f).cpu().numpy()
    ctx.set_precision(abi.FS_PREC_FP32)
    ctx.profile_enable()
    u32 = fcm.flow_solve(f).cpu().numpy()
    prof = ctx.profile()
    ctx.close()
    assert rel_err(u64, ref) < 1e-12
    assert rel_err(u32, ref) < FP32_REL
    warp = warp_fft_lengths_ok(dims)
    for k in ("k_fft_z_fwd", "k_fft_y_fwd", "k_fft_y_inv", "k_fft_z_inv"):
        assert (prof[k][1] > 0) == warp, (k, prof[k])


def test_fp32_within_1e5_of_fp64(case64):
    p, s, Y, F, T = case64
    V64, W64 = gpu_mobility(p, Y, F, T)
    V32, W32 = gpu_mobility(p, Y, F, T, abi.FS_PREC_FP32)
    assert rel_err(V32, V64) < FP32_REL
    assert rel_err(W32, W64) < FP32_REL


def test_repeat_is_bitwise_identical(case64):
    p, s, Y, F, T = case64
    V1, W1 = gpu_mobility(p, Y, F, T)
    V2, W2 = gpu_mobility(p, Y, F, T)
    assert np.array_equal(V1, V2) and np.array_equal(W1, W2)


def test_host_entry_equals_device_entry(case64):
    p, s, Y, F, T = case64
    ctx = Context(p, max_beads=Y.shape[0])
    V, W = mobility_host(ctx, Y, F, T)
    Vd, Wd = gpu_mobility(p, Y, F, T)
    assert np.array_equal(V, Vd) and np.array_equal(W, Wd)


def test_negative_and_boundary_positions(oracle):
    """fmod leaves Y in (-L, L); (int)(Y/dx) truncates toward zero (FCMfunctions.cpp:565-567)."""
    p = params_for(32)
    L = 32 * p.dx
    rng = np.random.default_rng(3)
    Y = np.array([[-0.3 * p.dx, 0.2, 5.0], [-L + 0.01, L - 0.01, -2.5 * p.dx], [0.0, -1e-14, 3 * p.dx],
                  [L / 2, -L / 2, 7.25], [-4.0 * p.dx, 11.0, -0.5]])
    F = rng.standard_normal(Y.shape)
    T = rng.standard_normal(Y.shape)
    V0, W0 = oracle.fcm_mobility(p, Y, F, T)
    V, W = gpu_mobility(p, Y, F, T)
    assert rel_err(V, V0) < FP64_REL
    assert rel_err(W, W0) < FP64_REL


def test_friction_mobility(oracle, case64):
    p, s, Y, F, T = case64
    V0, W0 = oracle.fcm_friction(p, F, T)
    ctx = Context(p, max_beads=Y.shape[0])
    fcm = Fcm(ctx, Y.shape[0])
    fcm.set(Y, F, T)
    fcm.friction_mobility_solve()
    assert np.array_equal(fcm.V.cpu().numpy(), V0)
    assert np.array_equal(fcm.W.cpu().numpy(), W0)


def test_single_bead_self_mobility():
    """Periodic self-mobility approaches 1/(6 pi mu a) with Hasimoto's O(a/L) correction."""
    p = params_for(64)
    L = 64 * p.dx
    Y = np.array([[L / 2 + 0.1, L / 2 - 0.2, L / 2 + 0.3]])
    V, W = gpu_mobility(p, Y, np.array([[0, 0, 1.0]]), np.zeros((1, 3)))
    expect = 1 / (6 * np.pi) * (1 - 2.8373 / L)
    assert abs(V[0, 2] / expect - 1) < 1e-3
    V, W = gpu_mobility(p, Y, np.zeros((1, 3)), np.array([[0, 0, 1.0]]))
    assert abs(W[0, 2] * 8 * np.pi - 1) < 1e-3


def test_empty_call():
    p = params_for(32)
    ctx = Context(p, max_beads=4)
    fcm = Fcm(ctx, 0)
    fcm.mobility_solve()
    ctx.synchronize()


def test_too_many_beads_rejected():
    p = params_for(32)
    ctx = Context(p, max_beads=2)
    fcm = Fcm(ctx, 3)
    with pytest.raises(abi.FsError):
        fcm.mobility_solve()


@pytest.mark.parametrize("shape,nfil,nw,seed", [((32, 32, 32), 6, 3, 41), ((48, 32, 64), 8, 4, 42)])
def test_reference_default_stencil_ngd20(oracle, gpu_lib, shape, nfil, nw, seed):
    """The reference's own stencil: ngd = 20 points per axis with dx = sigma_dip / 1.5
    (config_template.hpp:76, multi_filament_header.hpp:48), where a stencil reaches
    three 16-point tiles per axis. FP64 within 1e-10 of the oracle, FP32 within 1e-5
    of FP64, including beads outside the box."""
    from filsim_b200.abi import make_params
    from filsim_b200.suspension import random_forces, random_suspension, fcm_positions
    p = make_params(shape, ngd=20)
    assert abs(p.dx - p.sigma_dip / 1.5) < 1e-15
    s = random_suspension(p, nfil, nw, seed, min_sep=1.5)
    F, T = random_forces(s.np, seed + 1)
    X = s.X.copy()
    X[::3] -= np.array(shape) * p.dx  # negative coordinates
    Y = fcm_positions(p, X)
    V0, W0 = oracle.fcm_mobility(p, Y, F, T)
    V, W = gpu_mobility(p, Y, F, T)
    assert rel_err(V, V0) < FP64_REL
    assert rel_err(W, W0) < FP64_REL
    V32, W32 = gpu_mobility(p, Y, F, T, abi.FS_PREC_FP32)
    assert rel_err(V32, V) < FP32_REL
    assert rel_err(W32, W) < FP32_REL


@pytest.mark.parametrize("ngd", [11, 13])
def test_odd_stencil_widths(oracle, gpu_lib, ngd):
    """Odd ngd (the stencil starts ngd/2 - 1 points below the bead's cell, as in
    gaussian_setup): FP64 within 1e-10 of the oracle and FP32 within 1e-5 of FP64,
    with several interpolation warps per CTA (each warp's tables keep their
    alignment for odd ngd^2)."""
    from filsim_b200.abi import make_params
    from filsim_b200.suspension import random_forces, random_suspension, fcm_positions
    p = make_params((32, 32, 48), ngd=ngd)
    s = random_suspension(p, 6, 3, 51, min_sep=1.5)
    F, T = random_forces(s.np, 52)
    Y = fcm_positions(p, s.X)
    V0, W0 = oracle.fcm_mobility(p, Y, F, T)
    V, W = gpu_mobility(p, Y, F, T)
    assert rel_err(V, V0) < FP64_REL
    assert rel_err(W, W0) < FP64_REL
    V32, W32 = gpu_mobility(p, Y, F, T, abi.FS_PREC_FP32)
    assert rel_err(V32, V) < FP32_REL
    assert rel_err(W32, W) < FP32_REL


def test_stencil_limits_are_checked(gpu_lib):
    """ngd above 20, or above a grid dimension, is rejected at context creation."""
    from filsim_b200.abi import FsError, make_params
    for shape, ngd in (((32, 32, 32), 21), ((16, 32, 32), 20)):
        with pytest.raises(FsError) as e:
            Context(make_params(shape, ngd=ngd), max_beads=4)
        assert e.value.status == abi.FS_ERR_INVALID_ARG
