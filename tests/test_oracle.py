"""The CPU oracle against analytic known answers, numpy.fft and its own
committed fixtures (CPU only)."""
import os

import numpy as np
import pytest

from filsim_b200.abi import box_lengths
from filsim_b200.configs import make_mobility_case, params_for, sediment_params
from filsim_b200.suspension import fcm_positions, random_suspension

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("shape", [(8, 6, 10), (16, 12, 9), (12, 8, 16), (48, 8, 4)])
def test_fft_matches_numpy(oracle, shape):
    x = np.random.default_rng(0).standard_normal(shape)
    xh = oracle.fft_r2c_3d(x)
    ref = np.fft.rfftn(x)
    assert np.abs(xh - ref).max() < 1e-12 * np.abs(ref).max()
    back = oracle.fft_c2r_3d(xh, shape[2]) / np.prod(shape)
    assert np.abs(back - x).max() < 1e-13


def test_c2r_ignores_imaginary_dc_and_nyquist(oracle):
    """FFTW's halfcomplex inverse keeps only the real parts of the last axis's
    DC and Nyquist coefficients after the other axes' complex transforms."""
    rng = np.random.default_rng(1)
    xh = rng.standard_normal((6, 4, 5)) + 1j * rng.standard_normal((6, 4, 5))
    out = oracle.fft_c2r_3d(xh, 8)
    g = np.fft.ifft(np.fft.ifft(xh, axis=0), axis=1) * 24  # complex along x, y (unnormalised)
    full = np.zeros((6, 4, 8), dtype=complex)
    full[:, :, 0] = g[:, :, 0].real
    full[:, :, 4] = g[:, :, 4].real
    full[:, :, 1:4] = g[:, :, 1:4]
    full[:, :, 5:8] = np.conj(g[:, :, 3:0:-1])
    ref = (np.fft.ifft(full, axis=2) * 8).real
    assert np.abs(out - ref).max() < 1e-12


def test_sinusoidal_forcing_known_answer(oracle):
    """FCMfunctions.cpp:252-275: fz = sin(2 pi x / Nx) gives uz = fz / k^2."""
    p = params_for(32)
    f = np.zeros((3, 32, 32, 32))
    f[2] = np.sin(2 * np.pi * np.arange(32) / 32)[:, None, None]
    u = oracle.flow_solve(p, f)
    k = 2 * np.pi / box_lengths(p)[0]
    assert np.abs(u[2] - f[2] / k ** 2).max() < 1e-13
    assert np.abs(u[:2]).max() < 1e-13


def test_friction_known_answer(oracle):
    p = params_for(32)
    F = np.array([[1.0, -2.0, 3.0]])
    T = np.array([[0.5, 0.0, -1.0]])
    V, W = oracle.fcm_friction(p, F, T)
    assert np.allclose(V, F / (6 * np.pi), rtol=1e-15)
    assert np.allclose(W, T / (8 * np.pi), rtol=1e-15)


@pytest.mark.parametrize("npts", [32, 64])
def test_single_bead_self_mobility(oracle, npts):
    """Periodic FCM self-mobility: 1/(6 pi mu a) (1 - 2.8373 a/L) (Hasimoto)."""
    p = params_for(npts)
    L = box_lengths(p)[0]
    Y = np.array([[L / 2 + 0.1, L / 2 - 0.2, L / 2 + 0.3]])
    V, _ = oracle.fcm_mobility(p, Y, np.array([[0, 0, 1.0]]), np.zeros((1, 3)))
    assert abs(V[0, 2] / (1 / (6 * np.pi) * (1 - 2.8373 / L)) - 1) < 2e-3
    _, W = oracle.fcm_mobility(p, Y, np.zeros((1, 3)), np.array([[0, 0, 1.0]]))
    assert abs(W[0, 2] * 8 * np.pi - 1) < 2e-3


def test_pair_mobility_far_field(oracle):
    """Two well-separated beads: the change of the cross mobility between
    separations 6a and 10a follows the Oseen tensor of FCMStokeslet
    (FCMfunctions.cpp:811-863); the periodic images add a nearly constant
    offset that cancels in the difference."""
    p = params_for(64)
    L = box_lengths(p)[0]
    cross = []
    for r in (6.0, 10.0):
        Y = np.array([[L / 2 - r / 2, L / 2, L / 2], [L / 2 + r / 2, L / 2, L / 2]])
        F = np.array([[0.0, 0.0, 1.0], [0.0, 0.0, 0.0]])
        V, _ = oracle.fcm_mobility(p, Y, F, np.zeros((2, 3)))
        cross.append(V[1, 2])
    d_oseen = 1 / (8 * np.pi) * (1 / 6.0 - 1 / 10.0)
    assert abs((cross[0] - cross[1]) - d_oseen) < 0.05 * d_oseen


def test_mobility_is_symmetric(oracle):
    """The FCM mobility operator is symmetric: F2 . M F1 = F1 . M F2."""
    p, s, Y, F1, T1 = make_mobility_case(32, 4, 5, seed=3)
    rng = np.random.default_rng(9)
    F2, T2 = rng.standard_normal(F1.shape), rng.standard_normal(T1.shape)
    V1, W1 = oracle.fcm_mobility(p, Y, F1, T1)
    V2, W2 = oracle.fcm_mobility(p, Y, F2, T2)
    a = np.sum(F2 * V1) + np.sum(T2 * W1)
    b = np.sum(F1 * V2) + np.sum(T1 * W2)
    assert abs(a - b) < 1e-9 * abs(a)


def test_mobility_golden(oracle):
    g = np.load(os.path.join(GOLD, "mobility_64.npz"))
    V, W = oracle.fcm_mobility(params_for(64), g["Y"], g["F"], g["T"])
    assert np.abs(V - g["V"]).max() < 1e-13 * np.abs(g["V"]).max()
    assert np.abs(W - g["W"]).max() < 1e-13 * np.abs(g["W"]).max()


def test_barrier_golden_and_properties(oracle):
    g = np.load(os.path.join(GOLD, "barrier_dense.npz"))
    p = params_for(32)
    head, lst, mp = oracle.cells_link(p, g["X"])
    assert np.array_equal(head, g["head"]) and np.array_equal(lst, g["list"])
    Y = fcm_positions(p, g["X"])
    r = oracle.collision_barrier(p, Y, g["F0"], g["fil_id"], g["seg_id"], head, lst, mp, 5, max_pairs=1 << 16)
    assert np.array_equal(r["pairs"], g["pairs"])
    assert np.array_equal(r["F"], g["F"])
    assert r["min_dist2"] == float(g["min_dist2"])
    # equal and opposite forces
    assert abs((r["F"] - g["F0"]).sum(axis=0)).max() < 1e-9
    # the cell search finds every pair a brute-force minimum-image search finds
    L = np.array(box_lengths(p))
    d = Y[:, None, :] - Y[None, :, :]
    d -= L * np.floor(d / L + 0.5)
    r2 = (d * d).sum(-1)
    fid, sid = g["fil_id"], g["seg_id"]
    adj = (fid[:, None] == fid[None, :]) & (np.abs(sid[:, None] - sid[None, :]) == 1)
    i, j = np.nonzero(np.triu(r2 < 1.21 * 4.0, 1) & ~adj)
    brute = {(a, b) for a, b in zip(i, j)}
    found = {tuple(sorted(x)) for x in r["pairs"].tolist()}
    assert brute == found


def test_steps_golden(oracle):
    g = np.load(os.path.join(GOLD, "steps_small.npz"))
    p = sediment_params(32, tol=1e-10, broyden_maxiter=100)
    s = random_suspension(p, 6, 8, seed=31)
    assert np.array_equal(s.X, g["X0"])
    sysw = oracle.System(p, s)
    its, st = sysw.run_steps(1, 10)
    out = sysw.download()
    assert np.array_equal(its, g["iters"])
    assert np.abs(out["X"] - g["X"]).max() < 1e-10
    assert np.abs(out["q"] - g["q"]).max() < 1e-10


def test_steps_keep_bead_spacing(oracle):
    """unRobotArmify rebuilds positions from tangents: consecutive beads stay
    dl apart to rounding (Filament.hpp:489-505)."""
    p = sediment_params(32)
    s = random_suspension(p, 4, 8, seed=40)
    sysw = oracle.System(p, s)
    its, st = sysw.run_steps(1, 4)
    X = sysw.download()["X"].reshape(4, 8, 3)
    d = np.linalg.norm(np.diff(X, axis=1), axis=2)
    assert np.abs(d - p.dl).max() < 1e-4  # midpoint-tangent chords, not exact arcs
    assert its.max() < 300 and st == 0


def test_suspension_rejection_rule():
    p = params_for(64)
    s = random_suspension(p, 32, 15, 1000)
    L = np.array(box_lengths(p))
    d = s.X[:, None, :] - s.X[None, :, :]
    d -= L * np.floor(d / L + 0.5)
    r2 = (d * d).sum(-1)
    fid = s.fil_id
    other = fid[:, None] != fid[None, :]
    assert r2[other].min() >= (2.2 - 1e-9) ** 2


@pytest.mark.parametrize("npts,nfil,nw,seed,sep", [(64, 32, 15, 1000, 2.2), (32, 40, 6, 11, 1.2),
                                                    ((96, 64, 48), 20, 16, 7, 2.2)])
def test_cpu_generator_reproduces_the_library_bit_for_bit(oracle, npts, nfil, nw, seed, sep):
    """The CPU baseline builds its inputs with the oracle's restatement of the
    generator (no GPU library); both must give the same bits. The library's
    generator is host code, so this runs without a GPU."""
    p = params_for(npts)
    s = random_suspension(p, nfil, nw, seed, min_sep=sep)
    X, Q = oracle.suspension_random(p, nfil, nw, seed, min_sep=sep)
    assert np.array_equal(X, s.X)
    assert np.array_equal(Q, s.q)


def test_cpu_generator_at_the_512_cube_benchmark(oracle):
    """The 512^3 / 4096 x 32 benchmark suspension (seed 1002) from both generators."""
    from filsim_b200.configs import make_sediment_case
    p, s = make_sediment_case(512, 4096, 32, seed=1002)
    X, Q = oracle.suspension_random(p, 4096, 32, 1002)
    assert np.array_equal(X, s.X)
    assert np.array_equal(Q, s.q)


def _link_twist_norms(tau, nw):
    """Per-link torque magnitudes |w_i| of a filament whose beads receive
    +w_i (bead i) and -w_i (bead i+1): w_i is the prefix sum of the torques."""
    w = np.cumsum(tau[: nw - 1], axis=0)
    return np.linalg.norm(w, axis=1)


@pytest.mark.parametrize("sperm_decay", [False, True])
def test_swimming_drive_strain_twist(oracle, sperm_decay):
    """applyElasticTorques with the swimming drive (Filament.hpp:297-326) on
    straight filaments (q equal along each filament, lambda = 0): the elastic
    term vanishes, so link i carries the rotated (-C st0, -K st1, -K st2) with
    st1 = Beta facPref cos(k s - w t + phase), st2 = Alpha facPref sin(...)."""
    from filsim_b200.suspension import swim_parameters
    p = sediment_params(32)
    nfil, nw, nt = 3, 8, 7
    kap = np.array([0.7, 1.0, 1.6])
    s = random_suspension(p, nfil, nw, seed=61, kap=kap, c=1.0)
    sysw = oracle.System(p, s)
    swim = swim_parameters(s.fil_start, p, K0=1.0, Sp4=12.0, alpha=[0.3, 0.0, 1.1], beta=[1.0, 0.5, 0.0],
                           phase=[0.2, -1.0, 2.0], kap=kap)
    curvature = 8.25
    sysw.set_swimming(swim, curvature=curvature, sperm_decay=sperm_decay)
    sysw.filament_forces(nt)
    tau = sysw.download()["TAU"].reshape(nfil, nw, 3)
    F_swim = sysw.download()["F"]
    sysw.set_swimming(None)
    sysw.filament_forces(nt)
    assert np.array_equal(sysw.download()["F"], F_swim)  # the drive acts on torques only
    tt = nt * p.dt
    L, Llong = (nw - 1) * p.dl, nw * p.dl
    T0 = curvature / Llong
    for f in range(nfil):
        sarc = p.dl * np.arange(nw - 1) + 0.5 * p.dl
        if sperm_decay:
            fac = np.where(sarc > L / 2.0, T0 * 2.0 * (L - sarc) / L, T0)
        else:
            fac = T0 * (L - sarc) / L
        arg = swim[f, 3] * sarc - swim[f, 4] * tt + swim[f, 2]
        st1 = swim[f, 1] * fac * np.cos(arg)
        st2 = swim[f, 0] * fac * np.sin(arg)
        want = kap[f] * np.sqrt(st1 ** 2 + st2 ** 2)
        got = _link_twist_norms(tau[f], nw)
        assert np.allclose(got, want, rtol=1e-12, atol=1e-14), f


def test_spring_links_forces(oracle):
    """apply_spring_link_forces (spring_link_functions.cpp:24-45): the change of
    F from the links is -k (|d| - l0) d/|d| on the first bead and the opposite on
    the second, d the minimum-image displacement; links sharing a bead add up."""
    p = sediment_params(32)
    s = random_suspension(p, 3, 8, seed=62)
    sysw = oracle.System(p, s)
    nt = 5
    sysw.filament_forces(nt)
    F0 = sysw.download()["F"].copy()
    Xs = sysw.download()["Xs"]
    links = np.array([[0, 9], [9, 20], [3, 23]])
    k, l0 = 2.5, 3.0
    sysw.set_spring_links(links, k, l0)
    sysw.filament_forces(nt)
    F1 = sysw.download()["F"]
    Lb = np.array(box_lengths(p))
    want = np.zeros_like(F0)
    for a, b in links:
        d = Xs[a] - Xs[b]
        d = d - Lb * np.floor(d / Lb + 0.5)
        sf = -k * (np.linalg.norm(d) - l0) * d / np.linalg.norm(d)
        want[a] += sf
        want[b] -= sf
    assert np.abs((F1 - F0) - want).max() < 1e-12 * max(1.0, np.abs(want).max())


def _dense_case(seed):
    """A crowded box: filaments placed 2.0a apart, inside the barrier's 2.2a range."""
    p = sediment_params(32, tol=1e-10, broyden_maxiter=100)
    s = random_suspension(p, 10, 8, seed=seed, min_sep=2.0)
    return p, s


def test_barrier_modes_on_the_oracle(oracle):
    """The barrier variants differ only by their pair filter: without contacts
    between filament 0 and the others the not-swimmer barrier gives the plain
    trajectory bitwise; switching the barrier off changes a crowded run."""
    from filsim_b200 import abi
    p, s = _dense_case(91)
    runs = {}
    for mode in (abi.FS_BARRIER_ALL, abi.FS_BARRIER_NOT_SWIMMER, abi.FS_BARRIER_NOT_TEST_PARTICLES,
                 abi.FS_BARRIER_OFF):
        sysw = oracle.System(p, s)
        sysw.set_barrier_mode(mode)
        its, st = sysw.run_steps(1, 4)
        runs[mode] = sysw.download()["X"]
    assert not np.array_equal(runs[abi.FS_BARRIER_ALL], runs[abi.FS_BARRIER_OFF])
    # a filament far from every other: the swimmer filter changes nothing
    p2 = sediment_params(32, tol=1e-10, broyden_maxiter=100)
    s2 = random_suspension(p2, 2, 8, seed=92)
    a, b = oracle.System(p2, s2), oracle.System(p2, s2)
    b.set_barrier_mode(abi.FS_BARRIER_NOT_SWIMMER)
    a.run_steps(1, 3)
    b.run_steps(1, 3)
    assert np.array_equal(a.download()["X"], b.download()["X"])


def test_gait_reset_step_on_the_oracle(oracle):
    """main_gaitreset.cpp:302-830: the committed state advances once per step
    (the trial solves leave X, U, q alone) and the last solve is a full barrier
    solve from the trial solves' lambda."""
    p, s = _dense_case(93)
    g = oracle.System(p, s)
    g.run_steps(1, 2)
    before = g.download()
    its, vwf, st = g.step_gait_reset(3)
    after = g.download()
    assert its.min() >= 1 and vwf.shape == (3, 8, 9)
    assert np.array_equal(after["Xt"], before["X"])  # one Filament::step
    assert not np.array_equal(vwf[0], vwf[2])        # the three solves differ
