"""Autotuner (fs_tune.cu): every launch variant it chooses among gives the FCM
solve within the FP32 tolerance (1e-5 of FP64); the choice is one of them. 64^3
and 96^3 have both transforms (warp FFT, cuFFT); 48^3 has cuFFT only."""
import ctypes

import numpy as np
import pytest

from filsim_b200 import abi
from filsim_b200.configs import make_sediment_case
from filsim_b200.fcm import Context, Simulation

pytestmark = pytest.mark.gpu


def _vp(a):
    return a.ctypes.data_as(ctypes.c_void_p)


@pytest.mark.parametrize("npts", [64, 48, 96])
def test_all_variants_and_autotune(gpu_lib, npts):
    p, s = make_sediment_case(npts, 12, 8, seed=77)
    ctx = Context(p, max_beads=s.np, max_filaments=s.nfil)
    sim = Simulation(ctx, s)
    sim.initial_guess()
    sim.filament_forces(2)
    ctx.set_precision(abi.FS_PREC_FP64)
    Y, F, T = (sim.device_array(k, (s.np, 3)) for k in ("Y", "F", "TAU"))
    from filsim_b200.fcm import Fcm
    fcm = Fcm(ctx, s.np)
    fcm.Y.copy_(Y)
    fcm.F.copy_(F)
    fcm.T.copy_(T)
    fcm.mobility_solve()
    V64, W64 = fcm.V.cpu().numpy(), fcm.W.cpu().numpy()
    ctx.set_precision(abi.FS_PREC_FP32)
    for ch in (32, 64):
        for wpb in (4, 8, 16):
            for fft in (0, 1):
                for cx in (2, 4, 8):
                    abi.check(abi.lib().fs_set_tuning(ctx.h, _vp(np.array([ch, wpb, fft, cx], np.int32))),
                              "fs_set_tuning")
                    fcm.mobility_solve()
                    V, W = fcm.V.cpu().numpy(), fcm.W.cpu().numpy()
                    assert np.abs(V - V64).max() / np.abs(V64).max() < 1e-5, (ch, wpb, fft, cx)
                    assert np.abs(W - W64).max() / np.abs(W64).max() < 1e-5, (ch, wpb, fft, cx)
    choice = np.zeros(4, np.int32)
    ms = ctypes.c_float()
    abi.check(abi.lib().fs_autotune(ctx.h, 2, _vp(choice), ctypes.byref(ms)), "fs_autotune")
    assert choice[0] in (32, 64) and choice[1] in (4, 8, 16) and choice[2] in (0, 1) and ms.value > 0
    assert choice[3] in (2, 4, 8)
    for bad in ([48, 8, 0, 4], [64, 8, 0, 3], [64, 8, 0, 16]):
        assert abi.lib().fs_set_tuning(ctx.h, _vp(np.array(bad, np.int32))) == abi.FS_ERR_INVALID_ARG
    ctx.close()
