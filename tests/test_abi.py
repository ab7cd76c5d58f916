"""The C-ABI boundary without a GPU: the library builds, loads and exports every
symbol include/filsim_gpu.h declares, and the ctypes mirrors match the C
struct layouts. No compute calls are made here."""
import ctypes
import os
import subprocess
import textwrap

import pytest

from filsim_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def libpath():
    from filsim_b200 import build as fbuild
    return fbuild.build()


def test_library_exports_every_header_symbol(libpath):
    L = ctypes.CDLL(libpath)
    names = abi.header_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_no_device_status_without_gpu(libpath):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    L = abi.lib()
    p = abi.make_params(32)
    h = ctypes.c_void_p()
    assert L.fs_create(ctypes.byref(p), 10, 2, None, ctypes.byref(h)) == 2  # FS_ERR_NO_DEVICE
    assert L.fs_status_string(2) == b"no sm_100 CUDA device"
    assert L.fs_abi_version() == 2


def test_params_default_matches_reference_constants(libpath):
    L = abi.lib()
    p = abi.FsParams()
    L.fs_params_default(ctypes.byref(p), 64, 64, 64)
    q = abi.make_params(64)
    for f, _ in abi.FsParams._fields_:
        a, b = getattr(p, f), getattr(q, f)
        if hasattr(a, "__len__"):
            assert list(a) == list(b), f
        else:
            assert a == b or abs(a - b) < 1e-15 * abs(b), f
    # multi_filament_header.hpp:47-48,57
    assert abs(p.sigma_dip - 1 / (36 * abi.PI) ** (1 / 6)) < 1e-15
    assert abs(p.dx - p.sigma_dip / 1.5) < 1e-15


def test_struct_layouts_match_c(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(textwrap.dedent("""
        #include <stdio.h>
        #include <stddef.h>
        #include "filsim_gpu.h"
        int main(void) {
          printf("%zu %zu %zu\\n", sizeof(fs_params), sizeof(fs_diag), sizeof(fs_host_state));
          printf("%zu %zu %zu %zu\\n", offsetof(fs_params, tol), offsetof(fs_params, barrier_fs_over_2a),
                 offsetof(fs_params, lambda_extrap_step), offsetof(fs_diag, min_dist2));
          printf("%zu %zu\\n", offsetof(fs_host_state, lam), offsetof(fs_host_state, c));
          printf("%zu %zu %zu %zu %zu\\n", sizeof(fs_run_info), offsetof(fs_run_info, a),
                 offsetof(fs_run_info, box), offsetof(fs_run_info, dt),
                 offsetof(fs_run_info, network_spring_natural_length));
          return 0;
        }
    """))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    vals = [int(v) for v in out]
    P, D, H = abi.FsParams, abi.FsDiag, abi.FsHostState
    assert vals[:3] == [ctypes.sizeof(P), ctypes.sizeof(D), ctypes.sizeof(H)]
    assert vals[3] == P.tol.offset and vals[4] == P.barrier_fs_over_2a.offset
    assert vals[5] == P.lambda_extrap_step.offset and vals[6] == D.min_dist2.offset
    assert vals[7] == H.lam.offset and vals[8] == H.c.offset
    R = abi.FsRunInfo
    assert vals[9:] == [ctypes.sizeof(R), R.a.offset, R.box.offset, R.dt.offset,
                        R.network_spring_natural_length.offset]


def test_sources_have_no_cpu_fallback():
    """The product path never reaches the oracle."""
    pkg = os.path.join(ROOT, "filsim_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh")):
                text = open(os.path.join(dirpath, f)).read()
                assert "oracle" not in text.replace("the oracle", ""), f


def test_cpp_mirror_header_compiles_and_links(libpath, tmp_path):
    """include/filsim_gpu.hpp builds against the library; without a GPU the
    context constructor reports FS_ERR_NO_DEVICE through filsim::Error."""
    src = tmp_path / "drv.cpp"
    src.write_text(textwrap.dedent("""
        #include <cstdio>
        #include "filsim_gpu.hpp"
        int main() {
          fs_params p;
          fs_params_default(&p, 32, 32, 32);
          try {
            filsim::Context ctx(p, 8, 2);
            filsim::FcmGpu fcm(ctx, 8);
            filsim::LinkedListGpu ll(ctx);
            std::printf("context %d %d %d\\n", ll.cells()[0], ll.cells()[1], ll.cells()[2]);
            // the swimming, spring-link, barrier-mode and gait-reset wrappers compile and link
            // (taken by address, not run)
            auto sw = &filsim::SuspensionGpu::setSwimming;
            auto sl = &filsim::SuspensionGpu::setSpringLinks;
            auto bm = &filsim::SuspensionGpu::setBarrierMode;
            auto gr = &filsim::SuspensionGpu::stepGaitReset;
            std::printf("wrappers %d\\n", (sw != nullptr) + (sl != nullptr) + (bm != nullptr) + (gr != nullptr));
          } catch (const filsim::Error &e) {
            std::printf("error %d\\n", e.status);
          }
          return 0;
        }
    """))
    exe = tmp_path / "drv"
    libdir = os.path.dirname(libpath)
    subprocess.run(["g++", "-std=c++14", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L" + libdir, "-lfilsim_gpu", "-Wl,-rpath," + libdir], check=True)
    import torch
    if not torch.cuda.is_available():
        out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
        assert out.strip() == "error 2"
