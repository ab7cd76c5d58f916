"""The C++ mirror (include/filsim_gpu.hpp) driven on the GPU by a compiled C++
program, the form a FilSim main.cpp uses: one FcmGpu::mobility_solve_host
(Fcm::mobility_solve, FCMfunctions.cpp:175-464) and a SuspensionGpu running
implicit steps (main.cpp:284-754), each compared with the oracle; then the same
suspension stepped with the mixed-precision chain and the step options set
through the mirror (improved start, linear tensions, Broyden memory, velocity
predictor, precision escalation, captured steps), bitwise the same run driven
through the Python binding.

The program reads its inputs from a binary file the test writes (the fs_params
struct as the C compiler lays it out, then the arrays) and writes its outputs
to another."""
import os
import subprocess
import textwrap

import numpy as np
import pytest

from filsim_b200.configs import make_mobility_case, sediment_params
from filsim_b200.fcm import Context, Simulation
from filsim_b200.suspension import random_suspension

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

DRIVER = r"""
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "filsim_gpu.hpp"

template <typename T>
static void rd(FILE *f, T *p, size_t n) {
  if (fread(p, sizeof(T), n, f) != n) { std::fprintf(stderr, "short input\n"); std::exit(3); }
}

int main(int argc, char **argv) {
  FILE *in = std::fopen(argv[1], "rb");
  FILE *out = std::fopen(argv[2], "wb");
  // mobility case
  fs_params pm;
  rd(in, &pm, 1);
  int np = 0;
  rd(in, &np, 1);
  std::vector<double> Y(3 * np), F(3 * np), T(3 * np), V(3 * np), W(3 * np);
  rd(in, Y.data(), Y.size());
  rd(in, F.data(), F.size());
  rd(in, T.data(), T.size());
  // suspension case
  fs_params ps;
  rd(in, &ps, 1);
  int nfil = 0, ns = 0, nsteps = 0;
  rd(in, &nfil, 1);
  rd(in, &ns, 1);
  rd(in, &nsteps, 1);
  std::vector<int> fil_start(nfil + 1);
  rd(in, fil_start.data(), fil_start.size());
  std::vector<double> X(3 * ns), q(4 * ns), kap(nfil), c(nfil);
  rd(in, X.data(), X.size());
  rd(in, q.data(), q.size());
  rd(in, kap.data(), kap.size());
  rd(in, c.data(), c.size());
  fs_params po;
  int nsteps2 = 0;
  rd(in, &po, 1);
  rd(in, &nsteps2, 1);
  std::fclose(in);
  const std::vector<double> X0(X), q0(q);
  try {
    filsim::Context ctx(pm, np, 1);
    filsim::FcmGpu fcm(ctx, np);
    fcm.mobility_solve_host(Y.data(), F.data(), T.data(), V.data(), W.data());
    std::fwrite(V.data(), sizeof(double), V.size(), out);
    std::fwrite(W.data(), sizeof(double), W.size(), out);

    const int nl = ns - nfil;
    std::vector<double> Xs(X), Xt(X), U(3 * ns, 0.0), Us(U), Ut(U), Fb(U), TAU(U), qs(q), qt(q);
    std::vector<double> lam(3 * nl, 0.0), lam1(lam), lam2(lam);
    fs_host_state hs = {nfil, ns, fil_start.data(), X.data(), Xs.data(), Xt.data(), U.data(), Us.data(),
                        Ut.data(), q.data(), qs.data(), qt.data(), Fb.data(), TAU.data(), lam.data(),
                        lam1.data(), lam2.data(), kap.data(), c.data()};
    filsim::Context sctx(ps, ns, nfil);
    filsim::SuspensionGpu sus(sctx, hs);
    std::vector<int> its(nsteps);
    for (int k = 0; k < nsteps; ++k) its[k] = sus.stepImplicit(1 + k);
    sus.download(hs);
    std::fwrite(its.data(), sizeof(int), its.size(), out);
    std::fwrite(X.data(), sizeof(double), X.size(), out);
    std::fwrite(q.data(), sizeof(double), q.size(), out);

    // the step options, through the mirror, on the placed suspension again
    std::vector<double> X2(X0), q2(q0);
    std::vector<double> Xs2(X2), Xt2(X2), U2(3 * ns, 0.0), Us2(U2), Ut2(U2), F2(U2), T2(U2), qs2(q2), qt2(q2);
    std::vector<double> l0(3 * nl, 0.0), l1(l0), l2(l0);
    fs_host_state h2 = {nfil, ns, fil_start.data(), X2.data(), Xs2.data(), Xt2.data(), U2.data(), Us2.data(),
                        Ut2.data(), q2.data(), qs2.data(), qt2.data(), F2.data(), T2.data(), l0.data(),
                        l1.data(), l2.data(), kap.data(), c.data()};
    filsim::Context octx(po, ns, nfil);
    octx.set_precision(FS_PREC_FP32);
    octx.set_start_order(2);
    octx.set_tension_extrapolation(1);
    octx.set_broyden_memory(8, 3, 4, 12);
    octx.set_velocity_predictor(0.5);
    octx.set_precision_escalation(20);
    octx.set_graph_mode(true);
    filsim::SuspensionGpu sus2(octx, h2);
    std::vector<int> its2 = sus2.run(1, nsteps2);
    sus2.download(h2);
    std::fwrite(its2.data(), sizeof(int), its2.size(), out);
    std::fwrite(X2.data(), sizeof(double), X2.size(), out);
  } catch (const filsim::Error &e) {
    std::fprintf(stderr, "filsim error %d: %s\n", (int)e.status, e.what());
    return 2;
  }
  std::fclose(out);
  return 0;
}
"""


def test_cpp_mirror_runs_mobility_and_steps_on_the_gpu(oracle, gpu_lib, tmp_path):
    from filsim_b200 import abi
    src = tmp_path / "drv.cpp"
    src.write_text(textwrap.dedent(DRIVER))
    exe = tmp_path / "drv"
    libdir = os.path.dirname(abi.LIB_PATH)
    subprocess.run(["g++", "-std=c++14", "-O1", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L" + libdir, "-lfilsim_gpu", "-Wl,-rpath," + libdir], check=True)
    pm, s, Y, F, T = make_mobility_case(64, 32, 15, seed=1000)
    ps = sediment_params(32, tol=1e-10, broyden_maxiter=200)
    sus = random_suspension(ps, 6, 8, seed=31, kap=1.0, c=1.0)
    sus0 = sus.copy()  # the placed state, for the run with the step options
    nsteps = 4
    po = sediment_params(32, tol=1e-6, broyden_maxiter=200)  # the same box at the benchmark's tolerance
    nsteps2 = 24
    with open(tmp_path / "in.bin", "wb") as f:
        f.write(bytes(pm))
        f.write(np.int32(s.np).tobytes())
        for a in (Y, F, T):
            f.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())
        f.write(bytes(ps))
        f.write(np.array([sus.nfil, sus.np, nsteps], dtype=np.int32).tobytes())
        f.write(sus.fil_start.astype(np.int32).tobytes())
        for a in (sus.X, sus.q, sus.kap, sus.c):
            f.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())
        f.write(bytes(po))
        f.write(np.int32(nsteps2).tobytes())
    r = subprocess.run([str(exe), str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    raw = open(tmp_path / "out.bin", "rb").read()
    n3 = 3 * s.np
    V = np.frombuffer(raw, np.float64, n3, 0).reshape(-1, 3)
    W = np.frombuffer(raw, np.float64, n3, 8 * n3).reshape(-1, 3)
    off = 16 * n3
    its = np.frombuffer(raw, np.int32, nsteps, off)
    off += 4 * nsteps
    X = np.frombuffer(raw, np.float64, 3 * sus.np, off).reshape(-1, 3)
    q = np.frombuffer(raw, np.float64, 4 * sus.np, off + 24 * sus.np).reshape(-1, 4)
    off += 56 * sus.np
    its2 = np.frombuffer(raw, np.int32, nsteps2, off)
    X2 = np.frombuffer(raw, np.float64, 3 * sus.np, off + 4 * nsteps2).reshape(-1, 3)
    assert len(raw) == off + 4 * nsteps2 + 24 * sus.np

    V0, W0 = oracle.fcm_mobility(pm, Y, F, T)
    assert np.abs(V - V0).max() / np.abs(V0).max() < 1e-10
    assert np.abs(W - W0).max() / np.abs(W0).max() < 1e-10

    sysw = oracle.System(ps, sus)
    its0, st0 = sysw.run_steps(1, nsteps)
    o = sysw.download()
    assert st0 == 0
    assert np.array_equal(its, its0)
    assert np.abs(X - o["X"]).max() / (32 * ps.dx) < 1e-8
    assert np.abs(q - o["q"]).max() < 1e-8

    # the options run through the Python binding: bitwise the mirror's run
    ctx = Context(po, max_beads=sus.np, max_filaments=sus.nfil)
    ctx.set_precision(abi.FS_PREC_FP32)
    ctx.set_start_order(2)
    ctx.set_tension_extrapolation(1)
    ctx.set_broyden_memory(8, 3, 4, 12)
    ctx.set_velocity_predictor(0.5)
    ctx.set_precision_escalation(20)
    abi.check(abi.lib().fs_set_graph_mode(ctx.h, 1), "fs_set_graph_mode")
    sim = Simulation(ctx, sus0.copy())
    its_p, st_p = sim.run_steps(1, nsteps2)
    X_p = sim.download()["X"]
    ctx.close()
    assert st_p == abi.FS_OK
    assert np.array_equal(its2, its_p)
    assert np.array_equal(X2, X_p)
