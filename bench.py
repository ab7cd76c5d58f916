#!/usr/bin/env python
"""Benchmark: implicit BDF2 time steps of sedimenting elastic filaments.

Workload sediment_512: 512^3 periodic FCM grid, 4096 filaments x 32 beads
(131,072 beads) placed by seeded rejection sampling, gravity (0,0,-1) per bead,
K_B = K_T = 1, dt = 0.05, Broyden tolerance 1e-6 (the reference's absolute
max-norm test), barrier below 2.2a. One "step" is one implicit time step
(main.cpp:284-754): initial guess, forces, Jacobian build, cell link, then
Broyden iterations each with a collision barrier and an FCM mobility solve,
until converged. The metric is bead-steps per second.

The suspension first runs 12 untimed start-up steps (implicit Euler, then the
constant and linear tension extrapolation); W warm-up and K timed steps follow
in the steady BDF2 regime with the quadratic extrapolation, the regime of 188 of
the 200 steps of the configured run. Every arm starts from that same state.

value      mixed precision (FP32 spread/FFT/interpolation, FP64 Broyden and
           filament mechanics); each step starts with the first bead of every
           filament at 3X - 3Xt + Xtt (fs_set_start_order 2; the reference's start
           takes 2X - Xt, a first-order extrapolation of the position that carries
           the whole filament) and the tensions at 2 lam - lam1
           (fs_set_tension_extrapolation 1; the reference's quadratic
           extrapolation amplifies the converged tensions' tolerance noise); on top
           of that start, the learned warm start
           (trained untimed before the run by the library's own kernels on 20
           seeded runs of this workload with the same start, K_B log-uniform in
           [0.1, 10]) under its cost gate (fs_warm_start_gate, period 8: each step
           takes the start with the lower running mean of mobility solves per
           step, the learned one only when it saves at least 0.25 solves per step
           over at least two of its steps, and probes the other one after 8 steps,
           an interval that doubles up to 128 while the probes lose; steps without
           the learned start run as captured step graphs; learned.gate reports how
           many timed steps took each); a learned step compares both starts only
           every 8th learned step and in between checks each filament's learned
           start against the carried residual (fs_warm_start_bound). The Broyden
           loop and its convergence test (max |Err| <= 1e-6) are the reference's.
           Inputs resident in HBM, device-timed with CUDA events on the context's
           stream, max over ranks; weak scaling (one independent replica per GPU).
learned_every_step the same steps with the learned start on every step.
fp32_improved_start the same steps with that start alone (no learned start).
fp32_plain_start   the same steps from the reference's start (2X - Xt).
plain_fp64 the same steps with the FCM chain in FP64 and the reference's start.
e2e        the value arm through the C-ABI with HOST state: every step uploads
           the suspension's state from pinned host memory (fs_state_upload), steps,
           and downloads it (fs_state_download); the state is what the reference
           checkpoints (X, Xt, q, qt, U, Ut, lam, lam1, lam2) plus K_B and C.
--impl reference times the CPU restatement of the reference (the reference
           itself, MPI + FFTW 2.1.5 + Armadillo, cannot be built here) on this
           host's cores, without the GPU library: the inputs come from the
           restated generator in oracle/, and each of its steps is one full-size
           stage of a Broyden iteration (see run_reference).

Grids (3 x 512^3 reals + 3 x 512^2 x 257 complex, several GB) exceed the 126 MB
L2, so no flush is needed between steps.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "bead-steps/s & Broyden iters/step: learned+FP32 vs plain FP64 GPU, resid<=1e-6"
UNIT = "bead-steps/s"
WORKLOAD = dict(npts=512, nfil=4096, nw=32, seed=1002, name="sediment_512")
# untimed start-up steps before the measured window (the tension extrapolation
# becomes quadratic after step 12, Filament::step, Filament.hpp:455-478)
PREP_STEPS = 12
# warm-start training data: seeds TRAIN_SEED0.. of this workload, K_B log-uniform in [0.1, 10]
TRAIN_SEED0 = 7000
TRAIN_EPOCHS = 40
CHECKPOINT_FIELDS = ("X", "Xt", "q", "qt", "U", "Ut", "lam", "lam1", "lam2", "kap", "c")
GATE_PERIOD = 8  # the learned start's cost gate: first probe of the other start after 8 steps
BOUND_REFRESH = 8  # learned steps between comparisons with the plain start (fs_warm_start_bound)
ENSEMBLE_SEED = 3000
# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the FCM
# kernels, per grid point: the mean over the launches of each in one timed step of
# each FP32 arm of the 512^3 workload under ncu (a one-pass metric set).
NCU_TRAFFIC_PER_POINT = {
    "k_spread": (93.28e6 + 1553.20e6) / 512 ** 3,
    "k_fft_z_fwd": (1610.70e6 + 1564.94e6) / 512 ** 3,
    "k_fft_y_fwd": (1616.96e6 + 1565.83e6) / 512 ** 3,
    "project": (1617.05e6 + 1553.13e6) / 512 ** 3,
    "k_fft_y_inv": (1617.06e6 + 1565.69e6) / 512 ** 3,
    "k_fft_z_inv": (1617.00e6 + 1562.84e6) / 512 ** 3,
    "k_interp": (1557.31e6 + 6.21e6) / 512 ** 3,
}
NCU_TRAFFIC_SOURCE = "ncu capture of one timed step of each FP32 arm at 512^3 (17 launches per kernel), per grid point"


def start_label(start, tension):
    """The config's description of a step start (fs_set_start_order, fs_set_tension_extrapolation)."""
    pos = "first bead from 3X - 3Xt + Xtt" if start == 2 else "first bead from 2X - Xt (the reference's)"
    ten = "tensions 2 lam - lam1" if tension == 1 else "tensions 3 lam - 3 lam1 + lam2 (the reference's)"
    return "%s; %s after lambda_extrap_step" % (pos, ten)


# Broyden memory across steps (fs_set_broyden_memory): keep J0 and up to 16 history
# columns after a step of fewer than 8 iterations, carry the last 4 columns after a
# longer one, restart a step on carried state at 30 iterations
MEMORY_DEFAULT = (16, 4, 8, 30)
MEMORY_OFF = (0, 0, 0, 0)
# velocity predictor (fs_set_velocity_predictor): half the update predicted from
# the extrapolated velocities
PREDICTOR_DEFAULT = 0.5


def memory_label(mem):
    """The config's description of the Broyden memory (fs_set_broyden_memory)."""
    if tuple(mem) == MEMORY_OFF:
        return "off (the reference's iteration: J0 rebuilt and the history emptied every step)"
    k, c, t, r = mem
    return ("J0 and up to %d history columns kept after a step of fewer than %d iterations; the last %d columns "
            "carried beside a new J0 after a longer one; restart at %d iterations" % (k, t, c, r))


def warp_fft_length(n):
    """Grid lengths the FP32 warp transform covers on every axis (fs_fft.cu): 2^p in
    [64, 512] or 96, 192, 384; other grids run cuFFT."""
    return (64 <= n <= 512 and n & (n - 1) == 0) or n in (96, 192, 384)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip training; time the reference's start only")
    ap.add_argument("--no-graph", action="store_true", help="host-driven steps only (no CUDA graphs)")
    ap.add_argument("--start-order", type=int, default=2, choices=[1, 2],
                    help="start of the value arm's steps (fs_set_start_order): 2 the first bead from "
                         "3X - 3Xt + Xtt (default), 1 the reference's 2X - Xt; the plain arms always use 1")
    ap.add_argument("--tension-order", type=int, default=1, choices=[1, 2],
                    help="tension start of the value arm's steps (fs_set_tension_extrapolation): 1 linear "
                         "(default), 2 the reference's quadratic; the plain arms always use 2")
    ap.add_argument("--escalate", type=int, default=0,
                    help="fs_set_precision_escalation for the value arm and the ensemble: FP32 steps still not "
                         "converged after this many Broyden iterations finish in FP64 (0: off, the default; "
                         "trajectory_200 runs it beside the plain runs, at 15 unless given)")
    ap.add_argument("--broyden-memory", default=":".join(map(str, MEMORY_DEFAULT)),
                    help="fs_set_broyden_memory for the value arm and the ensemble, KEEP:CARRY:THRESHOLD:RESTART "
                         "(default %s); 0 turns it off (the reference's iteration)" % ":".join(map(str, MEMORY_DEFAULT)))
    ap.add_argument("--velocity-predictor", type=float, default=PREDICTOR_DEFAULT,
                    help="fs_set_velocity_predictor weight for the value arm and the ensemble: one Broyden update "
                         "of this weight from the residual with extrapolated velocities before each step's first "
                         "residual (default %g; 0 turns it off)" % PREDICTOR_DEFAULT)
    ap.add_argument("--train-seeds", type=int, default=20, help="plain-solver runs that generate training data")
    ap.add_argument("--workload", default="sediment_512",
                    choices=["sediment_512", "mobility_256", "ensemble_64", "mlp", "trajectory_200"],
                    help="sediment_512: implicit steps (the headline); mobility_256: FCM mobility solves, "
                         "FP32 against FP64, on 256^3 with 1024 x 30 beads; ensemble_64: 64 independent "
                         "boxes advanced by one graph launch per step; trajectory_200: the configured run "
                         "of sediment_512, steps 1-200 from the placed suspension, mixed precision and FP64, "
                         "with per-step iterations (a record, not a throughput benchmark)")
    ap.add_argument("--grid", default=None,
                    help="sediment_512 / mobility_256 on another cubic grid N, or mobility_256 on NX,NY,NZ "
                         "(profiling cases; the workload name in config says so)")
    ap.add_argument("--filaments", type=int, default=None, help="and another filament count")
    args = ap.parse_args()
    args.memory = MEMORY_OFF if args.broyden_memory == "0" else tuple(int(v) for v in args.broyden_memory.split(":"))
    if len(args.memory) != 4:
        ap.error("--broyden-memory wants KEEP:CARRY:THRESHOLD:RESTART or 0")
    if args.grid:
        g = tuple(int(v) for v in args.grid.split(","))
        if len(g) == 3 and args.workload == "mobility_256":
            args.grid = g  # a profiling case with lines of different lengths per axis
        elif len(g) == 1:
            args.grid = g[0]
        else:
            ap.error("--grid wants N, or NX,NY,NZ with --workload mobility_256")
    if args.grid or args.filaments:
        w = WORKLOAD if args.workload == "sediment_512" else None
        if args.workload == "mobility_256":
            from filsim_b200.configs import WORKLOADS
            w = WORKLOADS["mobility_256"]
        if w is not None:
            w["npts"] = args.grid or w["npts"]
            w["nfil"] = args.filaments or w["nfil"]
            base = "sediment" if args.workload == "sediment_512" else "mobility"
            gname = "x".join(map(str, w["npts"])) if isinstance(w["npts"], tuple) else "%d" % w["npts"]
            w["name"] = "%s_%s_%dx%d" % (base, gname, w["nfil"], w["nw"])
    return args


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ["index", "clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.active",
              "clocks_event_reasons.hw_slowdown", "clocks_event_reasons.hw_thermal_slowdown",
              "clocks_event_reasons.sw_thermal_slowdown", "clocks_event_reasons.sw_power_cap"]

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + ",".join(self.FIELDS), "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def state_bytes(s):
    n = 0
    for k, v in s.arrays.items():
        n += v.nbytes
    return n + s.fil_start.nbytes


def run_ours(args, rank, world):
    import numpy as np
    import torch
    from filsim_b200 import abi
    from filsim_b200.configs import make_sediment_case
    from filsim_b200.fcm import Context, Simulation
    from filsim_b200 import replicas
    from filsim_b200.learn import WarmStartModel, generate, set_warm_start

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", dev))
    K, W = args.steps, args.warmup
    nw = WORKLOAD["nw"]
    p, susp = make_sediment_case(WORKLOAD["npts"], WORKLOAD["nfil"], nw,
                                 seed=replicas.replica_seed(WORKLOAD["seed"], rank))
    npb = susp.np
    stream = torch.cuda.Stream()
    ctx = Context(p, max_beads=npb, max_filaments=susp.nfil, stream=stream)

    def barrier():
        replicas.barrier(dist)

    def max_over_ranks(x):
        return replicas.max_over_ranks(x, dist, device="cuda")

    # Start-up (untimed): the first PREP_STEPS steps use implicit Euler and the
    # constant / linear tension extrapolation; every timed step is in the
    # steady BDF2 regime with the quadratic extrapolation.
    ctx.set_precision(abi.FS_PREC_FP32)
    sim0 = Simulation(ctx, susp.copy())
    sim0.run_steps(1, PREP_STEPS)
    prep = susp.copy()
    sim0.download_into(prep)
    nt0 = PREP_STEPS + 1
    # the FP32 chain's error against FP64: one mobility solve of the prepared state in each
    from filsim_b200.fcm import Fcm
    sim_e = Simulation(ctx, prep.copy())
    sim_e.initial_guess()
    sim_e.filament_forces(nt0)
    fcm = Fcm(ctx, npb)
    for name, buf in (("Y", fcm.Y), ("F", fcm.F), ("TAU", fcm.T)):
        buf.copy_(sim_e.device_array(name, (npb, 3)))
    torch.cuda.synchronize()
    vel = {}
    for prec in (abi.FS_PREC_FP64, abi.FS_PREC_FP32):
        ctx.set_precision(prec)
        fcm.mobility_solve()
        vel[prec] = (fcm.V.cpu().numpy(), fcm.W.cpu().numpy())
    rel = lambda a, b: float(np.abs(a - b).max() / np.abs(b).max())
    fp32_err = {"U": rel(vel[abi.FS_PREC_FP32][0], vel[abi.FS_PREC_FP64][0]),
                "Omega": rel(vel[abi.FS_PREC_FP32][1], vel[abi.FS_PREC_FP64][1])}
    del fcm, sim_e
    ctx.set_precision(abi.FS_PREC_FP32)
    # launch variants for this grid and suspension (untimed)
    choice = np.zeros(4, np.int32)
    tune_ms = ctypes.c_float()
    abi.check(abi.lib().fs_autotune(ctx.h, 2, choice.ctypes.data_as(ctypes.c_void_p), ctypes.byref(tune_ms)),
              "fs_autotune")
    del sim0

    # Warm-start network, trained untimed by the library's kernels on plain-solver
    # data: TRAIN_SEEDS runs of this suspension's size with K_B log-uniform in
    # [0.1, 10], one recorded steady-state step each.
    learned = learned_failed = None
    if not args.no_learned:
        t0 = time.time()
        model = WarmStartModel(ctx, nw, hidden=256, batch_capacity=4096, seed=rank)

        def make_case(seed, kb):
            return make_sediment_case(WORKLOAD["npts"], WORKLOAD["nfil"], nw, seed=seed, kap=kb)

        seeds = [TRAIN_SEED0 + 100 * rank + i for i in range(args.train_seeds)]
        ctx.set_start_order(args.start_order)  # targets: corrections to the value arm's start
        ctx.set_tension_extrapolation(args.tension_order)
        feats, tgts, its_tr = generate(make_case, seeds, PREP_STEPS + 1, 1, model=model)
        t1 = time.time()
        model.fit_normalization(feats, tgts)
        try:
            losses = model.fit(feats, tgts, epochs=TRAIN_EPOCHS, batch=2048, lr=1e-3, lr_final=5e-5, seed=rank)
        except FloatingPointError as e:
            print("warm-start training failed: %s; timing the reference's start" % e, file=sys.stderr)
            losses = None
        t2 = time.time()
        learned = {"train_pairs": int(feats.shape[0]), "train_seeds": len(seeds), "data_seconds": t1 - t0,
                   "train_seconds": t2 - t1, "epochs": TRAIN_EPOCHS,
                   "loss_first": losses[0] if losses else None, "loss_last": losses[-1] if losses else None,
                   "plain_iters_in_data": float(np.mean(its_tr))}
        del feats, tgts
        if losses is None:
            learned_failed = learned
            learned = None

    def gate_stats():
        steps = np.zeros(2, np.int64)
        solves = np.zeros(2, np.float64)
        abi.check(abi.lib().fs_warm_start_gate_stats(ctx.h, steps.ctypes.data_as(ctypes.c_void_p),
                                                     solves.ctypes.data_as(ctypes.c_void_p)),
                  "fs_warm_start_gate_stats")
        return steps, solves

    def timed_steps(prec, mode, profile=False, gate=0, start=1, tension=2, esc=0, mem=MEMORY_OFF, pred=0.0):
        ctx.set_precision(prec)
        ctx.set_start_order(start)
        ctx.set_tension_extrapolation(tension)
        ctx.set_precision_escalation(esc)
        ctx.set_broyden_memory(*mem)
        ctx.set_velocity_predictor(pred)
        if learned:
            set_warm_start(ctx, mode)
            abi.check(abi.lib().fs_warm_start_gate(ctx.h, gate if mode else 0), "fs_warm_start_gate")
            abi.check(abi.lib().fs_warm_start_bound(ctx.h, BOUND_REFRESH if mode else 0), "fs_warm_start_bound")
        # steady steps with the reference's start run as one CUDA graph each (Broyden
        # loop on the device), also those the cost gate gives the plain start; steps
        # with the learned start run host-driven
        graph = 0 if args.no_graph else 1
        abi.check(abi.lib().fs_set_graph_mode(ctx.h, graph), "fs_set_graph_mode")
        sim = Simulation(ctx, prep.copy())
        sim.run_steps(nt0, W)
        barrier()
        g0 = gate_stats()[0] if learned else None
        if profile:
            ctx.profile_enable(True)
        launches0 = abi.lib().fs_kernel_launches()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        with ClockSampler(dev) as clk:
            torch.cuda.nvtx.range_push("timed_steps")
            ev0.record(stream)
            its, st = sim.run_steps(nt0 + W, K)
            ev1.record(stream)
            torch.cuda.synchronize()
            torch.cuda.nvtx.range_pop()
        ms = ev0.elapsed_time(ev1)
        launches = abi.lib().fs_kernel_launches() - launches0
        prof = ctx.profile() if profile else None
        if profile:
            ctx.profile_enable(False)
        diag = sim.diag()
        if learned:
            g1, gs = gate_stats()
            diag.gate = {"period": gate if mode else 0, "timed_plain_start_steps": int(g1[0] - g0[0]),
                         "timed_learned_start_steps": int(g1[1] - g0[1]),
                         "mean_solves_per_step": {"plain_start": float(gs[0]), "learned_start": float(gs[1])}}
        barrier()
        return max_over_ranks(ms), its, st, prof, clk.summary(), launches, diag

    mode = 1 if learned else 0
    gate = GATE_PERIOD if learned else 0
    start, tension = args.start_order, args.tension_order
    ms, its, st, _, clocks, launches, diag = timed_steps(abi.FS_PREC_FP32, mode, gate=gate, start=start,
                                                         tension=tension, esc=args.escalate, mem=args.memory,
                                                         pred=args.velocity_predictor)
    # stage breakdown: the same steps again, host-driven with CUDA-event stage timing
    # (graph-captured steps carry no events); not part of the timed value
    abi.check(abi.lib().fs_set_graph_mode(ctx.h, 0), "fs_set_graph_mode")
    ctx.set_start_order(start)
    ctx.set_tension_extrapolation(tension)
    ctx.set_precision_escalation(args.escalate)
    ctx.set_broyden_memory(*args.memory)
    ctx.set_velocity_predictor(args.velocity_predictor)
    if learned:
        set_warm_start(ctx, mode)
        abi.check(abi.lib().fs_warm_start_gate(ctx.h, gate), "fs_warm_start_gate")
        abi.check(abi.lib().fs_warm_start_bound(ctx.h, BOUND_REFRESH), "fs_warm_start_bound")
    simp = Simulation(ctx, prep.copy())
    simp.run_steps(nt0, W)
    ctx.profile_enable(True)
    simp.run_steps(nt0 + W, K)
    prof = ctx.profile()
    ctx.profile_enable(False)
    del simp
    value = replicas.job_throughput(npb, K, ms, world)
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 FCM chain + f64 Broyden/mechanics", "data": "synthetic (seeded rejection-placed filaments)",
        "config": {"workload": WORKLOAD["name"], "grid": [WORKLOAD["npts"]] * 3, "filaments": WORKLOAD["nfil"],
                   "beads_per_filament": nw, "beads": npb, "dt": p.dt, "tol": p.tol,
                   "precision": "mixed", "learned_warm_start": bool(learned),
                   "start": start_label(start, tension), "escalate_after_iters": args.escalate,
                   "broyden_memory": memory_label(args.memory), "velocity_predictor": args.velocity_predictor,
                   "timed_steps": [nt0 + W, nt0 + W + K - 1],
                   "start_up": "steps 1-%d (implicit Euler, constant/linear tension extrapolation) run untimed"
                               % PREP_STEPS,
                   "parallelism": "replicas x%d" % world, "l2": "inputs larger than L2 (grids ~10 GB)"},
        "iters_per_step": float(np.mean(its)), "status": abi.STATUS_NAMES.get(st, st),
        "mobility_solves_per_step": diag.mobility_solves / K,
        "clocks": clocks, "gpu_launches": int(launches),
        "fp32_velocity_error_vs_fp64": dict(fp32_err, norm="max |FP32 - FP64| / max |FP64|, one solve of the "
                                                          "prepared state"),
        "autotuned": {"spread_beads_per_pass": int(choice[0]), "interp_beads_per_cta": int(choice[1]),
                      "transform": "warp FFT" if (choice[2] == 0 and warp_fft_length(WORKLOAD["npts"])) else "cuFFT",
                      "spread_column_block": "%d x 16 x %d" % (choice[3], 16 // choice[3]),
                      "ms_per_solve": tune_ms.value},
    }
    if learned:
        nlf = diag.learned_filaments + diag.fallback_filaments
        learned["learned_fraction"] = diag.learned_filaments / max(1, nlf)
        learned["gate"] = diag.gate
        out["learned"] = learned
    elif learned_failed:
        out["learned"] = dict(learned_failed, error="training loss not finite; value is the reference's start")
    stage_ms = {k: v[0] for k, v in prof.items()}
    stage_calls = {k: v[1] for k, v in prof.items()}
    out["stage_ms_per_step"] = {k: v / K for k, v in stage_ms.items() if v > 0}

    # roofline of the dominant single kernel of this library (CUDA events around
    # each launch on the context's stream, host-driven steps); algorithmic bytes
    # per launch: each grid pass reads and writes the grid once
    peak, peak_kind = measured_peaks()
    npts = WORKLOAD["npts"]
    N = npts ** 3
    NH = npts * npts * (npts // 2 + 1)
    s_real = 4  # FP32 grids in the mixed path
    half = 3 * NH * 2 * s_real                         # the three half spectra, complex FP32
    alg_bytes = {
        "k_spread": 3 * s_real * N + npb * 9 * 8,      # write f once; read bead Y, F, T
        "k_fft_z_fwd": 3 * s_real * N + half,          # read f, write the half spectra
        "k_fft_y_fwd": 2 * half,
        "project": 2 * half,                           # the x pass with the projection
        "k_fft_y_inv": 2 * half,
        "k_fft_z_inv": half + 3 * s_real * N,
        "k_interp": 3 * s_real * N + npb * 9 * 8,      # read u once; bead Y in, V, W out
    }
    cands = {k: stage_ms[k] for k in alg_bytes if stage_ms.get(k, 0) > 0}
    dom = max(cands, key=cands.get)
    per_launch_ms = stage_ms[dom] / max(1, stage_calls[dom])
    achieved = alg_bytes[dom] / (per_launch_ms / 1e3) / 1e9
    out["roofline"] = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                       "frac": achieved / peak, "peak_source": "%s (MEASURED_PEAKS.json hbm_gbs)" % peak_kind,
                       "traffic": NCU_TRAFFIC_PER_POINT[dom] * N if dom in NCU_TRAFFIC_PER_POINT else None,
                       "traffic_source": NCU_TRAFFIC_SOURCE, "algorithmic_bytes": alg_bytes[dom],
                       "launch_ms": per_launch_ms,
                       "kernels": {k: {"ms_per_launch": stage_ms[k] / max(1, stage_calls[k]),
                                       "share_of_step": stage_ms[k] / max(1e-9, sum(stage_ms[x] for x in (
                                           "spread", "fft_fwd", "project", "fft_inv", "interp", "link", "barrier",
                                           "forces", "jacobian", "error_check", "broyden", "update", "learn"))),
                                       "frac": alg_bytes[k] / (stage_ms[k] / max(1, stage_calls[k]) / 1e3) / 1e9
                                       / peak} for k in cands}}
    fcm_ms = sum(stage_ms.get(k, 0) for k in ("spread", "fft_fwd", "project", "fft_inv", "interp"))
    solves = max(1, stage_calls.get("interp", 0))
    b_fcm = 24 * s_real * N
    out["fcm_chain"] = {"ms_per_solve": fcm_ms / solves, "bytes_per_solve": b_fcm,
                        "GBps": b_fcm / (fcm_ms / solves / 1e3) / 1e9, "frac": b_fcm / (fcm_ms / solves / 1e3) / 1e9 / peak}

    # the same steps from the reference's start (no learned iterate), FP32 chain,
    # and with the learned start on every step (no cost gate)
    if learned:
        msa, itsa, sta, _, _, _, da = timed_steps(abi.FS_PREC_FP32, mode, gate=0, start=start, tension=tension,
                                                  mem=args.memory, pred=args.velocity_predictor)
        nla = da.learned_filaments + da.fallback_filaments
        out["learned_every_step"] = {"value": world * npb * K / (msa / 1e3), "ms_per_step": msa / K,
                                     "iters_per_step": float(np.mean(itsa)),
                                     "status": abi.STATUS_NAMES.get(sta, sta),
                                     "mobility_solves_per_step": da.mobility_solves / K,
                                     "learned_fraction": da.learned_filaments / max(1, nla)}
    if learned and (start, tension) != (1, 2):
        msq, itsq, stq, _, _, _, dq = timed_steps(abi.FS_PREC_FP32, 0, start=start, tension=tension,
                                                  mem=args.memory, pred=args.velocity_predictor)
        out["fp32_improved_start"] = {"value": world * npb * K / (msq / 1e3), "ms_per_step": msq / K,
                                       "iters_per_step": float(np.mean(itsq)),
                                       "status": abi.STATUS_NAMES.get(stq, stq),
                                       "mobility_solves_per_step": dq.mobility_solves / K}
    if args.memory != MEMORY_OFF or args.velocity_predictor > 0:
        msn, itsn, stn, _, _, _, dn = timed_steps(abi.FS_PREC_FP32, 0, start=start, tension=tension)
        out["fp32_start_only"] = {"value": world * npb * K / (msn / 1e3), "ms_per_step": msn / K,
                                         "iters_per_step": float(np.mean(itsn)),
                                         "status": abi.STATUS_NAMES.get(stn, stn),
                                         "mobility_solves_per_step": dn.mobility_solves / K,
                                         "start": start_label(start, tension)}
    if learned or (start, tension) != (1, 2):
        ms0, its0, st0, _, _, _, d0 = timed_steps(abi.FS_PREC_FP32, 0, start=1, tension=2)
        out["fp32_plain_start"] = {"value": world * npb * K / (ms0 / 1e3), "ms_per_step": ms0 / K,
                                   "iters_per_step": float(np.mean(its0)), "status": abi.STATUS_NAMES.get(st0, st0),
                                   "mobility_solves_per_step": d0.mobility_solves / K}
    # plain FP64 FCM chain, reference start
    if not args.no_fp64:
        ms64, its64, st64, _, _, _, d64 = timed_steps(abi.FS_PREC_FP64, 0, start=1, tension=2)
        out["plain_fp64"] = {"value": world * npb * K / (ms64 / 1e3), "ms_per_step": ms64 / K,
                             "iters_per_step": float(np.mean(its64)), "status": abi.STATUS_NAMES.get(st64, st64)}
        out["speedup_vs_plain_fp64"] = out["value"] / out["plain_fp64"]["value"]

    # end to end through the C-ABI with pinned host state (same start and precision as value)
    if not args.no_e2e:
        ctx.set_precision(abi.FS_PREC_FP32)
        ctx.set_start_order(start)
        ctx.set_tension_extrapolation(tension)
        ctx.set_precision_escalation(args.escalate)
        ctx.set_broyden_memory(*args.memory)
        ctx.set_velocity_predictor(args.velocity_predictor)
        if learned:
            set_warm_start(ctx, mode)
            abi.check(abi.lib().fs_warm_start_gate(ctx.h, gate), "fs_warm_start_gate")
            abi.check(abi.lib().fs_warm_start_bound(ctx.h, BOUND_REFRESH), "fs_warm_start_bound")
        abi.check(abi.lib().fs_set_graph_mode(ctx.h, 0 if args.no_graph else 1), "fs_set_graph_mode")
        host = prep.copy()
        # the state a step needs, as the reference checkpoints it (.bak: X, Xt, q, qt, U, Ut,
        # lam, lam1, lam2) plus K_B and C; Xs, Us, qs, F and TAU are recomputed by every step
        # (initial guess, forces), so their upload and download are left out (NULL)
        host.arrays = {k: v for k, v in host.arrays.items() if k in CHECKPOINT_FIELDS}
        pinned = {}
        for k, v in host.arrays.items():
            t = torch.empty(v.shape, dtype=torch.float64, pin_memory=True)
            t.numpy()[...] = v
            pinned[k] = t
        host.arrays = {k: t.numpy() for k, t in pinned.items()}
        sim = Simulation(ctx, host)
        sim.run_steps(nt0, W)
        sim.download_into(host)
        barrier()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for k in range(K):
            sim.upload(host)                      # H2D of the step's input state
            sim.step_implicit(nt0 + W + k)
            sim.download_into(host)               # D2H of the step's result
        ev1.record(stream)
        torch.cuda.synchronize()
        ms_e2e = max_over_ranks(ev0.elapsed_time(ev1))
        nbytes = state_bytes(host)
        out["e2e"] = {"value": world * npb * K / (ms_e2e / 1e3), "unit": UNIT, "h2d_bytes_per_step": nbytes,
                      "d2h_bytes_per_step": nbytes, "ms_per_step": ms_e2e / K}

    # CPU baseline: the oracle on this host's cores, sampled
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(p, susp, out.get("plain_fp64", {}).get("iters_per_step",
                                                                                   out["iters_per_step"]))
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return out


def run_trajectory(args, rank, world):
    """Workload trajectory_200: the configured run of sediment_512, steps 1-200
    from the placed suspension (start-up steps included), once with the mixed-
    precision chain (FP32 spread/FFT/interpolation, FP64 Broyden and mechanics)
    and once in FP64, both from the reference's start, and mixed with the improved
    start (fs_set_start_order 2, fs_set_tension_extrapolation 1) four more times:
    alone, with precision escalation (fs_set_precision_escalation), with the
    Broyden memory (fs_set_broyden_memory), and with the memory and the velocity
    predictor (fs_set_velocity_predictor); all with graph-captured steady steps.
    Records per-step Broyden iterations, the status, the final barrier minimum
    squared distance, the wall time of each run and, for the improved start, how
    far its final positions are from the reference start's."""
    import numpy as np
    import torch
    from filsim_b200 import abi
    from filsim_b200.configs import make_sediment_case
    from filsim_b200.fcm import Context, Simulation

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    nsteps = args.steps if args.steps > 8 else 200
    p, susp = make_sediment_case(WORKLOAD["npts"], WORKLOAD["nfil"], WORKLOAD["nw"], seed=WORKLOAD["seed"])
    stream = torch.cuda.Stream()
    ctx = Context(p, max_beads=susp.np, max_filaments=susp.nfil, stream=stream)
    abi.check(abi.lib().fs_set_graph_mode(ctx.h, 1), "fs_set_graph_mode")
    out = {"workload": "trajectory_%d" % nsteps, "grid": [WORKLOAD["npts"]] * 3, "filaments": WORKLOAD["nfil"],
           "beads_per_filament": WORKLOAD["nw"], "beads": susp.np, "dt": p.dt, "tol": p.tol, "steps": nsteps}
    finals = {}
    esc = args.escalate if args.escalate > 0 else 15
    mem = args.memory if args.memory != MEMORY_OFF else MEMORY_DEFAULT
    pw = args.velocity_predictor if args.velocity_predictor > 0 else PREDICTOR_DEFAULT
    runs = (("mixed", abi.FS_PREC_FP32, 1, 2, 0, MEMORY_OFF, 0.0),
            ("mixed_improved_start", abi.FS_PREC_FP32, 2, 1, 0, MEMORY_OFF, 0.0),
            ("mixed_improved_start_escalated", abi.FS_PREC_FP32, 2, 1, esc, MEMORY_OFF, 0.0),
            ("mixed_improved_start_broyden_memory", abi.FS_PREC_FP32, 2, 1, 0, mem, 0.0),
            ("mixed_improved_start_memory_predictor", abi.FS_PREC_FP32, 2, 1, 0, mem, pw),
            ("fp64", abi.FS_PREC_FP64, 1, 2, 0, MEMORY_OFF, 0.0))
    for name, prec, start, tension, after, memory, weight in runs:
        ctx.set_precision(prec)
        ctx.set_start_order(start)
        ctx.set_tension_extrapolation(tension)
        ctx.set_precision_escalation(after)
        ctx.set_broyden_memory(*memory)
        ctx.set_velocity_predictor(weight)
        sim = Simulation(ctx, susp.copy())
        torch.cuda.synchronize()
        t0 = time.time()
        with ClockSampler(dev) as clk:
            its, st = sim.run_steps(1, nsteps)
        wall = time.time() - t0
        d = sim.diag()
        X = sim.download()["X"]
        out[name] = {"status": abi.STATUS_NAMES.get(st, st), "iters": [int(v) for v in its],
                     "iters_mean_steps_13_on": float(np.mean(its[12:])), "iters_max": int(its.max()),
                     "not_converged_steps": int(d.not_converged_steps), "nonfinite": int(d.nonfinite),
                     "final_min_dist2": d.min_dist2, "final_max_abs_err": d.last_max_abs_err,
                     "wall_s": wall, "mobility_solves": int(d.mobility_solves), "clocks": clk.summary(),
                     "final_mean_z": float(X[:, 2].mean()), "escalated_iters": int(d.escalated_iters)}
        finals[name] = X.copy()
    for name in ("mixed_improved_start", "mixed_improved_start_escalated", "mixed_improved_start_broyden_memory",
                 "mixed_improved_start_memory_predictor"):
        out[name]["start"] = start_label(2, 1)
        out[name]["final_max_dX_vs_mixed_over_dx"] = float(np.abs(finals[name] - finals["mixed"]).max() / p.dx)
    out["mixed_improved_start_escalated"]["escalate_after_iters"] = esc
    out["mixed_improved_start_broyden_memory"]["broyden_memory"] = memory_label(mem)
    out["mixed_improved_start_memory_predictor"]["broyden_memory"] = memory_label(mem)
    out["mixed_improved_start_memory_predictor"]["velocity_predictor"] = pw
    ctx.close()
    return out


def run_mobility(args, rank, world):
    """Workload mobility_256: one step is one FCM mobility solve (spread, FFT,
    projection, inverse FFT, interpolation) of 30,720 beads on 256^3, timed in
    FP32 (value) and FP64; the FP32 velocities are compared with the FP64 ones."""
    import numpy as np
    import torch
    from filsim_b200 import abi
    from filsim_b200.configs import WORKLOADS, make_mobility_case
    from filsim_b200.fcm import Context, Fcm

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    w = WORKLOADS["mobility_256"]
    p, s, Y, F, T = make_mobility_case(w["npts"], w["nfil"], w["nw"], w["seed"] + rank)
    stream = torch.cuda.Stream()
    ctx = Context(p, max_beads=s.np, max_filaments=s.nfil, stream=stream)
    fcm = Fcm(ctx, s.np)
    fcm.set(Y, F, T)
    K, W = args.steps, args.warmup
    res = {}
    for name, prec in (("fp32", abi.FS_PREC_FP32), ("fp64", abi.FS_PREC_FP64)):
        ctx.set_precision(prec)
        for _ in range(W):
            fcm.mobility_solve()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        launches0 = abi.lib().fs_kernel_launches()
        with ClockSampler(dev) as clk:
            torch.cuda.nvtx.range_push("timed_steps")
            ev0.record(stream)
            for _ in range(K):
                fcm.mobility_solve()
            ev1.record(stream)
            torch.cuda.synchronize()
            torch.cuda.nvtx.range_pop()
        res[name] = dict(ms=ev0.elapsed_time(ev1), V=fcm.V.cpu().numpy(), W=fcm.W.cpu().numpy(),
                         clocks=clk.summary(), launches=abi.lib().fs_kernel_launches() - launches0)
    ctx.close()
    relerr = lambda a, b: float(np.abs(a - b).max() / np.abs(b).max())
    ms = res["fp32"]["ms"]
    return {"metric": "FCM mobility bead-solves/s (FP32 chain; FP64 beside it)", "value": s.np * K / (ms / 1e3),
            "unit": "bead-solves/s", "n_gpus": 1, "steps": K, "warmup": W, "ms_per_step": ms / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded rejection-placed filaments, F, T ~ N(0,1))",
            "config": {"workload": w.get("name", "mobility_256"),
                       "grid": list(w["npts"]) if isinstance(w["npts"], tuple) else [w["npts"]] * 3,
                       "filaments": w["nfil"],
                       "beads_per_filament": w["nw"], "beads": s.np, "l2": "grids (~0.4 GB) larger than L2"},
            "fp64": {"value": s.np * K / (res["fp64"]["ms"] / 1e3), "ms_per_step": res["fp64"]["ms"] / K},
            "fp32_error_vs_fp64": {"U": relerr(res["fp32"]["V"], res["fp64"]["V"]),
                                   "Omega": relerr(res["fp32"]["W"], res["fp64"]["W"])},
            "clocks": res["fp32"]["clocks"], "gpu_launches": int(res["fp32"]["launches"])}


def run_ensemble(args, rank, world):
    """Workload ensemble_64: 64 independent boxes (grids 48^3-128^3, 8-256 filaments of
    16 beads capped at 5% bead volume fraction, K_B log-uniform in [0.1, 10],
    gravity, dt = 0.05), FP32 chain. After 12 untimed start-up steps per box, each
    ensemble step is one CUDA graph launch holding every box's step with its
    Broyden loop on the device. Beside it: the same boxes stepped one at a time by
    the host-driven step. With several ranks (one GPU each) the same 64 boxes are
    split by estimated cost (partition_boxes): each rank runs its share as one
    ensemble, the time is the slowest rank's, and the value is all boxes' bead-steps
    over it (strong scaling; no collective on the data)."""
    import numpy as np
    import torch
    from filsim_b200 import abi
    from filsim_b200 import replicas
    from filsim_b200.ensemble import Ensemble, make_boxes, partition_boxes

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", dev))
    K, W = args.steps, args.warmup
    all_boxes = make_boxes(ENSEMBLE_SEED)
    mine = partition_boxes(all_boxes, world)[rank]
    boxes = [all_boxes[i] for i in mine]
    ens = Ensemble(boxes, precision=abi.FS_PREC_FP32, start_order=args.start_order,
                   tension_order=args.tension_order, escalate=args.escalate, memory=args.memory,
                   predictor=args.velocity_predictor)
    t0 = time.time()
    ens.startup(PREP_STEPS)
    t_start = time.time() - t0
    tuned = ens.autotune(reps=3)
    nt0 = PREP_STEPS + 1
    ens.run(nt0, W)                                    # captures the ensemble graph, warms up
    launches0 = abi.lib().fs_kernel_launches()
    replicas.barrier(dist)
    with ClockSampler(dev) as clk:
        torch.cuda.nvtx.range_push("timed_steps")
        its, ms, total, st = ens.run(nt0 + W, K)
        torch.cuda.nvtx.range_pop()
    replicas.barrier(dist)
    launches = abi.lib().fs_kernel_launches() - launches0
    total = replicas.max_over_ranks(total, dist, device="cuda")
    beads = int(sum(b[2].np for b in all_boxes))
    value = beads * K / (total / 1e3)
    # the same boxes, one at a time, host-driven steps (no graphs, one sync per iteration)
    K2 = max(1, min(K, 4))
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    seq_ms = 0.0
    for c, sim in zip(ens.ctxs, ens.sims):
        abi.check(abi.lib().fs_set_graph_mode(c.h, 0), "fs_set_graph_mode")
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        sim.run_steps(nt0 + W + K, K2)
        c.synchronize()
        seq_ms += (time.perf_counter() - t1) * 1e3
    seq_ms = replicas.max_over_ranks(seq_ms, dist, device="cuda")
    seq_value = beads * K2 / (seq_ms / 1e3)
    grids = [b[0] for b in all_boxes]
    out = {"metric": "bead-steps/s (ensemble of 64 boxes, one graph launch per step)", "value": value,
           "unit": "bead-steps/s", "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": total / K,
           "higher_is_better": True, "scaling": "strong" if world > 1 else "weak", "vs_baseline": None,
           "dtype": "f32 FCM chain + f64 Broyden",
           "data": "synthetic (seeded rejection-placed filaments)",
           "config": {"workload": "ensemble_64", "boxes": len(all_boxes), "boxes_per_rank": len(boxes),
                      "grids": {str(g): grids.count(g) for g in sorted(set(grids))}, "beads": beads,
                      "filaments": int(sum(b[2].nfil for b in all_boxes)), "beads_per_filament": 16,
                      "timed_steps": [nt0 + W, nt0 + W + K - 1], "start_up_seconds": t_start,
                      "l2": "no flush; most boxes fit in L2 (the workload's own sizes)",
                      "start": start_label(args.start_order, args.tension_order),
                      "escalate_after_iters": args.escalate, "broyden_memory": memory_label(args.memory),
                      "velocity_predictor": args.velocity_predictor},
           "box_step_ms": {"p50": float(np.percentile(ms, 50)), "p99": float(np.percentile(ms, 99)),
                           "max": float(ms.max())},
           "iters_per_step": float(its.mean()), "status": abi.STATUS_NAMES.get(st, st),
           "clocks": clk.summary(), "gpu_launches": int(launches), "graph_launches": K,
           "autotuned": {str(g): {"spread_beads_per_pass": v[0], "interp_beads_per_cta": v[1],
                                  "transform": "warp FFT" if (v[2] == 0 and warp_fft_length(g)) else "cuFFT",
                                  "spread_column_block": "%d x 16 x %d" % (v[3], 16 // v[3]),
                                  "ms_per_solve": v[4]} for g, v in tuned.items()},
           "sequential_host_driven": {"value": seq_value, "ms_per_ensemble_step": seq_ms / K2, "steps": K2},
           "speedup_vs_sequential": value / seq_value}
    ens.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return out if rank == 0 else None


def run_mlp(args, rank, world):
    """Workload mlp: the tensor-core GEMM of the warm-start network (fs_gemm_bf16:
    tcgen05.mma, BF16 operands, FP32 accumulators in tensor memory) on 8192^3
    against the measured cuBLAS BF16 peak, and the network itself at the sizes of
    sediment_512 (888 features -> 3 x 256 -> 384 outputs): inference for 4096
    filaments and one Adam step on 4096 pairs."""
    import numpy as np
    import torch
    from filsim_b200.configs import params_for
    from filsim_b200.fcm import Context
    from filsim_b200.learn import WarmStartModel

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    K, W = args.steps, args.warmup
    ctx = Context(params_for(32), max_beads=64, max_filaments=8)
    n = 8192
    g = torch.Generator(device="cuda")
    g.manual_seed(rank)
    A = torch.randn((n, n), generator=g, device="cuda").to(torch.bfloat16)
    B = torch.randn((n, n), generator=g, device="cuda").to(torch.bfloat16)
    D = torch.empty((n, n), dtype=torch.float32, device="cuda")
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())
    for _ in range(W):
        ctx.call("fs_gemm_bf16", ptr(A), ptr(B), ptr(D), n, n, n)
    # the context's stream is a blocking stream, so events on torch's default stream
    # bracket its work; each call also waits for its own completion (error word)
    times = []
    stream = torch.cuda.current_stream()
    with ClockSampler(dev) as clk:
        for _ in range(K):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.call("fs_gemm_bf16", ptr(A), ptr(B), ptr(D), n, n, n)
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
    gemm_ms = float(np.median(times))
    gemm_tf = 2.0 * n ** 3 / (gemm_ms / 1e3) / 1e12
    ref = (A[:256].double() @ B[:256].double().T)
    gemm_err = float((D[:256, :256].double() - ref).abs().max() / ref.abs().max())
    del A, B, D
    peaks = {}
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        peaks = json.load(open(path))
    peak = peaks.get("bf16_tflops", 1590.0)
    # the network at the sizes of sediment_512
    model = WarmStartModel(ctx, WORKLOAD["nw"], hidden=256, batch_capacity=4096, seed=rank)
    rows = 4096
    feats = torch.randn((rows, model.n_features), generator=g, device="cuda")
    tgts = torch.randn((rows, model.n_targets), generator=g, device="cuda")
    model.fit_normalization(feats, tgts)
    d = model.dims
    fwd_flops = 2.0 * rows * sum(d[i] * d[i + 1] for i in range(4))
    for _ in range(W):
        model.forward(feats)
        model.train_step(feats, tgts, 1e-4)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(K):
        model.forward(feats)
    torch.cuda.synchronize()
    inf_ms = (time.perf_counter() - t0) / K * 1e3
    t0 = time.perf_counter()
    for _ in range(K):
        model.train_step(feats, tgts, 1e-4)
    torch.cuda.synchronize()
    train_ms = (time.perf_counter() - t0) / K * 1e3
    ctx.close()
    return {"metric": "BF16 tensor-core GEMM TFLOP/s (8192^3, tcgen05, FP32 accumulation)", "value": gemm_tf,
            "unit": "TFLOP/s", "n_gpus": 1, "steps": K, "warmup": W, "ms_per_step": gemm_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16 (fp32 accumulation)",
            "data": "synthetic (N(0,1) operands)",
            "config": {"workload": "mlp", "gemm": [n, n, n], "mlp_layers": d, "mlp_rows": rows},
            "roofline": {"kernel": "k_gemm_bf16", "bound": "tensor", "achieved": gemm_tf, "peak": peak,
                         "unit": "TFLOP/s", "frac": gemm_tf / peak,
                         "peak_source": "measured cuBLAS burst (MEASURED_PEAKS.json bf16_tflops)"
                         if "bf16_tflops" in peaks else "fallback"},
            "gemm_rel_error_vs_fp64": gemm_err,
            "mlp_inference": {"ms": inf_ms, "tflops": fwd_flops / (inf_ms / 1e3) / 1e12, "filaments": rows},
            "mlp_train_step": {"ms": train_ms, "tflops": 3 * fwd_flops / (train_ms / 1e3) / 1e12, "pairs": rows},
            "clocks": clk.summary()}


# The CPU arms time the oracle's stages of one Broyden iteration at full size
# (every work unit): per iteration the collision barrier, the FCM mobility solve
# (spread, forward FFTs, projection, inverse FFTs, interpolation) and the rest
# (forces, error check, two J0^-1 applications with 10 history columns); once
# per step the Jacobian build and inversion. A step costs
# jacobian + (iterations + 1) x iteration.
ITERATION_STAGES = ("barrier", "spread", "fft_fwd", "project", "fft_inv", "interp", "iteration_other")
STAGE_CYCLE = ITERATION_STAGES + ("jacobian",)
# Broyden iterations per step of sediment_512 (seed 1002) in FP64, steps 1-200,
# measured on a B200 by `python bench.py --workload trajectory_200` (the FP64
# GPU path takes the oracle's iteration counts, tests/test_gpu_configs.py);
# the reference arm, which runs without a GPU, averages the entries of the
# steps its window covers.
FP64_ITERS_BY_STEP = (
    85, 28, 28, 26, 26, 26, 26, 26, 26, 26, 26, 26, 12, 12, 14, 12, 12, 12, 12, 16,
    19, 14, 16, 22, 15, 23, 14, 23, 17, 23, 16, 23, 23, 22, 24, 14, 23, 21, 23, 23,
    23, 14, 23, 15, 23, 23, 23, 12, 23, 16, 23, 17, 23, 23, 23, 12, 23, 17, 23, 23,
    23, 23, 16, 23, 15, 23, 23, 23, 14, 23, 23, 23, 22, 24, 22, 24, 19, 23, 14, 24,
    23, 23, 22, 16, 23, 22, 23, 17, 23, 15, 24, 23, 26, 24, 18, 24, 19, 24, 19, 26,
    21, 27, 21, 27, 23, 22, 22, 14, 28, 20, 26, 21, 29, 23, 23, 24, 18, 22, 24, 19,
    23, 19, 26, 23, 20, 17, 22, 14, 22, 20, 21, 22, 22, 22, 22, 22, 23, 23, 22, 23,
    23, 23, 24, 22, 23, 23, 24, 15, 29, 22, 26, 22, 24, 22, 28, 23, 24, 24, 24, 23,
    25, 23, 24, 23, 24, 23, 28, 23, 24, 24, 24, 24, 14, 29, 20, 26, 12, 29, 20, 26,
    22, 24, 24, 24, 24, 12, 30, 14, 26, 12, 29, 21, 24, 22, 23, 24, 22, 24, 20, 27,
)


def oracle_step_seconds(stage_s, iters):
    per_iter = sum(stage_s[k] for k in ITERATION_STAGES)
    return stage_s["jacobian"] + (iters + 1) * per_iter, per_iter


def cpu_baseline(p, susp, iters_per_step):
    """One complete full-size Broyden iteration and Jacobian build of the oracle
    on this host's cores (the workspace is allocated and touched first, untimed)."""
    from oracle import oracle_py
    sysw = oracle_py.System(p, susp)
    sysw.initial_guess()
    sysw.filament_forces(1)
    sysw.stage_costs(["project"], 1)  # allocates and touches the grids
    t0 = time.time()
    parts, nth = sysw.stage_costs(STAGE_CYCLE, 1)
    wall = time.time() - t0
    step_s, per_iter = oracle_step_seconds(parts, iters_per_step)
    sysw.close()
    return {"value": susp.np / step_s, "unit": UNIT, "cores": nth, "kind": "port",
            "sample": "one full-size Broyden iteration (barrier, FCM solve, forces, error check, J0^-1 "
                      "applications) and one Jacobian build of sediment_512 by the oracle, every work unit, "
                      "%.1f s wall; step = Jacobian + (%.2f+1) iterations, the FP64 GPU arm's mean in this run "
                      "(the oracle takes the same counts)" % (wall, iters_per_step),
            "seconds_per_step": step_s, "seconds_per_iteration": per_iter, "stage_seconds": parts}


def reference_case():
    """The workload's parameters and suspension, built on the CPU without the GPU
    library (the oracle's restatement of the generator reproduces its bits)."""
    import numpy as np
    from filsim_b200.configs import sediment_params
    from filsim_b200.suspension import Suspension
    from oracle import oracle_py
    p = sediment_params(WORKLOAD["npts"])
    X, Q = oracle_py.suspension_random(p, WORKLOAD["nfil"], WORKLOAD["nw"], WORKLOAD["seed"])
    fil_start = np.arange(WORKLOAD["nfil"] + 1, dtype=np.int32) * WORKLOAD["nw"]
    return p, Suspension(fil_start, X, Q, kap=1.0, c=1.0)


def run_reference(args, rank, world):
    """The CPU restatement of the reference on this host's cores. Each step (warm-up
    and timed) runs ONE stage of a Broyden iteration at full size, cycling through
    barrier, spread, forward FFTs, projection, inverse FFTs, interpolation, the rest
    of the iteration and the Jacobian build, so ms_per_step is what each step
    really took and every 8 steps cover one complete iteration and Jacobian build.
    value = beads / (jacobian + (iterations + 1) x iteration), with the stage times
    averaged over the timed steps (warm-up times for stages the timed window does
    not reach) and the iteration count of FP64_ITERS_BY_STEP over the window the GPU
    arms time."""
    if rank != 0:
        return None
    import numpy as np
    from oracle import oracle_py
    p, susp = reference_case()
    sysw = oracle_py.System(p, susp)
    sysw.initial_guess()
    sysw.filament_forces(1)
    K, W = args.steps, args.warmup
    seen = {k: [] for k in STAGE_CYCLE}
    warm = {k: [] for k in STAGE_CYCLE}
    timed = []
    nth = 1
    for i in range(W + K):
        st = STAGE_CYCLE[i % len(STAGE_CYCLE)]
        t0 = time.perf_counter()
        parts, nth = sysw.stage_costs([st], 1)
        dt = time.perf_counter() - t0
        (seen if i >= W else warm)[st].append(parts[st])
        if i >= W:
            timed.append(dt)
    # fewer than one cycle of steps: the stages not reached run once more, untimed
    for st in STAGE_CYCLE:
        if not seen[st] and not warm[st]:
            parts, nth = sysw.stage_costs([st], 1)
            warm[st].append(parts[st])
    sysw.close()
    stage_s = {k: float(np.mean(seen[k] if seen[k] else warm[k])) for k in STAGE_CYCLE}
    nt0 = PREP_STEPS + 1
    window = list(range(nt0 + W, nt0 + W + K))
    iters = float(np.mean([FP64_ITERS_BY_STEP[min(nt, len(FP64_ITERS_BY_STEP)) - 1] for nt in window]))
    step_s, per_iter = oracle_step_seconds(stage_s, iters)
    value = susp.np / step_s
    sample = ("CPU restatement of the reference (oracle/fs_oracle.c, OpenMP, %d threads; the reference binary, "
              "MPI + FFTW 2.1.5 + Armadillo, is not buildable here), inputs from the restated generator "
              "(oracle/or_suspension.c), no GPU library loaded. Each step is one full-size stage of a Broyden "
              "iteration of sediment_512, cycling through %s; a simulated step costs jacobian + (%.2f+1) "
              "iterations = %.1f s, %.2f the FP64 iteration count of steps %d-%d (bench.py FP64_ITERS_BY_STEP)"
              % (nth, ", ".join(STAGE_CYCLE), iters, step_s, iters, window[0], window[-1]))
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": float(np.mean(timed)) * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded rejection-placed filaments)",
            "config": {"workload": WORKLOAD["name"], "grid": [WORKLOAD["npts"]] * 3,
                       "filaments": WORKLOAD["nfil"], "beads_per_filament": WORKLOAD["nw"], "beads": susp.np,
                       "timed_steps": [window[0], window[-1]]},
            "impl": "reference",
            "steps_are": "one full-size oracle stage per step (cycle of %d: %s)" % (len(STAGE_CYCLE),
                                                                                    ", ".join(STAGE_CYCLE)),
            "seconds_per_simulated_step": step_s, "seconds_per_iteration": per_iter,
            "iters_per_step": iters, "stage_seconds": stage_s,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nth, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus)))
    if args.impl == "reference":
        out = run_reference(args, rank, world)
    elif args.workload == "mobility_256":
        out = run_mobility(args, rank, world) if rank == 0 else None
    elif args.workload == "ensemble_64":
        out = run_ensemble(args, rank, world)
    elif args.workload == "mlp":
        out = run_mlp(args, rank, world) if rank == 0 else None
    elif args.workload == "trajectory_200":
        out = run_trajectory(args, rank, world) if rank == 0 else None
    else:
        out = run_ours(args, rank, world)
    if rank == 0 and out is not None:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
