"""Ensembles of independent periodic boxes advanced together (fs_batch_*).

Workload ensemble_64: 64 boxes with grids drawn uniformly from {48^3, 64^3, 96^3,
128^3} and 8-256 filaments of 16 beads each, K_B log-uniform in [0.1, 10],
gravity (0,0,-1) per bead, dt = 0.05, BDF2. Filament counts are capped at a bead
volume fraction of 5% (48^3: 12, 64^3: 30, 96^3: 102, 128^3: 243): the uncapped
draw is not placeable (256 filaments of 16 beads fill 99.8% of a 48^3 box).

Each box is its own context (grid, parameters, suspension, stream, step start:
fs_set_start_order, fs_set_tension_extrapolation). After the start-up steps every
ensemble step is one CUDA graph launch holding every box's captured step, Broyden
loops on the device (fs_graph.cu). Over several GPUs the boxes are split by estimated cost
(partition_boxes), one ensemble per rank; the boxes are independent, so no
collective touches the data.
"""
import ctypes
import math

import numpy as np

from . import abi
from .abi import check, lib
from .configs import DX, sediment_params
from .fcm import Context, Simulation
from .suspension import random_suspension

GRIDS = (48, 64, 96, 128)
NW = 16
PHI_MAX = 0.05


def filament_cap(npts, nw=NW, phi=PHI_MAX, a=1.0):
    """Most filaments of nw beads in an npts^3 box at bead volume fraction phi."""
    L = npts * DX
    return int(phi * L ** 3 / (nw * 4.0 / 3.0 * math.pi * a ** 3))


def make_boxes(seed, nboxes=64, grids=GRIDS, nfil_range=(8, 256), nw=NW, kb_range=(0.1, 10.0),
               broyden_maxiter=100):
    """[(npts, params, suspension, K_B)] drawn as the workload states, seeded."""
    rng = np.random.default_rng(seed)
    boxes = []
    for i in range(nboxes):
        npts = int(rng.choice(grids))
        nfil = min(int(rng.integers(nfil_range[0], nfil_range[1] + 1)), filament_cap(npts, nw))
        kb = float(np.exp(rng.uniform(np.log(kb_range[0]), np.log(kb_range[1]))))
        p = sediment_params(npts, broyden_maxiter=broyden_maxiter)
        s = random_suspension(p, nfil, nw, seed=seed * 1000 + i, kap=kb)
        boxes.append((npts, p, s, kb))
    return boxes


def box_cost(npts, nbeads):
    """Estimated cost of one box-step: its FCM solves stream the grid (npts^3
    points) and spread/interpolate 12^3-point stencils per bead; iterations per
    step are not known in advance and are taken as equal across boxes."""
    return float(npts) ** 3 + 12.0 ** 3 * nbeads


def partition_boxes(boxes, world):
    """Boxes (the make_boxes tuples) split over `world` ranks by estimated cost:
    the most expensive box first, each to the rank with the least cost so far
    (ties to the lower rank). Returns, per rank, the indices of its boxes in
    ascending order; every box goes to exactly one rank."""
    cost = [box_cost(npts, s.np) for npts, _, s, _ in boxes]
    order = sorted(range(len(boxes)), key=lambda i: (-cost[i], i))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += cost[i]
    return [sorted(p) for p in parts]


class Ensemble:
    """One context per box, all advanced by fs_batch_run."""

    def __init__(self, boxes, precision=abi.FS_PREC_FP32, start_order=1, tension_order=2, escalate=0,
                 memory=None, predictor=0.0):
        self.boxes = boxes
        self.ctxs, self.sims = [], []
        for npts, p, s, kb in boxes:
            c = Context(p, max_beads=s.np, max_filaments=s.nfil)
            c.set_precision(precision)
            c.set_start_order(start_order)
            c.set_tension_extrapolation(tension_order)
            c.set_precision_escalation(escalate)
            if memory is not None:
                c.set_broyden_memory(*memory)  # (keep, carry, threshold, restart): fs_set_broyden_memory
            c.set_velocity_predictor(predictor)
            check(lib().fs_set_graph_mode(c.h, 1), "fs_set_graph_mode")
            self.ctxs.append(c)
            self.sims.append(Simulation(c, s))
        self.n = len(boxes)
        self.beads = np.array([s.np for _, _, s, _ in boxes])
        arr = (ctypes.c_void_p * self.n)(*[c.h.value for c in self.ctxs])
        h = ctypes.c_void_p()
        check(lib().fs_batch_create(arr, self.n, ctypes.byref(h)), "fs_batch_create")
        self.h = h

    def startup(self, nsteps):
        """The start-up steps (implicit Euler, constant/linear tension extrapolation), box by box."""
        for sim in self.sims:
            its, st = sim.run_steps(1, nsteps)
            if st not in (abi.FS_OK, abi.FS_ERR_NOT_CONVERGED):
                check(st, "fs_run_steps")

    def autotune(self, reps=3):
        """fs_autotune on the first box of each grid size; the other boxes of that size
        take its choice. Returns {grid: (spread chunk, interp beads per CTA, fft, spread
        column width, ms)}."""
        chosen = {}
        for (npts, p, s, kb), c in zip(self.boxes, self.ctxs):
            if npts not in chosen:
                ch = np.zeros(4, np.int32)
                ms = ctypes.c_float()
                check(lib().fs_autotune(c.h, reps, ch.ctypes.data_as(ctypes.c_void_p), ctypes.byref(ms)),
                      "fs_autotune")
                chosen[npts] = (ch, ms.value)
            else:
                check(lib().fs_set_tuning(c.h, chosen[npts][0].ctypes.data_as(ctypes.c_void_p)), "fs_set_tuning")
        return {g: (int(v[0][0]), int(v[0][1]), int(v[0][2]), int(v[0][3]), v[1]) for g, v in chosen.items()}

    def run(self, nt_start, nsteps):
        """(iterations [nsteps x n], per-box step ms [nsteps x n], total ms, status)."""
        its = np.zeros((nsteps, self.n), np.int32)
        ms = np.zeros((nsteps, self.n), np.float32)
        tot = ctypes.c_float()
        st = lib().fs_batch_run(self.h, nt_start, nsteps, its.ctypes.data_as(ctypes.c_void_p),
                                ms.ctypes.data_as(ctypes.c_void_p), ctypes.byref(tot))
        if st not in (abi.FS_OK, abi.FS_ERR_NOT_CONVERGED):
            check(st, "fs_batch_run")
        return its, ms, tot.value, st

    def close(self):
        if getattr(self, "h", None):
            lib().fs_batch_destroy(self.h)
            self.h = None
        for c in self.ctxs:
            c.close()
        self.ctxs = []
