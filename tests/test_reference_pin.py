"""The oracle against the reference's own code (no GPU).

tests/golden/ref_pin.npz holds inputs and outputs of the reference's FCM
mobility solve (Fcm::mobility_solve, FCMfunctions.cpp:175-464) and collision
barrier (LinkedList::link + apply_collision_barrier,
CollisionBarrierFilament.cpp:24-433), compiled from the FilSim sources as one
process by oracle/refshim (written by tests/golden/make_ref_golden.py). The
oracle must give the same velocities to 1e-12 (the transforms differ: the
reference's stand-in FFT and the oracle's own) and the same barrier bit for
bit. Where the reference libraries are built (oracle/_ref), they must also
reproduce the fixture."""
import os

import numpy as np
import pytest

from filsim_b200.abi import make_params
from filsim_b200.configs import params_for
from filsim_b200.suspension import Suspension

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_pin.npz"))


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max()


@pytest.mark.parametrize("key,params", [("m64", lambda: params_for(64)),
                                        ("n20", lambda: make_params((48, 32, 64), ngd=20))])
def test_oracle_mobility_matches_the_reference_code(oracle, key, params):
    p = params()
    V, W = oracle.fcm_mobility(p, GOLD[key + "_Y"], GOLD[key + "_F"], GOLD[key + "_T"])
    assert rel(V, GOLD[key + "_V"]) < 1e-12
    assert rel(W, GOLD[key + "_W"]) < 1e-12


@pytest.mark.parametrize("key", ["b11", "b13"])
def test_oracle_barrier_matches_the_reference_code_bit_for_bit(oracle, key):
    p = params_for(32)
    nt = int(GOLD[key + "_nt"])
    if nt == 0:
        p.initial_friction_steps = 1
    X, F0, fil_start = GOLD[key + "_X"], GOLD[key + "_F0"], GOLD[key + "_fil_start"]
    s = Suspension(fil_start, X, np.tile([1.0, 0, 0, 0], (X.shape[0], 1)))
    head, lst, mp = oracle.cells_link(p, X)
    out = oracle.collision_barrier(p, np.fmod(X, 32 * p.dx), F0, s.fil_id, s.seg_id, head, lst, mp, nt)
    assert np.array_equal(head, GOLD[key + "_head"])
    assert np.array_equal(lst, GOLD[key + "_list"])
    assert np.array_equal(out["F"], GOLD[key + "_F"])
    assert out["min_dist2"] == float(GOLD[key + "_min_dist2"])
    assert np.abs(out["F"] - F0).max() > 1.0  # the barrier acted


def test_reference_libraries_reproduce_the_fixture(oracle):
    tags = ("fcm_64_ngd12", "fcm_48x32x64_ngd20", "barrier_32", "barrier_32_friction1")
    if not all(oracle.ref_available(t) for t in tags):
        pytest.skip("the reference libraries are built only where the FilSim sources are (oracle/refshim)")
    assert oracle.ref_config("fcm_64_ngd12")[:2] == ((64, 64, 64), 12)
    for key, tag in (("m64", "fcm_64_ngd12"), ("n20", "fcm_48x32x64_ngd20")):
        V, W = oracle.ref_fcm_mobility(tag, GOLD[key + "_Y"], GOLD[key + "_F"], GOLD[key + "_T"])
        assert np.array_equal(V, GOLD[key + "_V"]) and np.array_equal(W, GOLD[key + "_W"])
    for key, tag in (("b11", "barrier_32"), ("b13", "barrier_32_friction1")):
        X = GOLD[key + "_X"]
        F, head, lst, md = oracle.ref_barrier(tag, GOLD[key + "_fil_start"], X, np.fmod(X, 32 * params_for(32).dx),
                                              GOLD[key + "_F0"], int(GOLD[key + "_nt"]))
        assert np.array_equal(F, GOLD[key + "_F"]) and md == float(GOLD[key + "_min_dist2"])
