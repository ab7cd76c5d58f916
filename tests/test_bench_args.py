"""bench.py's command line on CPU (no GPU is touched): the step options of the
value arm (--broyden-memory, --velocity-predictor, --escalate) and the profiling
grids (--grid N or NX,NY,NZ), and their labels in the JSON config."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture()
def bench(monkeypatch):
    # parse() rewrites the workload tables it is given a grid for: restore them after
    import copy
    from filsim_b200 import configs
    saved = copy.deepcopy(configs.WORKLOADS)
    yield_mod = _load(monkeypatch)
    yield yield_mod
    configs.WORKLOADS.clear()
    configs.WORKLOADS.update(saved)


def _load(monkeypatch):
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)

    def parse(*argv):
        monkeypatch.setattr(sys, "argv", ["bench.py", *argv])
        return mod.parse()
    mod.parse_args = parse
    return mod


def test_defaults(bench):
    a = bench.parse_args()
    assert a.workload == "sediment_512" and a.gpus == 1
    assert a.memory == bench.MEMORY_DEFAULT == (16, 4, 8, 30)
    assert a.velocity_predictor == bench.PREDICTOR_DEFAULT == 0.5
    assert a.escalate == 0 and a.start_order == 2 and a.tension_order == 1


def test_step_options(bench):
    a = bench.parse_args("--broyden-memory", "0", "--velocity-predictor", "0", "--escalate", "15")
    assert a.memory == bench.MEMORY_OFF and a.velocity_predictor == 0.0 and a.escalate == 15
    assert "reference" in bench.memory_label(a.memory)
    a = bench.parse_args("--broyden-memory", "8:3:4:12")
    assert a.memory == (8, 3, 4, 12)
    assert "8 history columns" in bench.memory_label(a.memory) and "restart at 12" in bench.memory_label(a.memory)
    with pytest.raises(SystemExit):
        bench.parse_args("--broyden-memory", "8:3")


def test_grids(bench):
    a = bench.parse_args("--workload", "mobility_256", "--grid", "128,128,512", "--filaments", "64")
    assert a.grid == (128, 128, 512)
    from filsim_b200.configs import WORKLOADS
    assert WORKLOADS["mobility_256"]["name"] == "mobility_128x128x512_64x30"
    a = bench.parse_args("--grid", "384", "--filaments", "1728")
    assert a.grid == 384 and bench.WORKLOAD["name"] == "sediment_384_1728x32"
    with pytest.raises(SystemExit):
        bench.parse_args("--grid", "128,128,512")  # three lengths only for the mobility workload
    assert bench.warp_fft_length(384) and bench.warp_fft_length(512) and not bench.warp_fft_length(48)
