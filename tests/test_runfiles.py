"""The reference's run files (.par, .bak, .dat; file_functions.cpp,
Filament.hpp:509-748) written and read by libfilsim_gpu's host code (CPU only)."""
import numpy as np
import pytest

from filsim_b200 import runfiles
from filsim_b200.configs import sediment_params
from filsim_b200.suspension import Suspension, random_suspension


def filled_suspension(fil_start, seed):
    rng = np.random.default_rng(seed)
    fil_start = np.asarray(fil_start, dtype=np.int32)
    np_ = int(fil_start[-1])
    q = rng.standard_normal((np_, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    s = Suspension(fil_start, 50 * rng.random((np_, 3)) - 10, q, kap=rng.uniform(0.5, 2.0, len(fil_start) - 1))
    for k in ("Xt", "U", "Ut"):
        s.arrays[k][...] = rng.standard_normal((np_, 3)) * (10.0 if k == "Xt" else 1e-3)
    qt = rng.standard_normal((np_, 4))
    s.arrays["qt"][...] = qt / np.linalg.norm(qt, axis=1, keepdims=True)
    for k in ("lam", "lam1", "lam2"):
        s.arrays[k][...] = rng.standard_normal(s.arrays[k].shape)
    s.arrays["qs"][...] = s.arrays["q"]
    return s


def test_backup_text_is_the_reference_layout(tmp_path):
    """nt, then per bead X Xt qs qt U Ut and per link lam lam1 lam2, each value
    "%.16f" (precision(16), ios::fixed) followed by one space, no newline."""
    s = filled_suspension([0, 2], 1)
    path = tmp_path / "run.bak"
    runfiles.save_backup(path, s, 17)
    want = "17 "
    for b in range(2):
        for k in ("X", "Xt", "qs", "qt", "U", "Ut"):
            want += "".join("%.16f " % v for v in s.arrays[k][b])
    for k in ("lam", "lam1", "lam2"):
        want += "".join("%.16f " % v for v in s.arrays[k][0])
    assert path.read_text() == want


def test_backup_round_trip(tmp_path):
    fil_start = [0, 5, 12, 13, 21]  # ragged, one single-bead filament
    s = filled_suspension(fil_start, 2)
    path = tmp_path / "run.bak"
    runfiles.save_backup(path, s, 240)
    r, nt_next = runfiles.read_backup(path, fil_start)
    assert nt_next == 241  # continue_from_checkpoint resumes at nt + 1
    for k in ("X", "Xt", "q", "qt", "U", "Ut", "lam", "lam1", "lam2"):
        assert np.abs(r.arrays[k] - s.arrays[k]).max() <= 1e-16 * max(1.0, np.abs(s.arrays[k]).max()), k
    for a, b in (("Xs", "X"), ("qs", "q"), ("Us", "U")):
        assert np.array_equal(r.arrays[a], r.arrays[b]), a
    # values of magnitude >= 1 survive the 16-decimal text exactly
    big = np.abs(s.arrays["X"]) >= 1
    assert np.array_equal(r.arrays["X"][big], s.arrays["X"][big])


def test_backup_read_rejects_short_or_corrupt_files(tmp_path):
    s = filled_suspension([0, 4, 8], 3)
    path = tmp_path / "run.bak"
    runfiles.save_backup(path, s, 3)
    text = path.read_text()
    (tmp_path / "short.bak").write_text(text[: len(text) // 2])
    (tmp_path / "bad.bak").write_text(text.replace(text.split(" ")[5], "x1.0", 1))
    from filsim_b200.abi import FsError
    for name in ("short.bak", "bad.bak", "missing.bak"):
        with pytest.raises(FsError):
            runfiles.read_backup(tmp_path / name, [0, 4, 8])


def _reference_par_reader(text):
    """continue_from_checkpoint's reading of a .par (file_functions.cpp:236-272),
    restated with its getline(..., ' ') steps."""
    pos = text.index("\n") + 1                          # line 1: ignore
    items = []
    for _ in range(3):                                  # three space-delimited items of line 2
        end = text.index(" ", pos)
        items.append(text[pos:end])
        pos = end + 1
    nsw = int(items[2])
    pos = text.index("\n", pos) + 1                     # rest of line 2
    pos = text.index("\n", pos) + 1                     # line 3
    pos = text.index("\n", pos) + 1                     # line 4
    beads = []
    for _ in range(nsw):
        end = text.find(" ", pos)
        tok = text[pos:] if end < 0 else text[pos:end]
        beads.append(int(tok.split()[0]))               # stoi stops at the first non-digit
        pos = end + 1
    return nsw, beads


def test_parameters_file(tmp_path):
    p = sediment_params(32)
    fil_start = [0, 8, 16, 20, 32]
    s = filled_suspension(fil_start, 4)
    info = runfiles.run_info("sediment", "b200", p=p, kap=1.5, sp4=12.0, time_steps=1000, plot_steps=10)
    path = tmp_path / "run.par"
    runfiles.write_parameters(path, s, info)
    text = path.read_text()
    lines = text.split("\n")
    assert lines[0].split()[:4] == ["SimulationName", "SimulationTag", "Nsw", "Nworm"]
    assert len(lines[0].split()) == len(lines[1].split()) == 39
    assert lines[1].split()[:4] == ["sediment", "b200", "4", "12"]
    assert lines[2] == "" and lines[3] == "BeadNumbers" and lines[4] == "8 8 4 12"
    assert lines[6] == "BendingModuli are KAP*"
    assert np.allclose([float(x) for x in lines[7].split()], s.kap / 1.5, rtol=1e-5)
    assert _reference_par_reader(text) == (4, [8, 8, 4, 12])
    assert np.array_equal(runfiles.read_layout(path), fil_start)


def test_data_file(tmp_path):
    s = filled_suspension([0, 3, 5], 5)
    path = tmp_path / "run.dat"
    runfiles.save_data_column_names(path, s)
    runfiles.save_data(path, s, 0)
    s.arrays["Xs"][...] += 1.0
    runfiles.save_data(path, s, 10)
    lines = path.read_text().split("\n")
    assert lines[0].split() == ["it"] + ["X", "Y", "Z", "qr", "qi", "qj", "qk"] * 5
    row = lines[2].split(" ")
    assert row[0] == "10"
    vals = np.array([float(x) for x in row[1:-1]]).reshape(5, 7)
    assert np.abs(vals[:, :3] - s.Xs).max() < 1e-15 * 100 and np.abs(vals[:, 3:] - s.qs).max() < 1e-16
    assert lines[3] == ""


def test_resume_from_checkpoint_on_the_oracle(oracle, tmp_path):
    """Five steps, a checkpoint, three more from the restored state: the same
    trajectory as eight uninterrupted steps, to the text format's precision."""
    p = sediment_params(32, tol=1e-12, broyden_maxiter=100)
    s = random_suspension(p, 4, 8, seed=81)
    full = oracle.System(p, s)
    full.run_steps(1, 8)
    part = oracle.System(p, s)
    part.run_steps(1, 5)
    s5 = s.copy()
    s5.set_arrays(part.download())
    runfiles.write_parameters(tmp_path / "run.par", s5, runfiles.run_info(p=p))
    runfiles.save_backup(tmp_path / "run.bak", s5, 5)
    r, nt_next = runfiles.continue_from_checkpoint(tmp_path / "run")
    assert nt_next == 6
    resumed = oracle.System(p, r)
    resumed.run_steps(nt_next, 3)
    a, b = resumed.download(), full.download()
    assert np.abs(a["X"] - b["X"]).max() < 1e-9
    assert np.abs(a["q"] - b["q"]).max() < 1e-9


def test_layout_capacity_is_reported(tmp_path):
    """A .par holding more filaments than the caller's capacity: FS_ERR_CAPACITY,
    and read_layout retries with a larger array."""
    import ctypes
    from filsim_b200 import abi
    s = filled_suspension([0, 2, 4, 6, 8, 10], 6)
    path = tmp_path / "run.par"
    runfiles.write_parameters(path, s, runfiles.run_info())
    nfil, np_ = ctypes.c_int(), ctypes.c_int()
    fs = np.zeros(3, dtype=np.int32)
    st = abi.lib().fs_par_read_layout(str(path).encode(), ctypes.byref(nfil), ctypes.byref(np_),
                                      fs.ctypes.data_as(ctypes.c_void_p), 2)
    assert st == abi.FS_ERR_CAPACITY
    assert np.array_equal(runfiles.read_layout(path), [0, 2, 4, 6, 8, 10])


def test_files_ignore_the_callers_numeric_locale(tmp_path):
    """A caller under a comma-decimal locale still gets the reference's '.'
    number format (C++ streams with the classic locale)."""
    import locale
    s = filled_suspension([0, 3], 7)
    ref = tmp_path / "c.bak"
    runfiles.save_backup(ref, s, 4)
    old = locale.setlocale(locale.LC_NUMERIC)
    for name in ("de_DE.UTF-8", "fr_FR.UTF-8", "de_DE.utf8"):
        try:
            locale.setlocale(locale.LC_NUMERIC, name)
            break
        except locale.Error:
            continue
    else:
        pytest.skip("no comma-decimal locale installed")
    try:
        out = tmp_path / "l.bak"
        runfiles.save_backup(out, s, 4)
        r, nt = runfiles.read_backup(out, [0, 3])
    finally:
        locale.setlocale(locale.LC_NUMERIC, old)
    assert out.read_text() == ref.read_text() and nt == 5
    assert np.array_equal(r.X[np.abs(s.X) >= 1], s.X[np.abs(s.X) >= 1])
