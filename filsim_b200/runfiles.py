"""The reference's run files (.par, .bak, .dat) through libfilsim_gpu's host
code (fs_runfiles.cu), named as in file_functions.cpp:

  save_parameter_values_to_file   write_parameters   (.par)
  save_backup_data_to_file        save_backup        (.bak)
  continue_from_checkpoint        continue_from_checkpoint (.par layout + .bak)
  save_data_column_names_to_file  save_data_column_names (.dat header)
  save_data_to_file               save_data          (.dat row)

A run of this library therefore resumes the reference's checkpoints, the
reference resumes ours, and the .dat output feeds the reference's plotting
scripts. These calls need no GPU.
"""
import ctypes

import numpy as np

from .abi import FS_ERR_CAPACITY, FsRunInfo, check, lib
from .suspension import Suspension

RUN_INFO_DEFAULTS = dict(a=1.0, ah=1.0, dl=2.2, sp4=0.0, kap=1.0, c=1.0, mu=1.0, curvature=0.0, k0=0.0,
                         time_steps=0.0, steps_per_period=0.0, tol=1e-6, broyden_maxiter=100, plot_steps=1,
                         kap_network_filaments=0.0, bnumber=0.0, steps_per_settling_time=0.0, dt=0.0,
                         initial_friction_steps=0, enable_spring_links=0)


def run_info(name="filsim", tag="b200", p=None, **kw):
    """An fs_run_info; fields not given come from params p (when given) or the
    defaults above."""
    info = FsRunInfo()
    info.simulation_name = name.encode()[:127]
    info.simulation_tag = tag.encode()[:127]
    vals = dict(RUN_INFO_DEFAULTS)
    if p is not None:
        from .abi import box_lengths
        vals.update(a=p.a, ah=p.ah, dl=p.dl, mu=p.mu, tol=p.tol, broyden_maxiter=p.broyden_maxiter, dt=p.dt,
                    initial_friction_steps=p.initial_friction_steps)
        kw.setdefault("box", box_lengths(p))
        # fs_params holds (STRAINTWISTZ, X, Y); the .par columns are X, Y, Z
        kw.setdefault("strain_twist", (p.strain_twist[1], p.strain_twist[2], p.strain_twist[0]))
    vals.update(kw)
    for k, v in vals.items():
        if k in ("box", "strain_twist"):
            for i in range(3):
                getattr(info, k)[i] = float(v[i])
        else:
            setattr(info, k, v)
    return info


def write_parameters(path, susp, info):
    hs = susp.host_state()
    check(lib().fs_par_write(str(path).encode(), ctypes.byref(info), ctypes.byref(hs.struct)), "fs_par_write")


def read_layout(path, max_fil=1 << 24):
    """fil_start of the .par file's filaments."""
    nfil, np_ = ctypes.c_int(), ctypes.c_int()
    for cap in (1024, max_fil):
        fs = np.zeros(cap + 1, dtype=np.int32)
        st = lib().fs_par_read_layout(str(path).encode(), ctypes.byref(nfil), ctypes.byref(np_),
                                      fs.ctypes.data_as(ctypes.c_void_p), cap)
        if st == 0:
            return fs[: nfil.value + 1].copy()
        if st != FS_ERR_CAPACITY or cap == max_fil:  # too many filaments: retry with the full capacity
            check(st, "fs_par_read_layout")
    raise AssertionError("unreachable")


def save_backup(path, susp, nt):
    hs = susp.host_state()
    check(lib().fs_backup_write(str(path).encode(), ctypes.byref(hs.struct), nt), "fs_backup_write")


def read_backup(path, fil_start, kap=1.0, c=1.0):
    """A Suspension with the .bak file's state for layout fil_start, and the
    step to resume at (the file's nt + 1)."""
    fil_start = np.asarray(fil_start, dtype=np.int32)
    np_ = int(fil_start[-1])
    s = Suspension(fil_start, np.zeros((np_, 3)), np.tile([1.0, 0.0, 0.0, 0.0], (np_, 1)), kap=kap, c=c)
    hs = s.host_state()
    nt_next = ctypes.c_int()
    check(lib().fs_backup_read(str(path).encode(), ctypes.byref(hs.struct), ctypes.byref(nt_next)),
          "fs_backup_read")
    return s, nt_next.value


def continue_from_checkpoint(prefix, kap=1.0, c=1.0):
    """continue_from_checkpoint (file_functions.cpp:226-318): the layout from
    prefix.par, the state from prefix.bak; returns (Suspension, nt to resume at)."""
    fil_start = read_layout(str(prefix) + ".par")
    return read_backup(str(prefix) + ".bak", fil_start, kap=kap, c=c)


def save_data_column_names(path, susp):
    hs = susp.host_state()
    check(lib().fs_data_write_header(str(path).encode(), ctypes.byref(hs.struct)), "fs_data_write_header")


def save_data(path, susp, nt):
    hs = susp.host_state()
    check(lib().fs_data_append(str(path).encode(), ctypes.byref(hs.struct), nt), "fs_data_append")
