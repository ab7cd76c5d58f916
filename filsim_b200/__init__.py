"""filsim_b200: B200 (sm_100a) implementation of FilSim's FCM mobility +
collision barrier + implicit BDF2/Broyden step behind a C-ABI.
"""
from .abi import (FsParams, FsDiag, FsHostState, FsError, make_params, box_lengths, lib,
                  FS_PREC_FP64, FS_PREC_FP32)
