"""B200-native fTWA / time-dependent Hartree-Fock trajectory engine.

The compute path is libfpsg.so (hand-written sm_100a CUDA kernels behind the C ABI
of include/fpsg.h); the C++ host layer (libfpshost.so, the `fps` CLI) mirrors
FermiPhaseSpace's FHSystem / FHfTWASolver / FHHFSolver interface on top of it.
"""
from .engine import (  # noqa: F401
    Engine, FpsgError, RunResult, load,
    METHOD_FTWA, METHOD_HF, PREC_FP64, PREC_FP32, PREC_SPLIT_BF16X3, PREC_SPLIT_TF32X3,
    COUL_NULL, COUL_ONSITE, COUL_DISTANCE, PATH_AUTO, PATH_STREAM, PATH_RESIDENT, PATH_DENSE,
    OBS_DIAG, OBS_DIAG2, OBS_DOUBLONS, OBS_WHOLE, OBS_ENERGIES, OBS_DEFAULT,
)

__version__ = "0.1.0"
