"""B200-native (sm_100a) MHIT36 timestep hot path behind a C ABI.

``libmhit_b200.so`` (built from ``csrc/`` by ``build.py``) holds the CUDA kernels and the C ABI
declared in ``include/mhit_b200.h``; ``api`` is the Python host side over it (including the
reference's field-file and ``input.inp`` formats, read and written by the library), ``run`` the
time loop of ``program main``, ``synth`` the seeded synthetic initial conditions.
"""
from .api import (Ensemble, FIELD_P, FIELD_PHI, FIELD_U, FIELD_V, FIELD_W, MhitArgError, MhitCFLError,
                  MhitCudaError, MhitError, MhitIOError, MhitNaNError, MhitStateError, Params,
                  Solver, abi_version, read_input)

__all__ = [
    "Ensemble", "Params", "Solver", "read_input", "abi_version", "MhitError", "MhitArgError", "MhitCudaError",
    "MhitNaNError", "MhitCFLError", "MhitIOError", "MhitStateError",
    "FIELD_U", "FIELD_V", "FIELD_W", "FIELD_P", "FIELD_PHI",
]
