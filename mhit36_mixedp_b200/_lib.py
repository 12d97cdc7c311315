"""ctypes binding of libmhit_b200.so (the C ABI declared in include/mhit_b200.h).

The library is the product: there is no Python or CPU fallback.  ``load()`` raises if the
shared object is missing or lacks a symbol, so a missing build fails loudly.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmhit_b200.so")

MHIT_OK = 0
MHIT_ERR_ARG = -1
MHIT_ERR_CUDA = -2
MHIT_ERR_NAN = -3
MHIT_ERR_CFL = -4
MHIT_ERR_IO = -5
MHIT_ERR_STATE = -6
MHIT_ERR_TIMEOUT = -7
MHIT_STATS_NOALLOC_MAX_PLANES = 1024  # include/mhit_b200.h

POISSON = {"fp64": 0, "fp32": 1, "fp32_refined": 2, "fp32_incremental": 3}
LAPLACIAN = {"exact": 0, "modified": 1}
INTERP = {"linear1d": 0, "trilinear": 1}

# every function the header declares, with (restype, argtypes)
_c = ctypes
_P = _c.POINTER


class MhitParams(_c.Structure):
    _fields_ = [
        ("nx", _c.c_int), ("ny", _c.c_int), ("nz", _c.c_int),
        ("dt", _c.c_double), ("mu", _c.c_double), ("rho", _c.c_double),
        ("f1", _c.c_double), ("f2", _c.c_double), ("f3", _c.c_double), ("k0", _c.c_double),
        ("radius", _c.c_double), ("sigma", _c.c_double), ("epsr", _c.c_double),
        ("phiflag", _c.c_int), ("partflag", _c.c_int), ("npart", _c.c_int),
        ("poisson", _c.c_int), ("laplacian", _c.c_int), ("interp", _c.c_int),
        ("yz_shift", _c.c_int), ("use_graph", _c.c_int), ("device", _c.c_int), ("acdi_clamp", _c.c_int),
        ("zsolve_tc", _c.c_int),
    ]


class MhitRun(_c.Structure):
    _fields_ = [(n, _c.c_int) for n in ("restart", "tstart", "tfin", "dump", "inflow", "inphi", "inpart")]


class MhitDiag(_c.Structure):
    _fields_ = [
        ("nstep", _c.c_longlong), ("gumax", _c.c_double), ("cfl", _c.c_double),
        ("mean", _c.c_double * 3), ("maxdiv", _c.c_double), ("ke", _c.c_double),
        ("dissipation", _c.c_double), ("flags", _c.c_int),
    ]


class MhitDrop(_c.Structure):
    _fields_ = [("cells", _c.c_longlong), ("volume", _c.c_double), ("x", _c.c_double), ("y", _c.c_double),
                ("z", _c.c_double), ("u", _c.c_double), ("v", _c.c_double), ("w", _c.c_double)]


_dp = _P(_c.c_double)
SIGNATURES = {
    "mhit_abi_version": (_c.c_int, []),
    "mhit_last_error": (_c.c_char_p, []),
    "mhit_params_default": (_c.c_int, [_P(MhitParams)]),
    "mhit_read_input": (_c.c_int, [_c.c_char_p, _P(MhitParams), _P(MhitRun)]),
    "mhit_init": (_c.c_int, [_P(MhitParams), _P(_c.c_void_p)]),
    "mhit_destroy": (None, [_c.c_void_p]),
    "mhit_upload_fields": (_c.c_int, [_c.c_void_p, _dp, _dp, _dp, _dp]),
    "mhit_init_taylor_green": (_c.c_int, [_c.c_void_p]),
    "mhit_init_velocity_modes": (_c.c_int, [_c.c_void_p, _c.c_int, _dp, _c.c_double]),
    "mhit_init_drops": (_c.c_int, [_c.c_void_p, _c.c_int, _dp, _c.c_double]),
    "mhit_energy_spectrum": (_c.c_int, [_c.c_void_p, _dp, _c.c_int]),
    "mhit_init_particles": (_c.c_int, [_c.c_void_p, _c.c_int, _c.c_ulonglong]),
    "mhit_upload_particles": (_c.c_int, [_c.c_void_p, _dp, _c.c_int]),
    "mhit_download_particles": (_c.c_int, [_c.c_void_p, _dp, _c.c_int]),
    "mhit_step": (_c.c_int, [_c.c_void_p, _c.c_int]),
    "mhit_download_fields": (_c.c_int, [_c.c_void_p, _dp, _dp, _dp, _dp, _dp]),
    "mhit_diagnostics": (_c.c_int, [_c.c_void_p, _P(MhitDiag)]),
    "mhit_write_field": (_c.c_int, [_c.c_void_p, _c.c_char_p, _c.c_int, _c.c_int]),
    "mhit_read_field": (_c.c_int, [_c.c_void_p, _c.c_char_p, _c.c_int]),
    "mhit_write_checkpoint": (_c.c_int, [_c.c_void_p, _c.c_char_p]),
    "mhit_read_checkpoint": (_c.c_int, [_c.c_void_p, _c.c_char_p]),
    "mhit_label_drops": (_c.c_int, [_c.c_void_p, _c.c_double, _c.c_int, _P(MhitDrop), _c.c_int, _P(_c.c_int),
                                    _c.c_void_p]),
    "mhit_time_steps": (_c.c_int, [_c.c_void_p, _c.c_int, _dp]),
    "mhit_profile_step": (_c.c_int, [_c.c_void_p, _dp, _P(_c.c_char_p), _P(_c.c_int)]),
    "mhit_kernels_per_step": (_c.c_int, [_c.c_void_p, _P(_c.c_int)]),
    "mhit_ensemble_create": (_c.c_int, [_P(MhitParams), _c.c_int, _P(_c.c_void_p)]),
    "mhit_ensemble_destroy": (None, [_c.c_void_p]),
    "mhit_ensemble_box": (_c.c_int, [_c.c_void_p, _c.c_int, _P(_c.c_void_p)]),
    "mhit_ensemble_step": (_c.c_int, [_c.c_void_p, _c.c_int]),
    "mhit_ensemble_time_steps": (_c.c_int, [_c.c_void_p, _c.c_int, _dp]),
    "mhit_ensemble_autotune": (_c.c_int, [_c.c_void_p, _c.c_int, _P(_c.c_int)]),
    "mhit_ensemble_tuning": (_c.c_int, [_c.c_void_p, _P(_c.c_int), _P(_c.c_int), _P(_c.c_int)]),
    "mhit_ensemble_batched": (_c.c_int, [_c.c_void_p, _P(_c.c_int)]),
    "mhit_ensemble_set_batched": (_c.c_int, [_c.c_void_p, _c.c_int]),
    "mhit_field_stats_noalloc": (_c.c_int, [_c.c_int, _c.c_int, _c.c_int, _c.c_double, _c.c_void_p, _c.c_void_p,
                                            _c.c_void_p, _c.c_void_p, _c.c_void_p]),
    "mhit_debug_run_stage": (_c.c_int, [_c.c_void_p, _c.c_int]),
    "mhit_debug_commit_step": (_c.c_int, [_c.c_void_p]),
    "mhit_debug_set_label_bound": (_c.c_int, [_c.c_void_p, _c.c_longlong]),
    "mhit_debug_set_mom_tma": (_c.c_int, [_c.c_void_p, _c.c_int]),
    "mhit_debug_set_fused_projection": (_c.c_int, [_c.c_void_p, _c.c_int]),
    "mhit_debug_buffer_len": (_c.c_longlong, [_c.c_void_p, _c.c_int]),
    "mhit_debug_get_buffer": (_c.c_int, [_c.c_void_p, _c.c_int, _dp]),
}

STAGES = ["tracer", "phase", "momentum", "xfwd", "yfwd", "zsolve", "yinv", "xinv", "refine", "correct"]
BUFFERS = ["u", "v", "w", "un", "vn", "wn", "p", "phi", "phin", "ru", "rv", "rw", "rphi", "spec"]

_lib = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load the shared library once and attach the prototypes.  Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"libmhit_b200.so not built ({path}); run python -m mhit36_mixedp_b200.build")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)  # AttributeError if the symbol is not exported
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
