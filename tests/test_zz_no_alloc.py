"""The no-allocation statistics entry point against the allocating one.

mhit_field_stats_noalloc exists for callers that cannot let the library allocate device memory
(a host whose device arrays belong to its own runtime, or a run with the GPU's memory nearly
fully committed).  Through the C ABI it must return the same max|div u|, kinetic energy and
dissipation as mhit_diagnostics on the same fields, on consecutive calls (its scratch array is
shared and keeps the previous call's contents), on the default stream and on a caller's stream,
at the largest plane count its scratch holds; it must leave the device's free memory unchanged
once its module is loaded, turn a NaN in the fields into a NaN max|div u|, and reject sizes
beyond its scratch.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from mhit36_mixedp_b200 import Params, Solver, _lib, synth

pytestmark = pytest.mark.gpu
TOL = 1e-12


def device_fields(torch, u, v, w):
    du, dv, dw = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (u, v, w))
    out = torch.full((3,), float("nan"), dtype=torch.float64, device="cuda")
    return du, dv, dw, out


def call(lib, shape, du, dv, dw, out, nu, stream=None):
    nz, ny, nx = shape
    rc = lib.mhit_field_stats_noalloc(nx, ny, nz, nu, ctypes.c_void_p(du.data_ptr()), ctypes.c_void_p(dv.data_ptr()),
                                      ctypes.c_void_p(dw.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                      None if stream is None else ctypes.c_void_p(stream))
    assert rc == 0, lib.mhit_last_error()


def noalloc_stats(lib, torch, u, v, w, nu, stream=None):
    du, dv, dw, out = device_fields(torch, u, v, w)
    torch.cuda.synchronize()
    call(lib, u.shape, du, dv, dw, out, nu, stream)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def diagnostics(u, v, w, nu):
    nz, ny, nx = u.shape
    with Solver(Params(nx=nx, ny=ny, nz=nz, mu=nu, rho=1.0)) as s:
        s.upload(u, v, w)
        d = s.diagnostics()
    return np.array([d["maxdiv"], d["ke"], d["dissipation"]])


def test_noalloc_stats_match_diagnostics(gpu):
    import torch
    lib = _lib.load()
    nu = 0.006
    cases = [((64, 64, 64), 0, 0.0), ((32, 32, 32), 5, 0.25)]  # two calls in a row, different fields and sizes
    for (nx, ny, nz), seed, shift in cases:
        u, v, w = synth.solenoidal_velocity(nx, seed, ny=ny, nz=nz)
        u = u + shift
        got = noalloc_stats(lib, torch, u, v, w, nu)
        want = diagnostics(u, v, w, nu)
        rel = np.abs(got - want) / np.abs(want)
        assert np.all(rel < TOL), ((nx, ny, nz), got, want, rel)


def test_noalloc_max_planes_on_a_caller_stream(gpu):
    """nz = 1024 (the scratch's capacity) on a non-cubic box, launched on a torch stream."""
    import torch
    lib = _lib.load()
    nu = 0.004
    u, v, w = synth.solenoidal_velocity(16, 3, ny=16, nz=_lib.MHIT_STATS_NOALLOC_MAX_PLANES)
    want = diagnostics(u, v, w, nu)
    s = torch.cuda.Stream()
    for _ in range(2):
        got = noalloc_stats(lib, torch, u, v, w, nu, stream=s.cuda_stream)
        rel = np.abs(got - want) / np.abs(want)
        assert np.all(rel < TOL), (got, want, rel)


def test_noalloc_allocates_nothing(gpu):
    """After a warm-up call (which may load the library's kernels), a call leaves the device's
    free memory unchanged: it neither allocates nor frees."""
    import torch
    lib = _lib.load()
    u, v, w = synth.solenoidal_velocity(64, 9)
    du, dv, dw, out = device_fields(torch, u, v, w)
    torch.cuda.synchronize()
    call(lib, u.shape, du, dv, dw, out, 0.006)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    call(lib, u.shape, du, dv, dw, out, 0.006)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert np.all(np.isfinite(out.cpu().numpy()))


def test_noalloc_nan_field(gpu):
    import torch
    lib = _lib.load()
    u, v, w = synth.solenoidal_velocity(32, 4)
    u[5, 6, 7] = np.nan
    got = noalloc_stats(lib, torch, u, v, w, 0.006)
    assert np.isnan(got[0]) and np.isnan(got[1]), got


def test_noalloc_rejects_too_many_planes(gpu):
    lib = _lib.load()
    dummy = ctypes.c_void_p(1)
    rc = lib.mhit_field_stats_noalloc(16, 16, _lib.MHIT_STATS_NOALLOC_MAX_PLANES + 1, 0.006, dummy, dummy, dummy, dummy,
                                      None)
    assert rc == _lib.MHIT_ERR_ARG
    assert b"exceeds" in lib.mhit_last_error()
