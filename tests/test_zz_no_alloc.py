"""The no-allocation statistics entry point against the allocating one.

mhit_field_stats_noalloc exists for callers that cannot let the library allocate device memory
(a host whose device arrays belong to its own runtime, or a run with the GPU's memory nearly
fully committed).  Through the C ABI it must return the same max|div u|, kinetic energy and
dissipation as mhit_diagnostics on the same fields, on consecutive calls (its scratch array is
shared and keeps the previous call's contents), and reject sizes beyond its scratch.
This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from mhit36_mixedp_b200 import Params, Solver, _lib, synth

pytestmark = pytest.mark.gpu
TOL = 1e-12


def noalloc_stats(lib, torch, u, v, w, nu):
    nz, ny, nx = u.shape
    du, dv, dw = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (u, v, w))
    out = torch.full((3,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = lib.mhit_field_stats_noalloc(nx, ny, nz, nu, ctypes.c_void_p(du.data_ptr()), ctypes.c_void_p(dv.data_ptr()),
                                      ctypes.c_void_p(dw.data_ptr()), ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 0, lib.mhit_last_error()
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_stats_match_diagnostics(gpu):
    import torch
    lib = _lib.load()
    nu = 0.006
    cases = [(64, 0, 0.0), (32, 5, 0.25)]  # two calls in a row, different fields and sizes
    for n, seed, shift in cases:
        u, v, w = synth.solenoidal_velocity(n, seed)
        u = u + shift
        with Solver(Params(nx=n, mu=nu, rho=1.0)) as s:
            s.upload(u, v, w)
            d = s.diagnostics()
        got = noalloc_stats(lib, torch, u, v, w, nu)
        want = np.array([d["maxdiv"], d["ke"], d["dissipation"]])
        rel = np.abs(got - want) / np.abs(want)
        assert np.all(rel < TOL), (n, got, want, rel)


def test_noalloc_rejects_too_many_planes(gpu):
    lib = _lib.load()
    big = _lib.MHIT_ERR_ARG
    dummy = ctypes.c_void_p(1)
    rc = lib.mhit_field_stats_noalloc(16, 16, 1025, 0.006, dummy, dummy, dummy, dummy, None)
    assert rc == big
    assert b"exceeds" in lib.mhit_last_error()
