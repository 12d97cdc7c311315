"""Parity at the metric's size (512^3 NS+ACDI) through size-independent properties.

The bench workload itself is compared step for step with the C oracle in
tests/test_gpu_oracle_configs.py; these tests check, on a different input (an ABC velocity with
six drops), the identities that hold at any size and that the oracle comparison does not show.

* FP64 Poisson with the discrete Laplacian leaves a divergence at round-off
  (max |div| <= 1e-11 u_max n/2pi), the property that makes it the reference for matched
  divergence error.
* FP32 Poisson + one FP64 residual sweep reproduces that FP64 step to 1e-12.
* FP32 and FP64 Poisson with the reference's exact k^2 agree to FP32 rounding (1e-5 of u_max)
  and leave the same O(dx^2) divergence up to FP32 rounding of the divergence scale
  u_max n/2pi (two FP32 ulp: 1.2e-7 of it).
* The downloaded velocity has zero mean (the mean removal of multi/main.f90:977-981).
"""
import numpy as np
import pytest

from mhit36_mixedp_b200 import Params, Solver, synth

pytestmark = pytest.mark.gpu

N = 512


@pytest.fixture(scope="module")
def fields():
    u, v, w = synth.abc_velocity(N)
    phi = synth.drops_phi(N, synth.drop_centres(6, 4), 0.4, 2 * np.pi / N)
    return u, v, w, phi


def run(fields, nsteps=3, **kw):
    u, v, w, phi = fields
    prm = Params(nx=N, dt=2e-4, mu=0.003, phiflag=1, radius=0.4, sigma=0.3, acdi_clamp=1, **kw)
    with Solver(prm) as s:
        s.upload(u, v, w, phi)
        s.step(nsteps)
        out = s.download(fields=("u", "v", "w"))
        dg = s.diagnostics()
    return out, dg


def test_512_discrete_laplacian_divergence_and_refinement(gpu, fields):
    out64, dg64 = run(fields, poisson="fp64", laplacian="modified")
    umax = max(np.abs(out64[f]).max() for f in "uvw")
    assert dg64["maxdiv"] < 1e-11 * umax * N / (2 * np.pi), dg64["maxdiv"]
    for f in "uvw":
        assert abs(out64[f].mean()) < 1e-12 * umax
    outr, dgr = run(fields, poisson="fp32_refined", laplacian="modified")
    for f in "uvw":
        e = np.abs(outr[f] - out64[f]).max() / umax
        assert e < 1e-12, (f, e)
    assert dgr["maxdiv"] < 1e-11 * umax * N / (2 * np.pi)


def test_512_fp32_poisson_matches_fp64(gpu, fields):
    out64, dg64 = run(fields, poisson="fp64")
    out32, dg32 = run(fields, poisson="fp32")
    umax = max(np.abs(out64[f]).max() for f in "uvw")
    for f in "uvw":
        e = np.abs(out32[f] - out64[f]).max() / umax
        assert e < 1e-5, (f, e)
    assert abs(dg32["maxdiv"] - dg64["maxdiv"]) <= 1.2e-7 * umax * N / (2 * np.pi)
    assert abs(dg32["ke"] - dg64["ke"]) <= 1e-6 * dg64["ke"]
