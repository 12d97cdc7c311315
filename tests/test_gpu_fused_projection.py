"""The inverse x transform fused with the projection (k_xinv_correct) against the two passes.

By default a step transforms the y-inverted spectrum back along x inside the projection
(multi/main.f90:909-912 and :942-1003 in one pass), so the pressure never reaches HBM during
the step; it is transformed into its array, with the same arithmetic, only when something reads
it.  The test hook ``mhit_debug_set_fused_projection(ctx, 0)`` runs the two passes apart.

* Both must give the same fields up to rounding: the fused pass transforms in a radix-8
  schedule (the separate pass in radix 16 at nx = 256 and 512), its butterflies may contract
  multiply-adds differently, and it sums the per-block means over other blocks.  Bars, relative to
  each field's max: FP64 1e-13.  In the FP32 modes the two differ by FP32 rounding of the
  pressure (~6e-8 of it), which moves u by dt/rho dp/dx every step: the bars are those the FP32
  modes meet elsewhere (1e-7 for the fields against the FP64 step, 1e-4 for the FP32 pressure
  against the oracle: the first steps' FP32 solves carry rounding of the whole pressure).  The
  projected divergence must be as small either way.
  For every Poisson mode that fuses (FP64, FP32, incremental FP32), on cubic and non-cubic boxes
  whose ny is not a multiple of the fused pass's 7 lines per block (tail blocks), at nx = 192 (the
  radix-3 schedule) and nx = 1024 (the pressure carried in registers instead of shared memory),
  and at 256^3, the production tile shapes.
* The pressure must be the one the projection used: a download after a step equals a download
  after a call that reuses the spectrum (droplet labelling, energy spectrum) and after a second
  download, bit for bit.
"""
import numpy as np
import pytest

from mhit36_mixedp_b200 import Params, Solver, _lib, synth

pytestmark = pytest.mark.gpu


def tol(poisson, field):
    if poisson == "fp64":
        return 1e-13
    return 1e-4 if field == "p" else 1e-7


def check(shape, poisson, nsteps):
    a, da = run(shape, poisson, True, nsteps)
    b, db = run(shape, poisson, False, nsteps)
    for k in b:
        e = relerr(a[k], b[k])
        assert e < tol(poisson, k), (k, e)
    assert abs(da["gumax"] - db["gumax"]) <= tol(poisson, "u") * abs(db["gumax"])
    # the projected divergence is as small either way (a maximum over all cells)
    assert da["maxdiv"] <= 3 * db["maxdiv"] + 1e-13, (da["maxdiv"], db["maxdiv"])


def relerr(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def run(shape, poisson, fused, nsteps=4):
    nx, ny, nz = shape
    phiflag = int(nx == ny == nz)  # the host drop field is cubic; the projection does not read phi
    u, v, w = synth.solenoidal_velocity(nx, 5, ny=ny, nz=nz)
    phi = synth.drops_phi(nx, synth.drop_centres(6, 2), 0.4, 2 * np.pi / nx) if phiflag else None
    lap = "modified" if poisson == "fp32_incremental" else "exact"
    prm = Params(nx=nx, ny=ny, nz=nz, dt=2e-4, mu=0.004, phiflag=phiflag, radius=0.4, sigma=0.3, acdi_clamp=1,
                 poisson=poisson, laplacian=lap)
    with Solver(prm) as s:
        assert _lib.load().mhit_debug_set_fused_projection(s._ctx, int(fused)) == 0
        s.upload(u, v, w, phi)
        s.step(nsteps)
        out = s.download()
        dg = s.diagnostics()
    return out, dg


@pytest.mark.parametrize("poisson", ["fp64", "fp32", "fp32_incremental"])
@pytest.mark.parametrize("shape", [(64, 64, 64), (32, 16, 64), (64, 192, 32), (192, 32, 16), (1024, 16, 16)])
def test_fused_matches_separate_passes(gpu, shape, poisson):
    check(shape, poisson, 4)


@pytest.mark.parametrize("poisson", ["fp64", "fp32_incremental"])
def test_fused_matches_separate_passes_256(gpu, poisson):
    check((256, 256, 256), poisson, 3)


@pytest.mark.parametrize("poisson", ["fp64", "fp32_incremental"])
def test_pressure_survives_calls_that_reuse_the_spectrum(gpu, poisson):
    n = 64
    u, v, w = synth.solenoidal_velocity(n, 5)
    phi = synth.drops_phi(n, synth.drop_centres(6, 2), 0.4, 2 * np.pi / n)
    lap = "modified" if poisson == "fp32_incremental" else "exact"
    with Solver(Params(nx=n, dt=2e-4, mu=0.004, phiflag=1, radius=0.4, sigma=0.3, poisson=poisson,
                       laplacian=lap)) as s:
        s.upload(u, v, w, phi)
        s.step(3)
        s.label_drops()
        p1 = s.download(fields=("p",))["p"]
        s.energy_spectrum()
        p2 = s.download(fields=("p",))["p"]
        p3 = s.download(fields=("p",))["p"]
        np.testing.assert_array_equal(p1, p2)
        np.testing.assert_array_equal(p1, p3)
        # and the state the next step reads is untouched: continuing matches a run without the calls
        s.step(2)
        got = s.download()
    with Solver(Params(nx=n, dt=2e-4, mu=0.004, phiflag=1, radius=0.4, sigma=0.3, poisson=poisson,
                       laplacian=lap)) as s:
        s.upload(u, v, w, phi)
        s.step(3)
        q1 = s.download(fields=("p",))["p"]
        s.step(2)
        ref = s.download()
    np.testing.assert_array_equal(p1, q1)
    for k in ref:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
