"""Stage parity of the Poisson transforms at every length the scope-table configurations use.

The step tests run cubic boxes of 16-128 points and the Taylor-Green run 512^3; the 256^3
(NS+ACDI FP32 vs FP64), 1024^3 (NS) and 192^3 (ensemble) configurations need the 192-, 256-,
512- and 1024-point schedules on each axis, including the shared-memory-staged 256-point z
solve (``k_fft_cols_smem``) and the 512- and 1024-point x passes (M = 256, 512).  Each case is a
thin box with the length under test on one axis and 16 points on the other two, so it runs in
well under a second.

Every stage is checked in isolation: the stage runs on the GPU, and numpy (float64 pocketfft)
applies the same transform of ``multi/main.f90:853-912`` to the GPU's own input buffer of that
stage.  Tolerances are relative to the largest magnitude of the stage's output:
* FP64: 1e-12;
* FP32 storage: 4e-6 -- a few FP32 rounding steps per butterfly stage (eps32 = 6e-8), far below
  any indexing or twiddle error, which shows up at O(1) -- except the z solve, 3e-5: its divide
  by k^2 amplifies the forward transform's FP32 rounding at the smallest |k|, and on these thin
  boxes (1024 cells of dx along x, 16 along y and z) k^2 spans five decades.
The whole FP64 solve is also compared with the oracle's ``poisson_solve``.
"""
import numpy as np
import pytest

from mhit36_mixedp_b200 import Params, Solver, synth
from oracle import mhit_oracle as orc

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "fp32": 4e-6}


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def shapes():
    out = []
    for n in (192, 256, 512, 1024):
        out += [(n, 16, 16), (16, n, 16), (16, 16, n)]
    return out


def round32(a):
    if np.iscomplexobj(a):
        return a.astype(np.complex64).astype(np.complex128)
    return a.astype(np.float32).astype(np.float64)


@pytest.mark.parametrize("poisson", ["fp64", "fp32"])
@pytest.mark.parametrize("shape", shapes(), ids=lambda s: "x".join(map(str, s)))
def test_poisson_stages_at_length(gpu, shape, poisson):
    nx, ny, nz = shape
    prm = dict(nx=nx, ny=ny, nz=nz, dt=5e-4, mu=0.006, rho=1.0, poisson=poisson, laplacian="modified")
    u, v, w = synth.solenoidal_velocity(nx, 7, ny=ny, nz=nz)
    op = orc.Params(nx=nx, ny=ny, nz=nz, dt=5e-4, mu=0.006, rho=1.0, poisson=poisson, laplacian="modified")
    tol = TOL[poisson]
    f32 = poisson == "fp32"
    with Solver(Params(**prm)) as s:
        s.upload(u, v, w)
        s.run_stage("momentum")
        rhs = orc.poisson_rhs(op, s.buffer("un"), s.buffer("vn"), s.buffer("wn"))
        # x forward: rho/dt div u* (rounded to FP32 in the FP32 mode, :844), R2C along x (:853)
        s.run_stage("xfwd")
        want = np.fft.rfft(round32(rhs) if f32 else rhs, axis=2)
        got = s.buffer("spec")
        assert rel(got, want) < tol, ("xfwd", rel(got, want))
        # y forward (:860)
        prev = got
        s.run_stage("yfwd")
        got = s.buffer("spec")
        e = rel(got, np.fft.fft(prev, axis=1))
        assert e < tol, ("yfwd", e)
        # z forward, -1/k^2/N with the zero mode cleared, z inverse (:865, :883-896, :901)
        prev = got
        s.run_stage("zsolve")
        got = s.buffer("spec")
        hz = np.fft.fft(prev, axis=0)
        if f32:
            hz = round32(hz)
        with np.errstate(divide="ignore", invalid="ignore"):
            hz = -hz / orc.k2_table(op) / float(nx * ny * nz)
        hz[0, 0, 0] = 0.0
        if f32:
            hz = round32(hz)
        want = np.fft.ifft(hz, axis=0, norm="forward")
        e = rel(got, want)
        assert e < (3e-5 if f32 else tol), ("zsolve", e)
        # y inverse (:906)
        prev = got
        s.run_stage("yinv")
        got = s.buffer("spec")
        e = rel(got, np.fft.ifft(prev, axis=1, norm="forward"))
        assert e < tol, ("yinv", e)
        # x C2R into the pressure (:912); the imaginary parts of kx = 0 and nx/2 are ignored
        prev = got.copy()
        prev[:, :, 0] = prev[:, :, 0].real
        prev[:, :, -1] = prev[:, :, -1].real
        s.run_stage("xinv")
        got = s.buffer("p")
        e = rel(got, np.fft.irfft(prev, n=nx, axis=2, norm="forward"))
        assert e < tol, ("xinv", e)
        if not f32:
            e = rel(got, orc.poisson_solve(op, rhs))
            assert e < 1e-12, ("solve", e)
