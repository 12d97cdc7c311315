"""The tensor-core 512-point z solve (zsolve_tc = 1) against numpy and against the Stockham path.

The z stage of the FP32 Poisson solve (forward z transform, -1/(k^2 N) with the zero mode
cleared, inverse z transform; multi/main.f90:865, :883-896, :901) runs as BF16x3-split DFT-matrix
GEMMs (16 x 32 factorisation) on tcgen05 with FP32 accumulation in tensor memory.  Checked:

* the stage alone, on the GPU's own input buffer, against numpy's float64 transform of it, at
  the FP32 z-solve tolerance of the Stockham path (3e-5 of the output's max; the divide by k^2
  amplifies the forward transform's rounding at the smallest |k|), and against the Stockham
  FP32 z solve on the same input;
* whole steps (NS+ACDI, exact and discrete Laplacian, plain and incremental FP32 solve) against
  the same steps with the Stockham z solve, to FP32 round-off of the velocity (1e-5 of its max).
"""
import numpy as np
import pytest

from mhit36_mixedp_b200 import MhitArgError, Params, Solver, synth
from oracle import mhit_oracle as orc

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def zsolve_output(shape, tc, laplacian="modified"):
    nx, ny, nz = shape
    u, v, w = synth.solenoidal_velocity(nx, 7, ny=ny, nz=nz)
    with Solver(Params(nx=nx, ny=ny, nz=nz, dt=5e-4, mu=0.006, poisson="fp32", laplacian=laplacian,
                       zsolve_tc=int(tc))) as s:
        s.upload(u, v, w)
        s.run_stage("momentum")
        s.run_stage("xfwd")
        s.run_stage("yfwd")
        before = s.buffer("spec")
        s.run_stage("zsolve")
        after = s.buffer("spec")
    return before, after


@pytest.mark.parametrize("shape", [(16, 16, 512), (64, 32, 512), (512, 16, 512)], ids=lambda s: "x".join(map(str, s)))
def test_tc_zsolve_stage(gpu, shape):
    nx, ny, nz = shape
    before, got = zsolve_output(shape, True)
    op = orc.Params(nx=nx, ny=ny, nz=nz, dt=5e-4, mu=0.006, laplacian="modified")
    hz = np.fft.fft(before, axis=0)
    with np.errstate(divide="ignore", invalid="ignore"):
        hz = -hz / orc.k2_table(op) / float(nx * ny * nz)
    hz[0, 0, 0] = 0.0
    want = np.fft.ifft(hz, axis=0, norm="forward")
    e = rel(got, want)
    before32, stock = zsolve_output(shape, False)
    np.testing.assert_array_equal(before32, before)
    e_stock = rel(stock, want)
    print(shape, "tensor-core z solve vs numpy", e, "Stockham FP32 vs numpy", e_stock)
    assert e < 3e-5, e
    assert rel(got, stock) < 3e-5


@pytest.mark.parametrize("poisson,laplacian", [("fp32", "exact"), ("fp32", "modified"),
                                               ("fp32_incremental", "modified")])
def test_tc_zsolve_steps(gpu, poisson, laplacian):
    n = (64, 64, 512)
    u, v, w = synth.solenoidal_velocity(n[0], 1, ny=n[1], nz=n[2])
    outs = {}
    for tc in (0, 1):
        with Solver(Params(nx=n[0], ny=n[1], nz=n[2], dt=2e-4, mu=0.006, poisson=poisson, laplacian=laplacian,
                           zsolve_tc=tc)) as s:
            s.upload(u, v, w)
            s.step(6)
            outs[tc] = (s.download(fields=("u", "v", "w")), s.diagnostics())
    for f in "uvw":
        e = rel(outs[1][0][f], outs[0][0][f])
        assert e < 1e-5, (f, e)
    d0, d1 = outs[0][1], outs[1][1]
    assert abs(d1["ke"] - d0["ke"]) <= 1e-6 * d0["ke"]
    if poisson == "fp32_incremental":
        assert d1["maxdiv"] <= 10 * d0["maxdiv"] + 1e-9, (d1["maxdiv"], d0["maxdiv"])


def test_tc_zsolve_needs_512_and_fp32(gpu):
    with pytest.raises(MhitArgError):
        Solver(Params(nx=16, ny=16, nz=256, poisson="fp32", zsolve_tc=1))
    with pytest.raises(MhitArgError):
        Solver(Params(nx=16, ny=16, nz=512, poisson="fp64", zsolve_tc=1))
