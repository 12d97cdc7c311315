"""Energy spectrum on the device (mhit_energy_spectrum) against the oracle's numpy restatement,
Parseval against the kinetic energy of the diagnostics, and the Taylor-Green start's single
shell."""
import numpy as np
import pytest

from mhit36_mixedp_b200 import Params, Solver
from oracle import mhit_oracle as orc

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape,poisson", [((32, 32, 32), "fp64"), ((32, 16, 64), "fp64"), ((32, 32, 32), "fp32"),
                                           ((64, 64, 64), "fp32_refined")])
def test_spectrum_matches_oracle(gpu, shape, poisson):
    nx, ny, nz = shape
    lap = "modified" if poisson == "fp32_refined" else "exact"
    with Solver(Params(nx=nx, ny=ny, nz=nz, poisson=poisson, laplacian=lap, f1=1.0, f2=0.5, f3=0.25)) as s:
        s.init_solenoidal(seed=5, kmax=3)
        s.step(4)  # the forcing leaves a lazily removed mean in the stored velocity
        nb = s.energy_spectrum().size
        E = s.energy_spectrum()
        E8 = s.energy_spectrum(8)
        out = s.download(("u", "v", "w"))
        ke = s.diagnostics()["ke"]
    ref = orc.energy_spectrum(out["u"], out["v"], out["w"], nb)
    assert np.max(np.abs(E - ref)) <= 1e-12 * ref.sum()
    assert np.max(np.abs(E8 - ref[:8])) <= 1e-12 * ref.sum()
    assert abs(E.sum() - ke) <= 1e-12 * ke


def test_taylor_green_energy_sits_in_shell_two(gpu):
    n = 64
    with Solver(Params(nx=n)) as s:
        s.init_taylor_green()
        E = s.energy_spectrum()
    # sin x cos y cos z and cos x sin y cos z: wavevectors (+-1, +-1, +-1), |k| = sqrt(3) -> shell 2
    assert abs(E[2] - 0.125) <= 1e-15
    assert np.sum(np.delete(E, 2)) <= 1e-28


def test_spectrum_rejects_bad_arguments(gpu):
    with Solver(Params(nx=16)) as s:
        with pytest.raises(Exception):
            s.energy_spectrum(0)
        with pytest.raises(Exception):
            s.energy_spectrum(5000)
