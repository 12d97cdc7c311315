"""CPU checks of the oracle's energy spectrum: Parseval, the Taylor-Green shell, and the weight of
the conjugate half of the real-to-complex spectrum."""
import numpy as np

from mhit36_mixedp_b200 import synth
from oracle import mhit_oracle as orc


def test_parseval_and_taylor_green_shell():
    u, v, w = orc.taylor_green(orc.Params(nx=32))
    E = orc.energy_spectrum(u, v, w, 40)
    assert abs(E[2] - 0.125) < 1e-15 and abs(E.sum() - orc.kinetic_energy(u, v, w)) < 1e-15
    u, v, w = synth.solenoidal_velocity(32, 4, kmax=4)
    E = orc.energy_spectrum(u, v, w, 40)
    assert abs(E.sum() - orc.kinetic_energy(u, v, w)) < 1e-13
    assert E[5:].sum() < 1e-25  # modes |k| <= 4 only: shells 1..4 (rounded |k| <= 4)
    assert E[0] < 1e-25


def test_single_mode_including_nyquist():
    n = 16
    x = np.arange(n) * 2 * np.pi / n
    # a kx = 3 mode and the x Nyquist mode (weight 1/2 in the half spectrum)
    u = (np.cos(3 * x)[None, None, :] + np.cos(8 * x)[None, None, :]) * np.ones((n, n, 1))
    z = np.zeros_like(u)
    E = orc.energy_spectrum(u, z, z, 20)
    assert abs(E[3] - 0.25) < 1e-15 and abs(E[8] - 0.5) < 1e-15
    assert abs(E.sum() - orc.kinetic_energy(u, z, z)) < 1e-15
