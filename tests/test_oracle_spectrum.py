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


def test_seeded_particles_follow_splitmix64():
    """synth.seeded_particles (the numpy twin of mhit_init_particles) against a pure-integer
    restatement of splitmix64."""
    M = (1 << 64) - 1
    G = 0x9E3779B97F4A7C15

    def mix(z):
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        return z ^ (z >> 31)

    seed = 12345
    lengths = (2 * np.pi, np.pi, 4 * np.pi)
    part = synth.seeded_particles(50, seed, lengths)
    for i in (0, 1, 17, 49):
        for a in range(3):
            r = mix((seed + (3 * i + a + 1) * G) & M)
            assert part[i, 1 + a] == (r >> 11) * 2.0 ** -53 * lengths[a]
    assert np.array_equal(part[:, 0], np.arange(1, 51)) and not part[:, 4:].any()
    for a in range(3):
        assert (part[:, 1 + a] >= 0).all() and (part[:, 1 + a] < lengths[a]).all()


def test_solenoidal_modes_are_divergence_free_in_the_box_metric():
    """k . c = 0 with the physical wavenumbers of a box nx dx by ny dx by nz dx, and the
    non-cubic field holds only index wavenumbers |m| <= kmax along each axis (periodic)."""
    kmax = 3
    scale = (1.0, 2.0, 0.5)  # nx/ny, nx/nz for nx = 32, ny = 16, nz = 64
    c = synth.solenoidal_modes(9, kmax, scale)
    ks = np.arange(-kmax, kmax + 1)
    KZ, KY, KX = np.meshgrid(ks, ks, ks, indexing="ij")
    kdotc = KX * scale[0] * c[0] + KY * scale[1] * c[1] + KZ * scale[2] * c[2]
    assert np.max(np.abs(kdotc)) < 1e-12 * np.max(np.abs(c))
    u, v, w = synth.solenoidal_velocity(32, 9, kmax=kmax, ny=16, nz=64)
    for f in (u, v, w):
        F = np.abs(np.fft.fftn(f))
        mz = np.abs(np.fft.fftfreq(64, 1 / 64))[:, None, None]
        my = np.abs(np.fft.fftfreq(16, 1 / 16))[None, :, None]
        mx = np.abs(np.fft.fftfreq(32, 1 / 32))[None, None, :]
        outside = (mx > kmax) | (my > kmax) | (mz > kmax)
        assert F[np.broadcast_to(outside, F.shape)].max() < 1e-9 * F.max()
