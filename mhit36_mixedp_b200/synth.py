"""Seeded synthetic initial conditions (numpy, host side).

The reference reads such fields through its ``inflow=1`` / ``inphi=1`` file path
(multi/main.f90:338-343, 383-386) or builds Taylor-Green / one centred drop
(multi/main.f90:324-337, 370-382).  The generators here produce the inputs of the benchmark
configurations with explicit seeds (``numpy.random.default_rng``):

* ``solenoidal_velocity``: random Fourier modes 0 < |k| <= kmax with complex Gaussian
  amplitudes, Leray-projected (k . c = 0), sampled at the staggered face positions of the
  reference (u at x - dx/2 as in multi/main.f90:331, v at y - dx/2, w at z - dx/2) and scaled
  to unit rms per component.
* ``drops_phi``: phi = 0.5 (1 - tanh((r - R)/(2 eps))) with r the minimum-image distance to the
  nearest of ``ndrops`` uniformly placed centres (the max over spheres of the single-drop
  profile of multi/main.f90:377-378; distances are capped at R + 40 eps, where phi < 1e-17).
* ``uniform_particles``: the tracer table of multi/particles.f90:46-72 with seeded positions;
  ``seeded_particles``: the same table from the counter-based generator of mhit_init_particles.

Grid coordinates use the reference labelling: x = i dx, y = (j + s) dx, z = (k + s) dx with
s = yz_shift (1 for the reference, see multi/main.f90:327-331).
"""
from __future__ import annotations

import math

import numpy as np

LX = 8.0 * math.atan(1.0)


def _coords(n, s):
    dx = LX / n
    return (np.arange(n) + s) * dx


def solenoidal_modes(seed, kmax=4, scale=(1.0, 1.0, 1.0)):
    """The complex amplitudes c[component][kz][ky][kx] (index wavenumbers m from -kmax) of
    ``solenoidal_velocity``: Gaussian on 0 < |m| <= kmax, Leray-projected (k . c = 0) with the
    physical wavenumbers k = (m_x, m_y, m_z) * scale; scale = (1, nx/ny, nx/nz) for a box of
    nx dx by ny dx by nz dx (all ones for a cube)."""
    rng = np.random.default_rng(seed)
    ks = np.arange(-kmax, kmax + 1)
    KZ, KY, KX = np.meshgrid(ks, ks, ks, indexing="ij")
    m2 = KX ** 2 + KY ** 2 + KZ ** 2
    mask = (m2 > 0) & (m2 <= kmax * kmax)
    c = (rng.standard_normal((3,) + KX.shape) + 1j * rng.standard_normal((3,) + KX.shape)) * mask
    kv = np.stack([KX * float(scale[0]), KY * float(scale[1]), KZ * float(scale[2])])
    k2 = (kv * kv).sum(axis=0)
    with np.errstate(invalid="ignore", divide="ignore"):
        kdotc = (kv * c).sum(axis=0) / np.where(m2 > 0, k2, 1)
    c = c - kv * kdotc[None]
    return c * mask


def solenoidal_velocity(nx, seed, kmax=4, rms=1.0, yz_shift=1, ny=None, nz=None):
    ny = ny or nx
    nz = nz or nx
    ks = np.arange(-kmax, kmax + 1)
    c = solenoidal_modes(seed, kmax, (1.0, nx / ny, nx / nz))
    # index phase theta = (i + s) 2 pi / n per axis (the physical coordinate times the lowest
    # wavenumber of that axis); the component's own axis is sampled half a cell back
    x = _coords(nx, 0)
    y = _coords(ny, yz_shift)
    z = _coords(nz, yz_shift)
    out = []
    for comp in range(3):
        xs = x - (LX / nx) / 2 if comp == 0 else x
        ys = y - (LX / ny) / 2 if comp == 1 else y
        zs = z - (LX / nz) / 2 if comp == 2 else z
        ex = np.exp(1j * np.outer(xs, ks))   # (nx, K)
        ey = np.exp(1j * np.outer(ys, ks))   # (ny, K)
        ez = np.exp(1j * np.outer(zs, ks))   # (nz, K)
        a = c[comp] @ ex.T                    # (Kz, Ky, nx)
        b = np.einsum("jY,ZYi->Zji", ey, a)   # (Kz, ny, nx)
        b = b.reshape(len(ks), ny * nx)
        f = np.empty((nz, ny * nx))
        for z0 in range(0, nz, 64):
            z1 = min(nz, z0 + 64)
            f[z0:z1] = ez[z0:z1].real @ b.real - ez[z0:z1].imag @ b.imag
        f = f.reshape(nz, ny, nx)
        f *= rms / math.sqrt(float(np.mean(f * f)))
        out.append(f)
    return tuple(out)


def drop_centres(ndrops, seed):
    rng = np.random.default_rng(seed)
    return rng.uniform(0.0, LX, size=(ndrops, 3))


def drops_phi(nx, centres, radius, eps, yz_shift=1):
    n = nx
    dx = LX / n
    cap = radius + 40.0 * eps
    x = _coords(n, 0)
    y = _coords(n, yz_shift)
    z = _coords(n, yz_shift)
    rmin = np.full((n, n, n), cap)
    h = int(math.ceil(cap / dx)) + 1
    for cx, cy, cz in centres:
        ix = int(round(cx / dx))
        iy = int(round(cy / dx - yz_shift))
        iz = int(round(cz / dx - yz_shift))
        ii = np.arange(ix - h, ix + h + 1) % n
        jj = np.arange(iy - h, iy + h + 1) % n
        kk = np.arange(iz - h, iz + h + 1) % n
        if len(np.unique(ii)) < len(ii):
            ii, jj, kk = np.arange(n), np.arange(n), np.arange(n)
        ddx = x[ii] - cx
        ddy = y[jj] - cy
        ddz = z[kk] - cz
        ddx -= LX * np.round(ddx / LX)
        ddy -= LX * np.round(ddy / LX)
        ddz -= LX * np.round(ddz / LX)
        r = np.sqrt(ddz[:, None, None] ** 2 + ddy[None, :, None] ** 2 + ddx[None, None, :] ** 2)
        sub = rmin[np.ix_(kk, jj, ii)]
        rmin[np.ix_(kk, jj, ii)] = np.minimum(sub, r)
    return 0.5 * (1.0 - np.tanh((rmin - radius) / 2.0 / eps))


def uniform_particles(npart, seed):
    rng = np.random.default_rng(seed)
    part = np.zeros((npart, 12), dtype=np.float64, order="F")
    part[:, 0] = np.arange(1, npart + 1)
    part[:, 1:4] = rng.uniform(0.0, LX, size=(npart, 3))
    return part


_GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def _splitmix64(z):
    """The splitmix64 finaliser (Steele, Lea and Flood, OOPSLA 2014) on a uint64 array."""
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def seeded_particles(npart, seed, lengths=(LX, LX, LX)):
    """The tracer table that mhit_init_particles builds on the device (multi/particles.f90:37-76
    with a reproducible generator): coordinate a of tracer i is
    lengths[a] * (top 53 bits of splitmix64(seed + (3 i + a + 1) G)) / 2^53."""
    part = np.zeros((npart, 12), dtype=np.float64, order="F")
    part[:, 0] = np.arange(1, npart + 1)
    i = np.arange(npart, dtype=np.uint64)
    with np.errstate(over="ignore"):
        for a in range(3):
            r = _splitmix64(np.uint64(seed) + (np.uint64(3) * i + np.uint64(a + 1)) * _GOLDEN)
            part[:, 1 + a] = (r >> np.uint64(11)).astype(np.float64) * 2.0 ** -53 * lengths[a]
    return part


def sigma_from_weber(rho, u_rms, radius, weber):
    """sigma = rho u_rms^2 (2R) / We (the reference has no Weber number; this is the choice)."""
    return rho * u_rms * u_rms * (2.0 * radius) / weber


def abc_velocity(nx, modes=((1, 1.0), (3, 0.3)), ny=None, nz=None):
    """Arnold-Beltrami-Childress flow summed over wavenumbers k with amplitude a:
    u = a (sin kz + cos ky), v = a (sin kx + cos kz), w = a (sin ky + cos kx) at the staggered face
    positions.  Each component is independent of its own coordinate, so the discrete divergence is
    exactly zero; cheap to build at any size (outer sums of 1-D tables), used for large grids
    where the Fourier-mode generator above would need tens of GB of host memory."""
    ny = ny or nx
    nz = nz or nx
    dx = LX / nx
    x = (np.arange(nx) + 0.5) * dx
    y = (np.arange(ny) + 0.5) * dx
    z = (np.arange(nz) + 0.5) * dx
    u = np.zeros((nz, ny, nx))
    v = np.zeros((nz, ny, nx))
    w = np.zeros((nz, ny, nx))
    for k, a in modes:
        u += (a * np.sin(k * z))[:, None, None] + (a * np.cos(k * y))[None, :, None]
        v += (a * np.sin(k * x))[None, None, :] + (a * np.cos(k * z))[:, None, None]
        w += (a * np.sin(k * y))[None, :, None] + (a * np.cos(k * x))[None, None, :]
    return u, v, w
