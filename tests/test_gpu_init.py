"""Initial conditions synthesised on the device against their host restatements: the Taylor-Green
start of multi/main.f90:324-337 (oracle), the seeded random solenoidal velocity and the
multi-drop phase field of the benchmark configurations (synth), and the centred drop of
multi/main.f90:370-382 (oracle)."""
import math

import numpy as np
import pytest

from mhit36_mixedp_b200 import Params, Solver, synth
from oracle import mhit_oracle as orc

pytestmark = pytest.mark.gpu

SHAPES = [(32, 32, 32), (32, 16, 64)]


@pytest.mark.parametrize("shape", SHAPES)
def test_taylor_green_matches_oracle(gpu, shape):
    nx, ny, nz = shape
    with Solver(Params(nx=nx, ny=ny, nz=nz)) as s:
        s.init_taylor_green()
        out = s.download(("u", "v", "w"))
    u, v, w = orc.taylor_green(orc.Params(nx=nx, ny=ny, nz=nz))
    # the per-axis sines and cosines come from the host's libm: equal to numpy's within an ulp
    for f, ref in (("u", u), ("v", v)):
        assert np.max(np.abs(out[f] - ref)) <= 4e-16, f
    assert not out["w"].any()


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("yz_shift", [1, 0])
def test_solenoidal_modes_match_host_generator(gpu, shape, yz_shift):
    nx, ny, nz = shape
    with Solver(Params(nx=nx, ny=ny, nz=nz, yz_shift=yz_shift)) as s:
        s.init_solenoidal(seed=7, kmax=4, rms=1.3)
        out = s.download(("u", "v", "w"))
    ref = synth.solenoidal_velocity(nx, 7, kmax=4, rms=1.3, yz_shift=yz_shift, ny=ny, nz=nz)
    for f, r in zip("uvw", ref):
        assert np.max(np.abs(out[f] - r)) <= 1e-13 * np.max(np.abs(r)), f
        assert abs(math.sqrt(float(np.mean(out[f] ** 2))) - 1.3) < 1e-12


def test_solenoidal_modes_small_kmax_and_bad_arguments(gpu):
    n = 16
    with Solver(Params(nx=n)) as s:
        s.init_solenoidal(seed=3, kmax=1)
        out = s.download(("u", "v", "w"))
        ref = synth.solenoidal_velocity(n, 3, kmax=1)
        for f, r in zip("uvw", ref):
            assert np.max(np.abs(out[f] - r)) <= 1e-13 * np.max(np.abs(r))
        with pytest.raises(Exception):
            s.init_velocity_modes(np.zeros((3, 3, 3, 3), complex))  # a zero field has no rms
        with pytest.raises(Exception):
            s.init_velocity_modes(np.ones((3, 4, 4, 4), complex))  # even K


def test_drops_match_host_generator(gpu):
    n = 32
    dx = 2 * math.pi / n
    centres = synth.drop_centres(6, 5)
    with Solver(Params(nx=n, phiflag=1)) as s:
        s.init_drops(centres, 0.5)
        out = s.download(("phi",))
    ref = synth.drops_phi(n, centres, 0.5, dx)
    # CUDA's tanh against numpy's: within a few ulp of phi
    assert np.max(np.abs(out["phi"] - ref)) <= 1e-15


def test_centred_drop_matches_oracle(gpu):
    n = 32
    with Solver(Params(nx=n, phiflag=1, radius=0.7)) as s:
        s.init_drops([[math.pi, math.pi, math.pi]], 0.7)
        out = s.download(("phi",))
    ref = orc.single_drop(orc.Params(nx=n, phiflag=1, radius=0.7))
    # the oracle follows the reference's accumulated coordinates and summation order
    assert np.max(np.abs(out["phi"] - ref)) <= 1e-13


def test_device_start_steps_like_host_start(gpu):
    n = 32
    centres = synth.drop_centres(4, 2)
    prm = Params(nx=n, phiflag=1, radius=0.5, sigma=0.2, mu=0.01, dt=2e-4)
    with Solver(prm) as s:
        s.init_solenoidal(seed=11)
        s.init_drops(centres, 0.5)
        s.step(5)
        dev = s.download()
    u, v, w = synth.solenoidal_velocity(n, 11)
    phi = synth.drops_phi(n, centres, 0.5, 2 * math.pi / n)
    with Solver(prm) as s:
        s.upload(u, v, w, phi)
        s.step(5)
        host = s.download()
    for f in ("u", "v", "w", "phi"):
        assert np.max(np.abs(dev[f] - host[f])) <= 1e-12 * np.max(np.abs(host[f])), f


def test_init_drops_keeps_the_velocity(gpu):
    n = 32
    prm = Params(nx=n, phiflag=1, radius=0.5, sigma=0.2, mu=0.01, dt=2e-4, f1=1.0, f2=1.0, f3=1.0)
    with Solver(prm) as s:
        s.init_solenoidal(seed=1)
        s.init_drops([[1.0, 2.0, 3.0]], 0.5)
        s.step(3)  # forcing: the stored velocity now carries a lazily removed mean
        before = s.download(("u", "v", "w"))
        s.init_drops([[3.0, 2.0, 1.0]], 0.6)
        after = s.download(("u", "v", "w"))
    for f in "uvw":
        assert np.max(np.abs(after[f] - before[f])) <= 1e-15 * np.max(np.abs(before[f])), f


@pytest.mark.parametrize("shape", SHAPES)
def test_particles_match_host_twin(gpu, shape):
    nx, ny, nz = shape
    dx = 2 * math.pi / nx
    lengths = (synth.LX, synth.LX if ny == nx else dx * ny, synth.LX if nz == nx else dx * nz)
    with Solver(Params(nx=nx, ny=ny, nz=nz, partflag=1)) as s:
        s.init_particles(1000, 77)
        got = s.download_particles()
    assert np.array_equal(got, synth.seeded_particles(1000, 77, lengths))


def test_device_tracers_step_like_uploaded_ones(gpu):
    n = 32
    prm = Params(nx=n, partflag=1, mu=0.01, dt=5e-4)
    res = []
    for device_table in (True, False):
        with Solver(prm) as s:
            s.init_solenoidal(seed=2)
            if device_table:
                s.init_particles(500, 9)
            else:
                s.upload_particles(synth.seeded_particles(500, 9))
            s.step(4)
            res.append(s.download_particles())
    assert np.array_equal(res[0], res[1])


def test_velocity_inits_keep_phi_after_odd_steps(gpu):
    """The velocity generators write the current ping-pong slot: phi survives, whatever the
    parity of the step count."""
    n = 32
    prm = Params(nx=n, phiflag=1, radius=0.5, sigma=0.2, mu=0.01, dt=2e-4)
    with Solver(prm) as s:
        s.init_solenoidal(seed=1)
        s.init_drops([[1.0, 2.0, 3.0]], 0.5)
        s.step(3)
        before = s.download(("phi",))["phi"]
        s.init_solenoidal(seed=2)
        assert np.array_equal(s.download(("phi",))["phi"], before)
        s.step(1)
        before = s.download(("phi",))["phi"]
        s.init_taylor_green()
        assert np.array_equal(s.download(("phi",))["phi"], before)
        tg = s.download(("u",))["u"]
    u, _, _ = orc.taylor_green(orc.Params(nx=n))
    assert np.max(np.abs(tg - u)) <= 4e-16
