"""Full-step parity at the scope-table configurations' sizes against the C oracle.

The NumPy oracle steps 64^3 in a second but not 256^3 or 512^3; the C/OpenMP restatement of the
same loop (oracle/mhit_oracle.c, ``multi/main.f90:456-1007`` pass by pass, its own Stockham FFT)
does a 512^3 NS+ACDI step in about 2 s on 16 host cores and holds about 21 GB of host memory.
These tests run the configurations the benchmark and the configuration list name, on their own
inputs:

* the 256^3 NS+ACDI case (64 drops of radius 0.3 at seeded centres, eps = dx, We = 1,
  nu = 0.003, seeded solenoidal velocity), 20 steps;
* the 512^3 benchmark workload itself (the same recipe at 512^3, ``acdi_clamp=1``), 3 steps,
  which exercises the 256-plane ``k_phase`` chunk and the 64-plane ``k_mom`` / ``k_correct``
  chunks that only grids of 512^3 and up select;
* a 192^3 NS+ACDI box advanced inside an ensemble next to a 64^3 box (the radix-3 schedules of
  the ensemble configuration), 10 steps.

Tolerances (max norm relative to the field's max): FP64 Poisson 1e-12, the target of the FP64
step; FP32 Poisson against the oracle's FP32-storage solve (rounded to FP32 after each axis
like the library) 1e-5, FP32 round-off of the pressure carried through the projection.
"""
import math

import numpy as np
import pytest

from mhit36_mixedp_b200 import Ensemble, Params, Solver, synth
from oracle.coracle import COracle

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "fp32": 1e-5}


def relerr(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def drops_workload(n, ndrops=64, seed_drops=1, seed_vel=2, nu=0.003, we=1.0, dt=2e-4):
    """NS+ACDI at n^3: ndrops drops of radius 0.3 (eps = dx) at seeded uniform centres, seeded
    solenoidal velocity (unit rms), sigma from the Weber number, acdi_clamp on."""
    radius, rho = 0.3, 1.0
    u, v, w = synth.solenoidal_velocity(n, seed_vel)
    phi = synth.drops_phi(n, synth.drop_centres(ndrops, seed_drops), radius, 2 * math.pi / n)
    sigma = synth.sigma_from_weber(rho, 1.0, radius, we)
    prm = dict(nx=n, dt=dt, mu=nu, rho=rho, f1=1.0, f2=1.0, f3=1.0, k0=2.0, radius=radius, sigma=sigma,
               epsr=1.0, phiflag=1, partflag=0, acdi_clamp=1)
    return prm, u, v, w, phi


def oracle_fields(prm, u, v, w, phi, poisson, nsteps):
    c = COracle(poisson=poisson, **prm)
    try:
        c.set_fields(u, v, w, phi)
        c.step(nsteps)
        return c.fields()
    finally:
        c.close()


def compare(got, ref, poisson, label):
    errs = {f: relerr(got[f], ref[f]) for f in ("u", "v", "w", "phi")}
    print(label, poisson, errs)
    for f, e in errs.items():
        assert e < TOL[poisson], (label, poisson, f, e)


@pytest.mark.parametrize("poisson", ["fp64", "fp32"])
def test_ns_acdi_256_20_steps(gpu, poisson):
    prm, u, v, w, phi = drops_workload(256)
    with Solver(Params(poisson=poisson, **prm)) as s:
        s.upload(u, v, w, phi)
        s.step(20)
        got = s.download(fields=("u", "v", "w", "phi"))
    compare(got, oracle_fields(prm, u, v, w, phi, poisson, 20), poisson, "256^3 x 20")


@pytest.mark.parametrize("poisson", ["fp64", "fp32"])
def test_bench_workload_512_3_steps(gpu, poisson):
    prm, u, v, w, phi = drops_workload(512)
    with Solver(Params(poisson=poisson, **prm)) as s:
        s.upload(u, v, w, phi)
        s.step(3)
        got = s.download(fields=("u", "v", "w", "phi"))
    compare(got, oracle_fields(prm, u, v, w, phi, poisson, 3), poisson, "512^3 x 3")


@pytest.mark.parametrize("poisson", ["fp64", "fp32"])
def test_ensemble_192_box(gpu, poisson):
    small = drops_workload(64, ndrops=8, seed_drops=11, seed_vel=12, nu=0.005, we=2.0)
    big = drops_workload(192, ndrops=32, seed_drops=21, seed_vel=22, nu=0.004, we=1.5)
    with Ensemble([Params(poisson=poisson, **small[0]), Params(poisson=poisson, **big[0])]) as ens:
        for box, (prm, u, v, w, phi) in zip(ens.boxes, (small, big)):
            box.upload(u, v, w, phi)
        ens.step(10)
        got = ens.boxes[1].download(fields=("u", "v", "w", "phi"))
    prm, u, v, w, phi = big
    compare(got, oracle_fields(prm, u, v, w, phi, poisson, 10), poisson, "ensemble 192^3 x 10")
