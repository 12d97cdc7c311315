"""CPU tests of the oracle: pinned against the reference's own published Taylor-Green curve,
checked against the committed 16^3 fixtures, and cross-checked between the NumPy and the
C/OpenMP restatements."""
import json
import math
import os

import numpy as np
import pytest

from mhit36_mixedp_b200 import synth
from oracle import mhit_oracle as orc
from tests.golden.make_golden import CASES, NSTEPS, case_inputs

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def tg_curve(n=128):
    with open(os.path.join(GOLD, f"tg{n}_d2z.json")) as f:
        return json.load(f)


def postproc_dx(n):
    # post/compute_diss: dx = lx/(nx-1), lx = 2*pi with pi a default-REAL literal
    return 2.0 * float(np.float32(math.pi)) / (n - 1)


@pytest.mark.parametrize("n", [128, 512])
def test_tg_initial_dissipation_matches_reference(n):
    g = tg_curve(n)
    p = orc.Params(nx=n, mu=g["nu"], f1=0.0, f2=0.0, f3=0.0, dt=g["dt"])
    u, v, w = orc.taylor_green(p)
    eps0 = orc.dissipation(u, v, w, g["nu"], postproc_dx(n))
    t0, ref0 = g["t_eps"][0]
    assert t0 == 0.0
    # the n^3-term sum is accumulated in another order than the post-processor's: its rounding
    # grows with the number of terms (7e-12 at 512^3)
    assert abs(eps0 / ref0 - 1) < 1e-12 * (n / 128) ** 3


def test_tg_1000_steps_matches_reference_curve():
    """C/OpenMP oracle, 128^3 Taylor-Green, 1000 AB2 steps (t = 0.2) vs val/cudec_128_d2z.txt."""
    from oracle.coracle import COracle
    g = tg_curve()
    p = orc.Params(nx=128, mu=g["nu"], f1=0.0, f2=0.0, f3=0.0, dt=g["dt"])
    u, v, w = orc.taylor_green(p)
    c = COracle(nx=128, dt=g["dt"], mu=g["nu"], rho=1.0, f1=0.0, f2=0.0, f3=0.0, k0=2.0)
    c.set_fields(u, v, w)
    c.step(1000)
    f = c.fields()
    eps = orc.dissipation(f["u"], f["v"], f["w"], g["nu"], postproc_dx(128))
    t, ref = g["t_eps"][1]
    assert abs(t - 0.2) < 1e-12
    assert abs(eps / ref - 1) < 1e-11, eps / ref - 1


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_fixtures(name):
    prm, u, v, w, phi, part = case_inputs(name)
    op = orc.Params(**prm)
    st = orc.new_state(op, u, v, w, phi=phi, part=part)
    orc.run(op, st, NSTEPS)
    gold = np.load(os.path.join(GOLD, "oracle_16.npz"))
    for f in ("u", "v", "w", "p"):
        np.testing.assert_allclose(getattr(st, f), gold[f"{name}/{f}"], rtol=0, atol=1e-14)
    if phi is not None:
        np.testing.assert_allclose(st.phi, gold[f"{name}/phi"], rtol=0, atol=1e-14)
    if part is not None:
        np.testing.assert_allclose(st.part, gold[f"{name}/part"], rtol=0, atol=1e-13)


@pytest.mark.parametrize("name", CASES)
def test_c_oracle_matches_numpy_oracle(name):
    from oracle.coracle import COracle
    prm, u, v, w, phi, part = case_inputs(name)
    c = COracle(**prm)
    c.set_fields(u, v, w, phi)
    if part is not None:
        c.set_particles(part)
    c.step(NSTEPS)
    f = c.fields()
    gold = np.load(os.path.join(GOLD, "oracle_16.npz"))
    for k in ("u", "v", "w"):
        ref = gold[f"{name}/{k}"]
        assert np.max(np.abs(f[k] - ref)) / np.max(np.abs(ref)) < 1e-13
    if part is not None:
        assert np.max(np.abs(c.particles()[:, 1:7] - gold[f"{name}/part"][:, 1:7])) < 1e-13


def test_modified_laplacian_projects_to_zero_divergence():
    prm, u, v, w, _, _ = case_inputs("ns_fp64")
    op = orc.Params(laplacian="modified", **prm)
    st = orc.new_state(op, u, v, w)
    orc.step(op, st)
    div = orc.divergence(op, st.u, st.v, st.w)
    assert np.max(np.abs(div)) < 1e-11
    # the reference's exact-k^2 divide leaves an O(dx^2) divergence
    op2 = orc.Params(**prm)
    st2 = orc.new_state(op2, u, v, w)
    orc.step(op2, st2)
    assert np.max(np.abs(orc.divergence(op2, st2.u, st2.v, st2.w))) > 1e-6


def test_fp32_poisson_close_to_fp64():
    prm, u, v, w, _, _ = case_inputs("ns_fp64")
    a = orc.new_state(orc.Params(**prm), u, v, w)
    b = orc.new_state(orc.Params(poisson="fp32", **prm), u, v, w)
    orc.run(orc.Params(**prm), a, 5)
    orc.run(orc.Params(poisson="fp32", **prm), b, 5)
    assert np.max(np.abs(a.u - b.u)) / np.max(np.abs(a.u)) < 1e-5
    assert np.max(np.abs(a.u - b.u)) > 0


def test_forcing_tables_reference_labelling():
    """y/z tables read mysin(jg) with jg one entry on from x (multi/main.f90:709-714)."""
    p = orc.Params(nx=16, k0=2.0)
    sx, cx, sy, cy, sz, cz = orc.forcing_tables(p)
    np.testing.assert_array_equal(sy[:-1], sx[1:])
    np.testing.assert_array_equal(cz[:-1], cx[1:])
    # the entry one past the table is the periodic continuation for integer k0
    assert abs(sy[-1] - sx[0]) < 1e-14
    p0 = orc.Params(nx=16, k0=2.0, yz_shift=0)
    t0 = orc.forcing_tables(p0)
    np.testing.assert_array_equal(t0[2], t0[0])


def test_negative_phi_nan_and_clamp():
    """phi < -1e-16 makes the reference's psi NaN (multi/main.f90:527-528 clamps only above);
    acdi_clamp=1 clamps below as well and stays finite, equal to the unclamped step elsewhere."""
    prm, u, v, w, phi, _ = case_inputs("acdi_tracers")
    prm = dict(prm, partflag=0)
    phi = phi.copy()
    phi[3, 4, 5] = -1e-15
    a = orc.new_state(orc.Params(**prm), u, v, w, phi=phi)
    with np.errstate(invalid="ignore"):
        orc.step(orc.Params(**prm), a)
    assert np.isnan(a.phi).any()
    b = orc.new_state(orc.Params(acdi_clamp=1, **prm), u, v, w, phi=phi)
    orc.step(orc.Params(acdi_clamp=1, **prm), b)
    assert np.isfinite(b.phi).all() and np.isfinite(b.u).all()
    from oracle.coracle import COracle
    c = COracle(acdi_clamp=1, **prm)
    c.set_fields(u, v, w, phi)
    c.step(1)
    f = c.fields()
    assert np.max(np.abs(f["phi"] - b.phi)) < 1e-14


def test_mean_removed_and_gumax_signed():
    prm, u, v, w, _, _ = case_inputs("ns_fp64")
    op = orc.Params(**prm)
    st = orc.new_state(op, u + 0.3, v, w)
    orc.step(op, st)
    assert abs(st.u.mean()) < 1e-15 and abs(st.v.mean()) < 1e-15
    assert st.gumax == max(st.u.max(), st.v.max(), st.w.max())


def test_oracle_incremental_fp32_solve():
    """The oracle's incremental FP32 solve (one FP32 solve per step for the increment over the
    previous pressure, the residual in FP64) stays within FP32 round-off of its FP64 step and,
    from the third step on, leaves a divergence far below the plain FP32 solve's."""
    n = 32
    u, v, w = synth.solenoidal_velocity(n, 0)
    phi = synth.drops_phi(n, synth.drop_centres(8, 1), 0.3, 2 * np.pi / n)
    runs = {}
    for mode in ("fp64", "fp32", "fp32_incremental"):
        op = orc.Params(nx=n, dt=5e-4, mu=0.006, radius=0.3, sigma=0.5, phiflag=1, poisson=mode,
                        laplacian="modified")
        st = orc.new_state(op, u, v, w, phi=phi)
        divs = []
        for _ in range(6):
            orc.step(op, st)
            divs.append(float(np.abs(orc.divergence(op, st.u, st.v, st.w)).max()))
        runs[mode] = (st, divs)
    ref = runs["fp64"][0]
    st, divs = runs["fp32_incremental"]
    for f in ("u", "v", "w", "phi"):
        a, b = getattr(st, f), getattr(ref, f)
        assert np.abs(a - b).max() / np.abs(b).max() < 1e-8, f
    assert max(divs[3:]) < 1e-2 * min(runs["fp32"][1][3:]), (divs, runs["fp32"][1])
    assert st.p32.dtype == np.float32 and np.abs(st.p32 - st.p).max() <= 1e-6 * np.abs(st.p).max()


@pytest.mark.parametrize("laplacian", ["exact", "modified"])
def test_oracle_k2_table_non_cubic(laplacian):
    """On a box of nx x ny x nz cubic cells the wavenumbers are physical (index x nx/n per axis):
    only the zero mode has k^2 = 0, and with the modified Laplacian one FP64 step leaves the
    discrete divergence at round-off."""
    nx, ny, nz = 32, 16, 64
    op = orc.Params(nx=nx, ny=ny, nz=nz, dt=5e-4, mu=0.006, laplacian=laplacian)
    k2 = orc.k2_table(op)
    assert k2.shape == (nz, ny, nx // 2 + 1)
    assert k2[0, 0, 0] == 0.0 and np.count_nonzero(k2 == 0.0) == 1
    if laplacian == "exact":
        assert k2[0, 1, 0] == (nx / ny) ** 2 and k2[1, 0, 0] == (nx / nz) ** 2
    u, v, w = synth.solenoidal_velocity(nx, 3, ny=ny, nz=nz)
    st = orc.new_state(op, u, v, w)
    orc.step(op, st)
    div = np.abs(orc.divergence(op, st.u, st.v, st.w)).max()
    if laplacian == "modified":
        assert div < 1e-11 * np.abs(st.u).max() * nx / (2 * np.pi), div
