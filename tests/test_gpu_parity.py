"""GPU parity of libmhit_b200.so against the CPU oracle (oracle/mhit_oracle.py).

Each case builds the same seeded state for the oracle and for the library (through the C ABI
via mhit36_mixedp_b200.api), advances both, and compares fields in the max norm relative to
the field's max.  Tolerances: FP64 Poisson <= 1e-12 (the target of the FP64 step); FP32
Poisson compares against the oracle's FP32-storage solve, so its bound is FP32 round-off.
"""
import numpy as np
import pytest

from mhit36_mixedp_b200 import Params, Solver, synth
from oracle import mhit_oracle as orc

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


def relerr(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def make_case(n, phiflag=0, partflag=0, seed=0, npart=0, **kw):
    prm = dict(nx=n, dt=5e-4, mu=0.006, rho=1.0, f1=1.0, f2=1.0, f3=1.0, k0=2.0, radius=0.3, sigma=0.5,
               epsr=1.0, phiflag=phiflag, partflag=partflag)
    prm.update(kw)
    u, v, w = synth.solenoidal_velocity(n, seed)
    phi = part = None
    if phiflag:
        cen = synth.drop_centres(8, seed + 1)
        phi = synth.drops_phi(n, cen, prm["radius"], prm["epsr"] * (2 * np.pi / n))
    if partflag:
        part = synth.uniform_particles(npart, seed + 3)
    return prm, u, v, w, phi, part


def run_both(prm, u, v, w, phi, part, nsteps, oracle_kw=None):
    okw = dict(prm)
    okw.update(oracle_kw or {})
    op = orc.Params(**{k: okw[k] for k in okw if k in orc.Params.__dataclass_fields__})
    st = orc.new_state(op, u, v, w, phi=phi, part=part)
    orc.run(op, st, nsteps)
    gp = Params(**{k: prm[k] for k in prm if k in Params.__dataclass_fields__})
    with Solver(gp) as s:
        s.upload(u, v, w, phi)
        if part is not None:
            s.upload_particles(part)
        s.step(nsteps)
        out = s.download()
        dg = s.diagnostics()
        gpart = s.download_particles() if part is not None else None
    return st, out, dg, gpart


@pytest.mark.parametrize("n", [16, 32])
def test_ns_fp64_one_step(gpu, n):
    prm, u, v, w, phi, part = make_case(n)
    st, out, dg, _ = run_both(prm, u, v, w, phi, part, 1)
    for f in ("u", "v", "w"):
        assert relerr(out[f], getattr(st, f)) < TOL64, f
    assert relerr(out["p"], st.p) < TOL64
    assert abs(dg["gumax"] - st.gumax) <= TOL64 * abs(st.gumax)


def test_ns_fp64_100_steps_64(gpu):
    """The 64^3 NS case (FP64 Poisson, seeded solenoidal start, 100 steps): <= 1e-12 relative."""
    prm, u, v, w, phi, part = make_case(64)
    st, out, dg, _ = run_both(prm, u, v, w, phi, part, 100)
    errs = {f: relerr(out[f], getattr(st, f)) for f in ("u", "v", "w")}
    print("64^3 NS FP64 100 steps rel err", errs)
    for f, e in errs.items():
        assert e < TOL64, (f, e)


@pytest.mark.parametrize("n", [16, 32])
def test_acdi_fp64(gpu, n):
    prm, u, v, w, phi, part = make_case(n, phiflag=1)
    st, out, dg, _ = run_both(prm, u, v, w, phi, part, 5)
    for f in ("u", "v", "w", "phi"):
        e = relerr(out[f], getattr(st, f))
        assert e < TOL64, (f, e)


def test_acdi_fp64_64_multichunk(gpu):
    """64^3: several x tiles and z chunks of the marching phase/momentum kernels."""
    prm, u, v, w, phi, part = make_case(64, phiflag=1)
    st, out, dg, _ = run_both(prm, u, v, w, phi, part, 4)
    for f in ("u", "v", "w", "phi"):
        e = relerr(out[f], getattr(st, f))
        assert e < TOL64, (f, e)


def planted_undershoot(n):
    prm, u, v, w, phi, part = make_case(n, phiflag=1)
    phi = phi.copy()
    phi[n // 2, n // 3, n // 4] = -1e-15  # below -1e-16: the reference's psi is log(<0) = NaN
    return prm, u, v, w, phi


def test_acdi_negative_phi_reference_semantics(gpu):
    """Default: psi = eps log((min(phi,1)+1e-16)/(...)) as multi/main.f90:527-528, so phi < -1e-16
    gives NaN like the reference; the library reports it as MhitNaNError."""
    from mhit36_mixedp_b200 import MhitNaNError
    prm, u, v, w, phi = planted_undershoot(16)
    op = orc.Params(**{k: prm[k] for k in prm if k in orc.Params.__dataclass_fields__})
    st = orc.new_state(op, u, v, w, phi=phi)
    with np.errstate(invalid="ignore"):
        orc.step(op, st)
    assert np.isnan(st.phi).any()
    with Solver(Params(**prm)) as s:
        s.upload(u, v, w, phi)
        with pytest.raises(MhitNaNError):
            s.step(1)


def test_acdi_clamp_matches_oracle(gpu):
    prm, u, v, w, phi = planted_undershoot(32)
    prm["acdi_clamp"] = 1
    st, out, dg, _ = run_both(prm, u, v, w, phi, None, 3)
    for f in ("u", "v", "w", "phi"):
        assert np.isfinite(out[f]).all()
        e = relerr(out[f], getattr(st, f))
        assert e < TOL64, (f, e)


@pytest.mark.parametrize("interp", ["linear1d", "trilinear"])
def test_tracers_fp64(gpu, interp):
    prm, u, v, w, phi, part = make_case(32, partflag=1, npart=500, interp=interp)
    st, out, dg, gpart = run_both(prm, u, v, w, phi, part, 5)
    assert np.max(np.abs(gpart[:, 1:4] - st.part[:, 1:4])) < 1e-12
    assert relerr(gpart[:, 4:7], st.part[:, 4:7]) < TOL64
    assert relerr(gpart[:, 8:11], st.part[:, 8:11]) < TOL64


def test_ns_fp32_poisson(gpu):
    prm, u, v, w, phi, part = make_case(32, poisson="fp32")
    st, out, dg, _ = run_both(prm, u, v, w, phi, part, 5)
    errs = {f: relerr(out[f], getattr(st, f)) for f in ("u", "v", "w", "p")}
    print("32^3 FP32 Poisson 5 steps rel err", errs)
    for f in ("u", "v", "w"):
        assert errs[f] < 1e-5, (f, errs[f])
    assert errs["p"] < 1e-4


def test_modified_laplacian_divergence(gpu):
    prm, u, v, w, phi, part = make_case(32, laplacian="modified")
    st, out, dg, _ = run_both(prm, u, v, w, phi, part, 3)
    for f in ("u", "v", "w"):
        assert relerr(out[f], getattr(st, f)) < TOL64
    umax = max(np.abs(out[f]).max() for f in ("u", "v", "w"))
    assert dg["maxdiv"] < 1e-11 * umax * (32 / (2 * np.pi))


def test_fp32_refined_recovers_fp64(gpu):
    """FP32 Poisson + one FP64 residual sweep (modified Laplacian): u matches the FP64 solve and
    the refined oracle to 1e-12 and the projected divergence is round-off, while the plain FP32
    solve is off by ~1e-10."""
    prm, u, v, w, phi, part = make_case(32, laplacian="modified", poisson="fp32_refined")
    st, out, dg, _ = run_both(prm, u, v, w, phi, part, 5)
    for f in ("u", "v", "w"):
        assert relerr(out[f], getattr(st, f)) < TOL64, f
    prm64 = dict(prm, poisson="fp64")
    st64, out64, dg64, _ = run_both(prm64, u, v, w, phi, part, 5)
    for f in ("u", "v", "w"):
        assert relerr(out[f], out64[f]) < TOL64, f
    umax = max(np.abs(out[f]).max() for f in ("u", "v", "w"))
    assert dg["maxdiv"] < 1e-11 * umax * (32 / (2 * np.pi))


def test_fp32_refined_needs_modified_laplacian(gpu):
    from mhit36_mixedp_b200 import MhitArgError
    with pytest.raises(MhitArgError, match="MODIFIED"):
        Solver(Params(nx=32, poisson="fp32_refined"))


@pytest.mark.parametrize("poisson,tol", [("fp64", TOL64), ("fp32", 1e-5)])
def test_noncubic_box(gpu, poisson, tol):
    """nx != ny != nz (32 x 16 x 64, spacing 2 pi/nx in every direction): every kernel's y and
    z wraps, the 16- and 64-point column transforms and the tracers on a non-cubic box."""
    nx, ny, nz = 32, 16, 64
    dx = 2 * np.pi / nx
    u, v, w = synth.solenoidal_velocity(nx, 4, ny=ny, nz=nz)
    x = (np.arange(nx) + 0.5) * dx
    y = (np.arange(ny) + 0.5) * dx
    z = (np.arange(nz) + 0.5) * dx
    r = np.sqrt((x[None, None, :] - np.pi) ** 2 + (y[None, :, None] - ny * dx / 2) ** 2
                + (z[:, None, None] - nz * dx / 2) ** 2)
    phi = 0.5 * (1.0 - np.tanh((r - 0.8) / (2 * dx)))
    part = synth.uniform_particles(300, 9)
    part[:, 2] *= ny / nx  # positions inside the y and z extents
    part[:, 3] *= nz / nx
    prm = dict(nx=nx, ny=ny, nz=nz, dt=5e-4, mu=0.006, rho=1.0, f1=1.0, f2=1.0, f3=1.0, k0=2.0, radius=0.8,
               sigma=0.5, epsr=1.0, phiflag=1, partflag=1, poisson=poisson)
    st, out, dg, gpart = run_both(prm, u, v, w, phi, part, 4)
    for f in ("u", "v", "w", "phi"):
        e = relerr(out[f], getattr(st, f))
        assert e < tol, (f, e)
    # positions integrate the velocity: dt * steps * (velocity difference) bounds them
    assert np.max(np.abs(gpart[:, 1:4] - st.part[:, 1:4])) < (1e-10 if poisson == "fp64" else 1e-7)
