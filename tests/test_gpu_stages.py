"""Stage-by-stage GPU parity: each kernel of the step against the matching oracle block.

Runs the pipeline one stage at a time through the C-ABI test hooks (mhit_debug_run_stage /
mhit_debug_get_buffer) and compares the stage's output buffer with the oracle function that
restates the same lines of multi/main.f90.  FP64 everywhere, tolerance 1e-12 relative to the
buffer's max.
"""
import numpy as np
import pytest

from mhit36_mixedp_b200 import Params, Solver, synth
from oracle import mhit_oracle as orc

pytestmark = pytest.mark.gpu
TOL = 1e-12


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def setup(n, phiflag=0, partflag=0, **kw):
    prm = dict(nx=n, dt=5e-4, mu=0.006, rho=1.0, f1=1.0, f2=1.0, f3=1.0, k0=2.0, radius=0.3, sigma=0.5,
               epsr=1.0, phiflag=phiflag, partflag=partflag)
    prm.update(kw)
    u, v, w = synth.solenoidal_velocity(n, 0)
    phi = synth.drops_phi(n, synth.drop_centres(8, 1), 0.3, 2 * np.pi / n) if phiflag else None
    part = synth.uniform_particles(300, 3) if partflag else None
    op = orc.Params(**{k: prm[k] for k in prm if k in orc.Params.__dataclass_fields__})
    st = orc.new_state(op, u, v, w, phi=phi, part=part)
    s = Solver(Params(**prm))
    s.upload(u, v, w, phi)
    if part is not None:
        s.upload_particles(part)
    return op, st, s


@pytest.mark.parametrize("n", [16, 32, 64])
def test_stages_ns(gpu, n):
    op, st, s = setup(n)
    with s:
        tab = orc.forcing_tables(op)
        orc.momentum_step(op, st, tab)
        s.run_stage("momentum")
        assert rel(s.buffer("un"), st.u) < TOL
        assert rel(s.buffer("vn"), st.v) < TOL
        assert rel(s.buffer("wn"), st.w) < TOL
        assert rel(s.buffer("ru"), st.rhsu_o) < TOL
        rhsp = orc.poisson_rhs(op, st.u, st.v, st.w)
        hx = np.fft.rfft(rhsp, axis=2)
        s.run_stage("xfwd")
        e = rel(s.buffer("spec"), hx)
        assert e < TOL, ("xfwd", e)
        hy = np.fft.fft(hx, axis=1)
        s.run_stage("yfwd")
        e = rel(s.buffer("spec"), hy)
        assert e < TOL, ("yfwd", e)
        hz = np.fft.fft(hy, axis=0)
        with np.errstate(divide="ignore", invalid="ignore"):
            hz = -hz / orc.k2_table(op) / float(n ** 3)
        hz[0, 0, 0] = 0.0
        hz = np.fft.ifft(hz, axis=0, norm="forward")
        s.run_stage("zsolve")
        e = rel(s.buffer("spec"), hz)
        assert e < TOL, ("zsolve", e)
        hy = np.fft.ifft(hz, axis=1, norm="forward")
        s.run_stage("yinv")
        e = rel(s.buffer("spec"), hy)
        assert e < TOL, ("yinv", e)
        pr = orc.poisson_solve(op, rhsp)
        s.run_stage("xinv")
        e = rel(s.buffer("p"), pr)
        assert e < TOL, ("xinv", e)
        means = orc.correct(op, st, pr)
        s.run_stage("correct")
        for f, m, name in (("un", means[0], "u"), ("vn", means[1], "v"), ("wn", means[2], "w")):
            e = rel(s.buffer(f) - m, getattr(st, name))
            assert e < TOL, (f, e)
        s.commit_step()
        d = s.diagnostics()
        assert abs(d["gumax"] - st.gumax) <= TOL * abs(st.gumax)
        for q in range(3):
            assert abs(d["mean"][q] - means[q]) < 1e-14


@pytest.mark.parametrize("n", [16, 32, 64])
def test_stage_phase(gpu, n):
    op, st, s = setup(n, phiflag=1)
    with s:
        orc.phase_step(op, st)
        s.run_stage("phase")
        e = rel(s.buffer("phin"), st.phi)
        assert e < TOL, e
        e = rel(s.buffer("rphi"), st.rhsphi_o)
        assert e < TOL, e
        tab = orc.forcing_tables(op)
        orc.momentum_step(op, st, tab)
        s.run_stage("momentum")
        for f, name in (("un", "u"), ("vn", "v"), ("wn", "w")):
            e = rel(s.buffer(f), getattr(st, name))
            assert e < TOL, (f, e)


@pytest.mark.parametrize("interp", ["linear1d", "trilinear"])
def test_stage_tracer(gpu, interp):
    op, st, s = setup(32, partflag=1, interp=interp)
    with s:
        orc.tracer_step(op, st)
        s.run_stage("tracer")
        s.commit_step()
        gp = s.download_particles()
        assert np.max(np.abs(gp[:, 1:4] - st.part[:, 1:4])) < 1e-13
        assert rel(gp[:, 4:7], st.part[:, 4:7]) < TOL
