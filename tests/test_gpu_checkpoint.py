"""Exact-resume checkpoints and state-preserving downloads.

The reference restarts from its field files with an Euler step (rhs_o is not in them,
multi/main.f90:440-441).  ``write_checkpoint`` / ``read_checkpoint`` also keep the AB2 history,
the device scalars (lazily removed mean, gumax of the last projection) and the tracer table, so a
run stopped and resumed in a new context must give the same bits as one that never stopped.
``download`` materialises the lazily removed mean on the device; that must not change a bit of
what later steps compute either.
"""
import numpy as np
import pytest

from mhit36_mixedp_b200 import MhitArgError, MhitIOError, Params, Solver, synth

pytestmark = pytest.mark.gpu


def case(n=32, poisson="fp64", **kw):
    lap = "modified" if poisson in ("fp32_refined", "fp32_incremental") else "exact"
    prm = Params(nx=n, dt=5e-4, mu=0.006, phiflag=1, partflag=1, radius=0.3, sigma=0.5, poisson=poisson,
                 laplacian=lap, **kw)
    u, v, w = synth.solenoidal_velocity(n, 0)
    phi = synth.drops_phi(n, synth.drop_centres(8, 1), 0.3, 2 * np.pi / n)
    part = synth.uniform_particles(300, 3)
    return prm, u, v, w, phi, part


def run_straight(prm, u, v, w, phi, part, nsteps):
    with Solver(prm) as s:
        s.upload(u, v, w, phi)
        s.upload_particles(part)
        s.step(nsteps)
        return s.download(), s.download_particles(), s.diagnostics()


@pytest.mark.parametrize("poisson", ["fp64", "fp32", "fp32_refined", "fp32_incremental"])
def test_checkpoint_resume_is_bit_exact(gpu, tmp_path, poisson):
    prm, u, v, w, phi, part = case(poisson=poisson)
    ref, ref_part, ref_dg = run_straight(prm, u, v, w, phi, part, 7)
    ck = str(tmp_path / "state.ckp")
    with Solver(prm) as s:
        s.upload(u, v, w, phi)
        s.upload_particles(part)
        s.step(3)
        s.write_checkpoint(ck)
    with Solver(prm) as s:
        s.read_checkpoint(ck)
        s.step(4)
        got, got_part, dg = s.download(), s.download_particles(), s.diagnostics()
    for f in ref:
        np.testing.assert_array_equal(got[f], ref[f], err_msg=f)
    np.testing.assert_array_equal(got_part, ref_part)
    assert dg["nstep"] == ref_dg["nstep"] == 7
    assert dg["gumax"] == ref_dg["gumax"]


def test_download_mid_run_changes_nothing(gpu):
    prm, u, v, w, phi, part = case()
    ref, ref_part, _ = run_straight(prm, u, v, w, phi, part, 6)
    with Solver(prm) as s:
        s.upload(u, v, w, phi)
        s.upload_particles(part)
        s.step(2)
        s.download()
        s.step(2)
        s.download(fields=("u", "p"))
        s.step(2)
        got = s.download()
    for f in ref:
        np.testing.assert_array_equal(got[f], ref[f], err_msg=f)


def test_checkpoint_rejects_other_sizes_and_files(gpu, tmp_path):
    prm, u, v, w, phi, part = case()
    ck = str(tmp_path / "state.ckp")
    with Solver(prm) as s:
        s.upload(u, v, w, phi)
        s.upload_particles(part)
        s.step(1)
        s.write_checkpoint(ck)
    prm16 = case(n=16)[0]
    with Solver(prm16) as s:
        with pytest.raises(MhitArgError):
            s.read_checkpoint(ck)
    prm32 = case(poisson="fp32")[0]
    with Solver(prm32) as s:
        with pytest.raises(MhitArgError):
            s.read_checkpoint(ck)
    junk = tmp_path / "junk.ckp"
    junk.write_bytes(b"not a checkpoint" * 8)
    with Solver(prm) as s:
        with pytest.raises(MhitIOError):
            s.read_checkpoint(str(junk))
        with pytest.raises(MhitIOError):
            s.read_checkpoint(str(tmp_path / "missing.ckp"))
    short = tmp_path / "short.ckp"
    short.write_bytes(open(ck, "rb").read()[:5000])
    with Solver(prm) as s:
        with pytest.raises(MhitIOError):
            s.read_checkpoint(str(short))
    # a checkpoint cut off in its last array is rejected before any device state changes
    cut = tmp_path / "cut.ckp"
    cut.write_bytes(open(ck, "rb").read()[:-8])
    prm_, u_, v_, w_, phi_ = case()[:5]
    with Solver(prm) as s:
        s.upload(u_, v_, w_, phi_)
        s.step(2)
        before = s.download()
        nstep = s.diagnostics()["nstep"]
        with pytest.raises(MhitIOError, match="needs"):
            s.read_checkpoint(str(cut))
        after = s.download()
        assert s.diagnostics()["nstep"] == nstep
        for k in before:
            np.testing.assert_array_equal(after[k], before[k])
