"""Ensemble of boxes of uneven sizes: one graph launch per step must give exactly the fields of
stepping every box on its own (the same kernels; z-chunk and stream choices of the autotuner do
not change any cell's arithmetic), and the boxes must match the oracle."""
import numpy as np
import pytest

from mhit36_mixedp_b200 import Ensemble, MhitStateError, Params, Solver, synth
from oracle import mhit_oracle as orc

pytestmark = pytest.mark.gpu


def box_cases():
    specs = [(16, 0, "fp64"), (32, 1, "fp32"), (64, 1, "fp64"), (32, 0, "fp64")]
    out = []
    for b, (n, phiflag, poisson) in enumerate(specs):
        prm = Params(nx=n, dt=5e-4, mu=0.004 + 0.001 * b, radius=0.3, sigma=0.5, phiflag=phiflag, poisson=poisson)
        u, v, w = synth.solenoidal_velocity(n, 100 + b)
        phi = synth.drops_phi(n, synth.drop_centres(4 + b, 200 + b), 0.3, 2 * np.pi / n) if phiflag else None
        out.append((prm, u, v, w, phi))
    return out


def standalone(prm, u, v, w, phi, nsteps):
    with Solver(prm) as s:
        s.upload(u, v, w, phi)
        s.step(nsteps)
        return s.download()


@pytest.mark.parametrize("tune", [False, True])
def test_ensemble_matches_standalone(gpu, tune):
    cases = box_cases()
    with Ensemble([c[0] for c in cases]) as ens:
        if tune:
            t = ens.autotune(trials=1)
            assert 1 <= t["lanes"] <= len(cases)
            assert all(z in (8, 16, 32, 64, 128) for z in t["zchunk_mom"])
        for box, (prm, u, v, w, phi) in zip(ens.boxes, cases):
            box.upload(u, v, w, phi)
        ens.step(6)
        got = [box.download() for box in ens.boxes]
    for (prm, u, v, w, phi), g in zip(cases, got):
        ref = standalone(prm, u, v, w, phi, 6)
        for k in ref:
            np.testing.assert_array_equal(g[k], ref[k])


def test_ensemble_box_matches_oracle(gpu):
    prm, u, v, w, phi = box_cases()[2]
    with Ensemble([c[0] for c in box_cases()]) as ens:
        for box, (p_, u_, v_, w_, phi_) in zip(ens.boxes, box_cases()):
            box.upload(u_, v_, w_, phi_)
        ens.step(4)
        g = ens.boxes[2].download()
    op = orc.Params(nx=64, dt=5e-4, mu=prm.mu, radius=0.3, sigma=0.5, phiflag=1)
    st = orc.new_state(op, u, v, w, phi=phi)
    orc.run(op, st, 4)
    for k in ("u", "v", "w", "phi"):
        ref = getattr(st, k)
        assert np.max(np.abs(g[k] - ref)) / np.max(np.abs(ref)) < 1e-12


def test_ensemble_requires_boxes_in_step(gpu):
    cases = box_cases()[:2]
    with Ensemble([c[0] for c in cases]) as ens:
        for box, (prm, u, v, w, phi) in zip(ens.boxes, cases):
            box.upload(u, v, w, phi)
        ens.boxes[0].step(1)
        with pytest.raises(MhitStateError):
            ens.step(1)


def test_ensemble_follows_a_tracer_reupload(gpu):
    """Uploading a new tracer table to a box after the ensemble graphs were captured (they bake in
    the tracer kernel and its table) must rebuild them: the box then matches a standalone box that
    did the same."""
    specs = [(16, 200), (32, 300)]
    prms = [Params(nx=n, dt=5e-4, mu=0.005, partflag=1) for n, _ in specs]
    fields = [synth.solenoidal_velocity(n, 10 + b) for b, (n, _) in enumerate(specs)]
    first = [synth.uniform_particles(npart, 20 + b) for b, (_, npart) in enumerate(specs)]
    second = synth.uniform_particles(150, 30)
    with Ensemble(prms) as ens:
        for box, (u, v, w), part in zip(ens.boxes, fields, first):
            box.upload(u, v, w)
            box.upload_particles(part)
        ens.step(4)                       # Euler + graph-replayed steps
        ens.boxes[0].upload_particles(second)
        ens.step(3)
        got = ens.boxes[0].download()
        got_part = ens.boxes[0].download_particles()
    with Solver(prms[0]) as s:
        s.upload(*fields[0])
        s.upload_particles(first[0])
        s.step(4)
        s.upload_particles(second)
        s.step(3)
        ref = s.download()
        ref_part = s.download_particles()
    for k in ref:
        np.testing.assert_array_equal(got[k], ref[k])
    np.testing.assert_array_equal(got_part, ref_part)


def batchable_cases(phiflag):
    out = []
    for b, n in enumerate((32, 64, 128, 64)):
        prm = Params(nx=n, dt=2e-4, mu=0.003 + 0.001 * b, radius=0.3, sigma=0.4, phiflag=phiflag, acdi_clamp=1,
                     poisson="fp32" if b % 2 else "fp64")
        u, v, w = synth.solenoidal_velocity(n, 300 + b)
        phi = synth.drops_phi(n, synth.drop_centres(5 + b, 400 + b), 0.3, 2 * np.pi / n) if phiflag else None
        out.append((prm, u, v, w, phi))
    return out


@pytest.mark.parametrize("phiflag", [1, 0])
def test_batched_schedule_matches_lanes_and_standalone(gpu, phiflag):
    """The batched schedule (phase and momentum of all boxes as one persistent launch each, work
    items from a device queue, largest boxes first) gives every box the bits of the per-box
    lanes and of a standalone box, with the default and with autotuned z chunks."""
    cases = batchable_cases(phiflag)
    got = {}
    for mode in ("batched", "lanes", "tuned"):
        with Ensemble([c[0] for c in cases]) as ens:
            if mode == "tuned":
                ens.autotune(trials=1)
            else:
                ens.set_batched(mode == "batched")
            assert mode == "tuned" or ens.tuning()["batched"] == (mode == "batched")
            for box, (prm, u, v, w, phi) in zip(ens.boxes, cases):
                box.upload(u, v, w, phi)
            ens.step(6)
            got[mode] = [box.download() for box in ens.boxes]
    for b, (prm, u, v, w, phi) in enumerate(cases):
        ref = standalone(prm, u, v, w, phi, 6)
        for mode in got:
            for k in ref:
                np.testing.assert_array_equal(got[mode][b][k], ref[k], err_msg=f"{mode} box {b} {k}")

