"""Field files and run control on the GPU path.

writefield (multi/readwrite.f90:1-96) writes raw float64, x fastest, no header, interior only,
named <dir>/{u,v,w,p,phi}_%08d.dat; readfield / readfield_restart (:107-318) read the same
layout.  A restart from files starts with an Euler step (rhs_o is not in the files,
multi/main.f90:440-441), so it reproduces a fresh run started from the same fields.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from mhit36_mixedp_b200 import FIELD_P, FIELD_PHI, FIELD_U, FIELD_V, FIELD_W, MhitIOError, Params, Solver, synth

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def make(n=32):
    prm = Params(nx=n, dt=5e-4, mu=0.006, phiflag=1, radius=0.3, sigma=0.5)
    u, v, w = synth.solenoidal_velocity(n, 0)
    phi = synth.drops_phi(n, synth.drop_centres(8, 1), 0.3, 2 * np.pi / n)
    return prm, u, v, w, phi


def test_writefield_layout_and_names(gpu, tmp_path):
    prm, u, v, w, phi = make()
    with Solver(prm) as s:
        s.upload(u, v, w, phi)
        s.step(3)
        out = s.download()
        for f in (FIELD_U, FIELD_V, FIELD_W, FIELD_P, FIELD_PHI):
            s.writefield(str(tmp_path), 3, f)
    for name, key in (("u", "u"), ("v", "v"), ("w", "w"), ("p", "p"), ("phi", "phi")):
        path = tmp_path / f"{name}_00000003.dat"
        raw = path.read_bytes()
        assert len(raw) == 8 * 32 ** 3            # no header, no halo
        arr = np.frombuffer(raw, dtype="<f8").reshape(32, 32, 32)  # Fortran (nx,ny,nz) == C (nz,ny,nx)
        np.testing.assert_array_equal(arr, out[key])


def test_restart_from_files_matches_fresh_run(gpu, tmp_path):
    prm, u, v, w, phi = make()
    for name, a in (("u", u), ("v", v), ("w", w), ("phi", phi)):
        a.astype("<f8").tofile(tmp_path / f"{name}.dat")
    with Solver(prm) as a, Solver(prm) as b:
        a.upload(u, v, w, phi)
        a.step(4)
        ref = a.download()
        for name, f in (("u", FIELD_U), ("v", FIELD_V), ("w", FIELD_W), ("phi", FIELD_PHI)):
            b.readfield(str(tmp_path / f"{name}.dat"), f)
        b.step(4)
        got = b.download()
    for k in ("u", "v", "w", "phi", "p"):
        np.testing.assert_array_equal(got[k], ref[k])


def test_readfield_errors(gpu, tmp_path):
    prm, u, v, w, phi = make()
    short = tmp_path / "short.dat"
    np.zeros(100).tofile(short)
    with Solver(prm) as s:
        with pytest.raises(MhitIOError, match="short read"):
            s.readfield(str(short), FIELD_U)
        with pytest.raises(MhitIOError, match="cannot open"):
            s.readfield(str(tmp_path / "missing.dat"), FIELD_U)


def test_driver_runs_input_file(gpu, tmp_path):
    """python -m mhit36_mixedp_b200.run with an input.inp: Taylor-Green start, dumps every 2 steps."""
    inp = tmp_path / "input.inp"
    inp.write_text("\n".join(["0", "0", "4", "2", "0", "0", "0.0002", "0.006", "1.0", "1.0", "1.0", "1.0", "2.0",
                              "0.5", "1.0d0", "1.0", "0", "1"]) + "\n")
    out = tmp_path / "output"
    r = subprocess.run([sys.executable, "-m", "mhit36_mixedp_b200.run", "--input", str(inp), "--n", "32",
                        "--outdir", str(out)], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    names = sorted(os.listdir(out))
    assert names == sorted(f"{f}_{t:08d}.dat" for f in ("u", "v", "w", "p") for t in (0, 2, 4))
