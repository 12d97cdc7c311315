"""The C++ host driver on the GPU: the same run as the Python driver (run.py) writes the same
field files (Taylor-Green and centred-drop initial conditions of multi/main.f90:322-382, dumps of
:1023-1034).  The two build the initial fields with different sin/cos/tanh implementations, so
the comparison allows 1e-12 of the field maximum."""
import os
import subprocess
import sys

import numpy as np
import pytest

from mhit36_mixedp_b200 import build
from tests.test_abi import INPUT_INP

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("phiflag", [0, 1])
def test_cpp_driver_matches_python_driver(gpu, tmp_path, phiflag):
    inp = tmp_path / "input.inp"
    inp.write_text(INPUT_INP.replace("10000           ! Final", "6           ! Final")
                   .replace("100000           ! Saving", "3           ! Saving"))
    common = ["--input", str(inp), "--n", "32", "--phiflag", str(phiflag)]
    out_c, out_p = tmp_path / "cpp", tmp_path / "py"
    r = subprocess.run([build.build_host()] + common + ["--outdir", str(out_c), "--quiet"], capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([sys.executable, "-m", "mhit36_mixedp_b200.run"] + common + ["--outdir", str(out_p)],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    names = ["u", "v", "w", "p"] + (["phi"] if phiflag else [])
    for t in (0, 3, 6):
        for name in names:
            a = np.fromfile(out_c / f"{name}_{t:08d}.dat")
            b = np.fromfile(out_p / f"{name}_{t:08d}.dat")
            assert a.size == b.size == 32 ** 3
            scale = max(np.abs(b).max(), 1e-300)
            assert np.abs(a - b).max() <= 1e-12 * scale, (name, t)
