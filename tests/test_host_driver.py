"""The C++ host driver (mhit36_mixedp_b200/host/mhit_main.cpp) over the C ABI: it builds, prints
its usage, and reads input.inp exactly as the Python binding does (--dry-run touches no GPU)."""
import json
import os
import subprocess

import pytest

from mhit36_mixedp_b200 import api, build
from tests.test_abi import INPUT_INP


@pytest.fixture(scope="module")
def driver():
    return build.build_host()


def test_driver_usage(driver):
    r = subprocess.run([driver, "--help"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "usage: mhit_main" in r.stdout
    r = subprocess.run([driver, "--bogus"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2


def test_driver_reads_input_like_the_binding(driver, tmp_path):
    p = tmp_path / "input.inp"
    p.write_text(INPUT_INP.replace("1.0d0", "2.5D-1").replace("10000           ! Final", "40           ! Final"))
    r = subprocess.run([driver, "--input", str(p), "--n", "64", "--dry-run"], capture_output=True, text=True,
                       timeout=60)
    assert r.returncode == 0, r.stderr
    got = json.loads(r.stdout)
    prm, run = api.read_input(str(p), nx=64)
    for k in ("dt", "mu", "rho", "f1", "f2", "f3", "k0", "radius", "sigma", "epsr", "npart"):
        assert got[k] == getattr(prm, k), k
    for k, v in run.items():
        assert got[k] == v, k
    assert got["steps"] == run["tfin"] - run["tstart"] == 40
    r = subprocess.run([driver, "--input", str(tmp_path / "missing.inp"), "--dry-run"], capture_output=True,
                       text=True, timeout=60)
    assert r.returncode == 1 and "mhit_read_input" in r.stderr
