"""Error paths of the step and of the droplet labelling, driven from the host without a fault.

* CFL: the reference stops when cou = gumax dt dxi exceeds 7 (``multi/main.f90:1003-1007``).
  A time step large enough to push the Courant number past 7 must make ``mhit_step`` return
  MHIT_ERR_CFL with the device flag set, and the reported Courant number must be gumax dt dxi of
  the step's own velocity; a time step below the limit must not raise it.
* Droplet labelling: every union-find loop is bounded and sets an error flag when the bound runs
  out (a corrupted parent chain would otherwise loop).  The test hook lowers the bound to 1, so
  ordinary chains of a drop run out; ``mhit_label_drops`` must return MHIT_ERR_STATE, and with the
  default bound the same call must succeed.
"""
import ctypes
import math

import numpy as np
import pytest

from mhit36_mixedp_b200 import MhitCFLError, MhitStateError, Params, Solver, _lib, synth

pytestmark = pytest.mark.gpu


def test_cfl_above_seven_stops_the_step(gpu):
    n = 32
    u, v, w = synth.solenoidal_velocity(n, 0)
    dxi = n / (2 * math.pi)
    # gumax of a unit-rms field is about 3: dt = 1 gives a Courant number far above 7
    with Solver(Params(nx=n, dt=1.0, mu=0.006)) as s:
        s.upload(u, v, w)
        lib = _lib.load()
        rc = lib.mhit_step(s._ctx, 1)
        assert rc == _lib.MHIT_ERR_CFL, (rc, lib.mhit_last_error())
        assert b"CFL" in lib.mhit_last_error()
        d = s.diagnostics()
        assert d["flags"] & 2, d["flags"]
        assert not (d["flags"] & 1)  # no NaN: the stop is the Courant number's
        assert d["cfl"] > 7.0
        assert abs(d["cfl"] - d["gumax"] * 1.0 * dxi) <= 1e-12 * d["cfl"]
        out = s.download(fields=("u", "v", "w"))
        assert abs(d["gumax"] - max(out[f].max() for f in "uvw")) <= 1e-12 * abs(d["gumax"])
        with pytest.raises(MhitCFLError):
            s.step(1)


def test_cfl_below_seven_runs(gpu):
    n = 32
    u, v, w = synth.solenoidal_velocity(n, 0)
    with Solver(Params(nx=n, dt=5e-4, mu=0.006)) as s:
        s.upload(u, v, w)
        s.step(3)
        d = s.diagnostics()
        assert d["flags"] == 0
        assert 0.0 < d["cfl"] < 7.0


def test_label_bound_exhaustion_is_an_error_status(gpu):
    n = 64
    u, v, w = synth.solenoidal_velocity(n, 1)
    phi = synth.drops_phi(n, synth.drop_centres(6, 2), 0.5, 2 * np.pi / n)
    with Solver(Params(nx=n, phiflag=1, radius=0.5, sigma=0.5)) as s:
        s.upload(u, v, w, phi)
        lib = _lib.load()
        ok = s.label_drops(0.5, 6)
        assert len(ok["cells"]) >= 1
        assert lib.mhit_debug_set_label_bound(s._ctx, 1) == 0
        with pytest.raises(MhitStateError, match="bound exceeded"):
            s.label_drops(0.5, 6)
        with pytest.raises(MhitStateError, match="bound exceeded"):
            s.label_drops(0.5, 26)
        assert lib.mhit_debug_set_label_bound(s._ctx, 0) == 0
        again = s.label_drops(0.5, 6)
        np.testing.assert_array_equal(again["cells"], ok["cells"])
        assert lib.mhit_debug_set_label_bound(s._ctx, ctypes.c_longlong(-1)) == _lib.MHIT_ERR_ARG
