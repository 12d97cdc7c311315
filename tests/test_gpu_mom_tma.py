"""The momentum kernel's two ways of filling its plane rings give the same bits.

k_mom keeps rings of u, v, w and phi^{n+1} planes in shared memory.  Tiles whose rings need no
periodic wrap in x and y fill them with TMA boxes (cp.async.bulk.tensor, completion on an
mbarrier); the others copy 16-byte pairs per thread.  The ring contents, and so every result,
must not depend on which way a tile took: the same steps with TMA switched off must give the
same bits, at sizes with interior tiles (x tiles of 32 cells and y tiles of 8 not touching the
boundary), with and without the phase field, and against the oracle.
"""
import numpy as np
import pytest

from mhit36_mixedp_b200 import Params, Solver, _lib, synth
from oracle import mhit_oracle as orc

pytestmark = pytest.mark.gpu


def run(shape, phiflag, tma, nsteps=3):
    nx, ny, nz = shape
    u, v, w = synth.solenoidal_velocity(nx, 3, ny=ny, nz=nz)
    phi = synth.drops_phi(nx, synth.drop_centres(6, 4), 0.4, 2 * np.pi / nx) if phiflag else None
    with Solver(Params(nx=nx, ny=ny, nz=nz, dt=2e-4, mu=0.004, phiflag=phiflag, radius=0.4, sigma=0.3,
                       acdi_clamp=1)) as s:
        assert _lib.load().mhit_debug_set_mom_tma(s._ctx, int(tma)) == 0
        s.upload(u, v, w, phi)
        s.step(nsteps)
        return s.download(fields=("u", "v", "w") + (("phi",) if phiflag else ())), (u, v, w, phi)


@pytest.mark.parametrize("phiflag", [0, 1])
@pytest.mark.parametrize("n", [128, 256])
def test_tma_rings_bit_identical(gpu, n, phiflag):
    a, _ = run((n, n, n), phiflag, True)
    b, _ = run((n, n, n), phiflag, False)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])


def test_tma_rings_match_oracle(gpu):
    n = 128
    got, (u, v, w, phi) = run((n, n, n), 1, True, nsteps=2)
    op = orc.Params(nx=n, dt=2e-4, mu=0.004, phiflag=1, radius=0.4, sigma=0.3, acdi_clamp=1)
    st = orc.new_state(op, u, v, w, phi=phi)
    orc.run(op, st, 2)
    for k in got:
        ref = getattr(st, k)
        e = np.abs(got[k] - ref).max() / np.abs(ref).max()
        assert e < 1e-12, (k, e)
