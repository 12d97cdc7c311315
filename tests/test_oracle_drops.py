"""The droplet-labelling oracle (oracle/mhit_oracle.py: label_components, drop_statistics) on
cases whose answer is known without it: the synthetic sphere of
post/unionfind_periodic/main.f90:124-129, a drop wrapped through the periodic corner, and two
blocks that touch only along an edge (one drop with 26 neighbours, two with 6)."""
import math

import numpy as np
import pytest

from oracle import mhit_oracle as orc


def stats(phi, conn=6):
    lab = orc.label_components(phi, 0.5, conn)
    z = np.zeros_like(phi)
    return lab, orc.drop_statistics(lab, z, z, z)


@pytest.mark.parametrize("nx", [32, 64])
def test_reference_sphere(nx):
    phi, (cx, cy, cz, r2) = orc.reference_test_sphere(nx)
    lab, st = stats(phi)
    dx = 2 * math.pi / nx
    assert list(st["cells"]) == [int(phi.sum())]
    # 1-based centre index c -> cell centre (c - 1/2) dx
    for key, c in (("x", cx), ("y", cy), ("z", cz)):
        assert abs(st[key][0] - (c - 0.5) * dx) < 1e-12
    assert st["volume"][0] == phi.sum() * dx * dx * dx  # real(cells)*dx*dx*dx, :436
    assert st["label"][0] == np.flatnonzero(phi.ravel() >= 0.5)[0]


def test_drop_through_the_periodic_corner():
    n = 32
    idx = np.arange(n)
    d = np.minimum(idx, n - idx)  # periodic distance to cell 0
    phi = ((d[None, None, :] ** 2 + d[None, :, None] ** 2 + d[:, None, None] ** 2) <= 16).astype(float)
    lab, st = stats(phi)
    assert len(st["cells"]) == 1 and st["cells"][0] == int(phi.sum())
    dx = 2 * math.pi / n
    for key in ("x", "y", "z"):  # circular mean of cells ... -1, 0, 1 ... is the centre of cell 0
        c = st[key][0]
        assert min(abs(c - 0.5 * dx), abs(c - 0.5 * dx - 2 * math.pi)) < 1e-12


def test_edge_contact_needs_26_neighbours():
    n = 16
    phi = np.zeros((n, n, n))
    phi[2:5, 2:5, 2:5] = 1.0
    phi[2:5, 5:8, 5:8] = 1.0  # shares only the edge along z at (y, x) = (4|5, 4|5)
    assert len(stats(phi, 6)[1]["cells"]) == 2
    assert len(stats(phi, 26)[1]["cells"]) == 1
    phi2 = np.zeros((n, n, n))
    phi2[2:4, 2:4, 2:4] = 1.0
    phi2[4:6, 4:6, 4:6] = 1.0  # corner contact only
    assert len(stats(phi2, 6)[1]["cells"]) == 2
    assert len(stats(phi2, 26)[1]["cells"]) == 1


def test_threshold_is_inclusive():
    phi = np.zeros((8, 8, 8))
    phi[3, 3, 3] = 0.5
    assert list(stats(phi)[1]["cells"]) == [1]
    phi[3, 3, 3] = np.nextafter(0.5, 0.0)
    assert len(stats(phi)[1]["cells"]) == 0
