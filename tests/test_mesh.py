"""Mesh generator sanity: closed cells and consistent orientation."""
import numpy as np
import pytest

from phenlei_b200 import mesh as M
from oracle.oracle import Oracle


@pytest.mark.parametrize("m", [M.channel_bump(8, 4, 2), M.tet_cube(3), M.flat_plate(12, 6, 2)])
def test_cells_closed_and_positive(m):
    o = Oracle(m, {"refMachNumber": 0.5})
    nc, nb = m.n_cell, m.n_bface
    s = np.zeros((nc, 3))
    a = o.geo["area"]
    n = np.stack([o.geo["xfn"] * a, o.geo["yfn"] * a, o.geo["zfn"] * a], axis=1)
    np.add.at(s, m.left, n)
    np.add.at(s, m.right[nb:], -n[nb:])
    assert np.max(np.abs(s)) < 1e-12
    assert np.all(o.geo["vol"][:nc] > 0)
    # normals point from left to right cell centres
    d = np.stack([o.geo["xfc"] - o.geo["xcc"][m.left], o.geo["yfc"] - o.geo["ycc"][m.left],
                  o.geo["zfc"] - o.geo["zcc"][m.left]], axis=1)
    assert np.all(np.einsum("ij,ij->i", d, n) > 0)


def test_face_ordering():
    m = M.channel_bump(8, 4, 2)
    assert np.all(m.right[: m.n_bface] == -1)
    assert np.all(m.right[m.n_bface:] >= 0)
    assert m.n_cell == 64
