"""The reference build used as the CPU baseline (oracle/refbuild): the OpenMP
build (one zone per thread over the reference's OpenMP zone loops) gives the
same iterations as the serial build on the same zones, bit for bit.  Runs
only where the reference build exists.  CPU only."""
import os

import numpy as np
import pytest

from oracle import refrun
from phenlei_b200 import cases
from phenlei_b200 import mesh as M
from phenlei_b200 import partition as P

pytestmark = pytest.mark.skipif(not (refrun.available() and os.path.exists(refrun.HARNESS_OMP)),
                                reason="the reference build (oracle/_ref) is absent")


@pytest.mark.parametrize("case,params", [("laminar", dict(cases.LAMINAR)), ("sa", dict(cases.SA_BUMP))])
def test_openmp_reference_equals_serial_zones(case, params):
    m = M.channel_bump(32, 16, 4)
    parts = P.split(m, P.slab_owner(m, 6))
    q0 = cases.perturbed_state(m, params, seed=3)
    wd = M.wall_distance(m) if case == "sa" else None
    nt = lambda p: p.mesh.n_cell + p.mesh.n_bface  # noqa: E731
    kw = dict(dumps=[("q", 5, nt)], states=[q0[:, p.cells] for p in parts],
              wall_dists=None if wd is None else [wd[p.cells] for p in parts])
    a = refrun.run_reference_zones(parts, params, 3, **kw)
    b = refrun.run_reference_zones(parts, params, 3, threads=4, **kw)
    assert np.array_equal(a["res_hist"], b["res_hist"])
    for za, zb in zip(a["zones"], b["zones"]):
        assert np.array_equal(za["q"], zb["q"])
