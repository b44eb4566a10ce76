"""Two benchmark cases run as stated, against the oracle (the CPU
restatement of the reference path, pinned bit-exact to the reference build).

* The Euler bump (64x32x4 hexes, uniform free stream, CFL ramp to 10): all
  2,000 iterations.  The FP64 path follows the oracle's residual
  history (1e-9) and wall force sums (1e-10) over the whole run, and the mixed
  path's CL and CD after 2,000 iterations lie within 1e-4 of the oracle's:
  the accuracy condition of the headline metric, on the case the oracle can
  run to the end in seconds.
* The laminar cube at its full size (100^3 hexes x 6 jittered tets,
  6,000,000 cells, least-squares gradient, free stream plus seeded
  sinusoids): one residual and one LU-SGS sweep.  Residual 1e-12 (FP64) and
  1e-5 (mixed); dq after the sweep 1e-12 (FP64) and 1e-4 (mixed).

Tolerances are norm-wise, max|a-b| / max|ref|.
"""
import numpy as np
import pytest

from phenlei_b200 import cases
from phenlei_b200 import mesh as M
from phenlei_b200 import solver as S
from tests.conftest import rel_err

pytestmark = pytest.mark.gpu

EULER_BUMP_STEPS = 2000


@pytest.fixture(scope="module")
def euler_bump_run():
    from oracle.oracle import Oracle

    m = M.channel_bump(64, 32, 4)
    params = dict(cases.EULER_BUMP)
    o = Oracle(m, params)
    hist = o.iterate(EULER_BUMP_STEPS)
    return m, params, hist, o.forces(), o.q.copy()


def test_euler_bump_fp64_full_run_matches_oracle(euler_bump_run):
    m, params, ho, fo, qo = euler_bump_run
    s = S.NSSolverUnstruct(m, precision="fp64", **params)
    hs = s.Relaxation(EULER_BUMP_STEPS)
    # the run converges: the residual monitor drops by more than three orders
    assert ho[-1] < 1e-3 * ho[0]
    assert rel_err(hs, ho) <= 1e-9
    assert rel_err(s.AirForceCoef()["sums"], fo) <= 1e-10
    assert rel_err(s.get(S.PHX_Q)[:, : m.n_cell], qo[:, : m.n_cell]) <= 1e-10


def test_euler_bump_mixed_forces_within_1e4_of_oracle(euler_bump_run):
    m, params, ho, fo, _ = euler_bump_run
    s = S.NSSolverUnstruct(m, precision="mixed", **params)
    hs = s.Relaxation(EULER_BUMP_STEPS)
    f = s.AirForceCoef()
    ref = S.force_coefficients(fo, params.get("attackd", 0.0), params.get("angleSlide", 0.0))
    assert abs(f["CL"] - ref["CL"]) <= 1e-4
    assert abs(f["CD"] - ref["CD"]) <= 1e-4
    # the mixed run converges as far as the FP64 one
    assert hs[-1] <= 2.0 * ho[-1]


def test_laminar_cube_6M_residual_and_sweep():
    from oracle.oracle import Oracle

    m = M.tet_cube(100, jitter=0.15, seed=1)
    assert m.n_cell == 6_000_000
    params = dict(cases.LAMINAR, gradientName="lsq")
    q0 = cases.perturbed_state(m, params, seed=1)
    o = Oracle(m, params)
    o.set_state(q0)
    o.iterate(1)
    nc = m.n_cell
    res_o, dq_o, q_o = o.work("res")[:, :nc].copy(), o.work("dq")[:, :nc].copy(), o.q[:, :nc].copy()
    del o
    for precision, tol_res, tol_dq in (("fp64", 1e-12, 1e-12), ("mixed", 1e-5, 1e-4)):
        s = S.NSSolverUnstruct(m, precision=precision, **params)
        s.set_q_cells(q0)
        s.Relaxation(1)
        assert rel_err(s.get(S.PHX_RES)[:, :nc], res_o) <= tol_res, precision
        assert rel_err(s.get(S.PHX_DQ)[:, :nc], dq_o) <= tol_dq, precision
        assert rel_err(s.get(S.PHX_Q)[:, :nc], q_o) <= tol_res, precision
        s.close()
