"""Laminar NS on the CUDA path (through the C ABI): Sutherland viscosity,
GG-cell and least-squares gradients, temperature gradient, viscous flux,
viscous spectral radius and the viscous LU-SGS terms, against golden vectors
of the reference solver and against the oracle.

Tolerances (norm-wise, max|a-b|/max|ref|): FP64 path 1e-12 per array after
one iteration; mixed path 1e-5 for the single-residual quantities.
"""
import pytest

from phenlei_b200 import cases
from phenlei_b200 import mesh as M
from phenlei_b200 import solver as S
from tests.conftest import rel_err

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MIXED_TOL = 1e-5

LAMINAR = cases.LAMINAR


def _solver(m, params, precision="fp64"):
    return S.NSSolverUnstruct(m, precision=precision, **params)


@pytest.mark.parametrize("name", ["laminar_bump_16x8x2_lsq_step1", "laminar_tetcube_4_lsq_step3"])
def test_fp64_laminar_matches_reference_golden(golden, name):
    d = golden(name)
    m = d["mesh_obj"]
    nc = m.n_cell
    s = _solver(m, d["params_dict"])
    if "state_in" in d:
        s.set_q_cells(d["state_in"][:, :nc])
    hist = s.Relaxation(int(d["nsteps"]))
    assert rel_err(hist, d["res_hist"]) <= FP64_TOL
    assert rel_err(s.get(S.PHX_Q)[:, :nc], d["q"][:, :nc]) <= FP64_TOL
    assert rel_err(s.get(S.PHX_RES)[:, :nc], d["res"][:, :nc]) <= FP64_TOL
    assert rel_err(s.get(S.PHX_DT)[:nc], d["dt"][:nc]) <= FP64_TOL
    assert rel_err(s.get(S.PHX_VISSPEC), d["visSpectralRadius"]) <= FP64_TOL
    assert rel_err(s.get(S.PHX_GRADY)[:, :nc], d["gradPrimtiveVarY"][:, :nc]) <= FP64_TOL
    assert rel_err(s.AirForceCoef()["sums"], d["forces"]) <= FP64_TOL


def test_fp64_laminar_history_matches_reference_golden(golden):
    d = golden("laminar_bump_16x8x2_step20")
    m = d["mesh_obj"]
    s = _solver(m, d["params_dict"])
    hist = s.Relaxation(int(d["nsteps"]))
    assert rel_err(hist, d["res_hist"]) <= 1e-10
    assert rel_err(s.get(S.PHX_Q)[:, : m.n_cell], d["q"][:, : m.n_cell]) <= 1e-11


@pytest.mark.parametrize("grad", ["ggcell", "lsq"])
@pytest.mark.parametrize("precision,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
def test_laminar_single_iteration_vs_oracle(grad, precision, tol):
    """8,192-hex bump with no-slip walls, perturbed state: every intermediate array."""
    from oracle.oracle import Oracle

    m = M.channel_bump(64, 32, 4)
    params = dict(LAMINAR, gradientName=grad)
    o = Oracle(m, params)
    q0 = cases.perturbed_state(m, params, seed=3)
    o.set_state(q0)
    o.iterate(1)
    s = _solver(m, params, precision)
    s.set_q_cells(q0)
    s.Relaxation(1)
    nc = m.n_cell
    assert rel_err(s.get(S.PHX_GRADX)[:, :nc], o.work("dqdx")[:, :nc]) <= tol
    assert rel_err(s.get(S.PHX_VISSPEC), o.work("vis_spec")) <= tol
    assert rel_err(s.get(S.PHX_RES)[:, :nc], o.work("res")[:, :nc]) <= tol
    assert rel_err(s.get(S.PHX_DT)[:nc], o.work("dt")[:nc]) <= tol
    assert rel_err(s.get(S.PHX_DQ)[:, :nc], o.work("dq")[:, :nc]) <= tol * (10 if precision == "mixed" else 1)
    assert rel_err(s.get(S.PHX_Q)[:, :nc], o.q[:, :nc]) <= tol


def test_laminar_tet_cube_vs_oracle():
    """The laminar cube's element type: jittered tetrahedra, LSQ, far field all round."""
    from oracle.oracle import Oracle

    m = M.tet_cube(10, jitter=0.15, seed=5)
    params = dict(LAMINAR, gradientName="lsq")
    o = Oracle(m, params)
    q0 = cases.perturbed_state(m, params, seed=2)
    o.set_state(q0)
    o.iterate(2)
    s = _solver(m, params)
    s.set_q_cells(q0)
    s.Relaxation(2)
    nc = m.n_cell
    assert rel_err(s.get(S.PHX_RES)[:, :nc], o.work("res")[:, :nc]) <= FP64_TOL
    assert rel_err(s.get(S.PHX_Q)[:, :nc], o.q[:, :nc]) <= FP64_TOL


def test_euler_lsq_vs_oracle():
    """Least-squares gradient on the inviscid path."""
    from oracle.oracle import Oracle

    m = M.channel_bump(32, 16, 4)
    params = dict(cases.EULER_BUMP, gradientName="lsq")
    o = Oracle(m, params)
    q0 = cases.perturbed_state(m, params, seed=8)
    o.set_state(q0)
    o.iterate(3)
    s = _solver(m, params)
    s.set_q_cells(q0)
    s.Relaxation(3)
    nc = m.n_cell
    assert rel_err(s.get(S.PHX_Q)[:, :nc], o.q[:, :nc]) <= 1e-11


def test_laminar_residual_history_150_steps_vs_oracle():
    from oracle.oracle import Oracle

    m = M.channel_bump(32, 16, 4)
    o = Oracle(m, LAMINAR)
    ho = o.iterate(150)
    s = _solver(m, LAMINAR)
    hs = s.Relaxation(150)
    assert rel_err(hs, ho) <= 1e-9
