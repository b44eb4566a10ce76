"""Parity of the CUDA path (through the C ABI) against the reference's golden
vectors and against the oracle on larger seeded cases.

Tolerances (norm-wise, max|a-b|/max|ref|): FP64 path 1e-12 per array after one
iteration; mixed path 1e-5 for the single-residual quantities.
"""
import numpy as np
import pytest

from phenlei_b200 import cases
from phenlei_b200 import mesh as M
from phenlei_b200 import solver as S
from tests.conftest import rel_err

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MIXED_TOL = 1e-5


def _solver(m, params, precision="fp64"):
    return S.NSSolverUnstruct(m, precision=precision, **params)


@pytest.mark.parametrize("name", ["euler_bump_16x8x2_step1", "euler_tetcube_4_step3"])
def test_fp64_matches_reference_golden(golden, name):
    d = golden(name)
    m = d["mesh_obj"]
    nc = m.n_cell
    s = _solver(m, d["params_dict"])
    for k in ("xfn", "area", "xcc", "vol"):
        assert rel_err(s.geometry(k), d[k]) <= 1e-14, k
    if "state_in" in d:
        s.set_q_cells(d["state_in"][:, :nc])
    hist = s.Relaxation(int(d["nsteps"]))
    assert rel_err(hist, d["res_hist"]) <= FP64_TOL
    assert rel_err(s.get(S.PHX_Q)[:, :nc], d["q"][:, :nc]) <= FP64_TOL
    assert rel_err(s.get(S.PHX_RES)[:, :nc], d["res"][:, :nc]) <= FP64_TOL
    assert rel_err(s.get(S.PHX_DT)[:nc], d["dt"][:nc]) <= FP64_TOL
    assert rel_err(s.get(S.PHX_LIMIT), d["limit"]) <= FP64_TOL
    assert rel_err(s.get(S.PHX_GRADX)[:, :nc], d["gradPrimtiveVarX"][:, :nc]) <= FP64_TOL
    assert rel_err(s.get(S.PHX_GRADY)[:, :nc], d["gradPrimtiveVarY"][:, :nc]) <= FP64_TOL
    assert rel_err(s.get(S.PHX_INVSPEC), d["invSpectralRadius"]) <= FP64_TOL
    assert rel_err(s.AirForceCoef()["sums"], d["forces"]) <= FP64_TOL


def test_fp64_residual_history_matches_reference_golden(golden):
    d = golden("euler_bump_16x8x2_step40")
    m = d["mesh_obj"]
    s = _solver(m, d["params_dict"])
    hist = s.Relaxation(int(d["nsteps"]))
    assert rel_err(hist, d["res_hist"]) <= 1e-10
    assert rel_err(s.get(S.PHX_Q)[:, : m.n_cell], d["q"][:, : m.n_cell]) <= 1e-11


def _oracle_case(m, params, seed):
    from oracle.oracle import Oracle

    o = Oracle(m, params)
    q0 = cases.perturbed_state(m, params, seed=seed)
    o.set_state(q0)
    return o, q0


@pytest.mark.parametrize("precision,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
def test_single_iteration_vs_oracle_euler_bump_64x32x4(precision, tol):
    """The Euler bump mesh (8,192 hexes), perturbed state: every intermediate array."""
    m = M.channel_bump(64, 32, 4)
    params = cases.EULER_BUMP
    o, q0 = _oracle_case(m, params, seed=1)
    o.iterate(1)
    s = _solver(m, params, precision)
    s.set_q_cells(q0)
    s.Relaxation(1)
    nc = m.n_cell
    assert rel_err(s.get(S.PHX_GRADX)[:, :nc], o.work("dqdx")[:, :nc]) <= tol
    assert rel_err(s.get(S.PHX_LIMIT)[:nc], o.work("limit")[:nc]) <= max(tol, 1e-12) * (1e2 if precision == "mixed" else 1)
    assert rel_err(s.get(S.PHX_RES)[:, :nc], o.work("res")[:, :nc]) <= tol
    assert rel_err(s.get(S.PHX_DT)[:nc], o.work("dt")[:nc]) <= tol
    assert rel_err(s.get(S.PHX_DQ)[:, :nc], o.work("dq")[:, :nc]) <= tol * (10 if precision == "mixed" else 1)
    assert rel_err(s.get(S.PHX_Q)[:, :nc], o.q[:, :nc]) <= tol


def test_tet_cube_single_iteration_vs_oracle():
    """Jittered tetrahedra (unstructured LU-SGS schedule with irregular levels)."""
    m = M.tet_cube(12, jitter=0.15, seed=5)
    params = dict(cases.EULER_BUMP, refMachNumber=0.3)
    o, q0 = _oracle_case(m, params, seed=2)
    o.iterate(1)
    s = _solver(m, params)
    s.set_q_cells(q0)
    s.Relaxation(1)
    nc = m.n_cell
    assert rel_err(s.get(S.PHX_RES)[:, :nc], o.work("res")[:, :nc]) <= FP64_TOL
    assert rel_err(s.get(S.PHX_DQ)[:, :nc], o.work("dq")[:, :nc]) <= FP64_TOL
    assert rel_err(s.get(S.PHX_Q)[:, :nc], o.q[:, :nc]) <= FP64_TOL


def test_residual_history_200_steps_vs_oracle():
    m = M.channel_bump(64, 32, 4)
    params = cases.EULER_BUMP
    from oracle.oracle import Oracle

    o = Oracle(m, params)
    ho = o.iterate(200)
    s = _solver(m, params)
    hs = s.Relaxation(200)
    assert rel_err(hs, ho) <= 1e-9
    assert rel_err(s.get(S.PHX_Q)[:, : m.n_cell], o.q[:, : m.n_cell]) <= 1e-10


def test_mixed_converges_like_fp64():
    m = M.channel_bump(32, 16, 2)
    params = cases.EULER_BUMP
    a = _solver(m, params, "fp64").Relaxation(300)
    b = _solver(m, params, "mixed").Relaxation(300)
    assert rel_err(b, a) <= 1e-3


def test_phase_entry_points_equal_relaxation():
    """Calling the phases one by one gives what the fused driver gives."""
    m = M.channel_bump(16, 8, 2)
    params = cases.EULER_BUMP
    q0 = cases.perturbed_state(m, params, seed=4)
    a = _solver(m, params)
    a.set_q_cells(q0)
    a.Relaxation(1)
    b = _solver(m, params)
    b.set_q_cells(q0)
    b.step = 1
    b.Boundary()
    b.ComputeGradientAndLimiter()
    b.UpdateResiduals()
    b.LUSGS()
    b.UpdateFlowField()
    assert np.array_equal(a.get(S.PHX_Q), b.get(S.PHX_Q))


def test_positivity_repair_matches_oracle():
    """A state that drives cells negative exercises the ordered SolutionFix."""
    m = M.channel_bump(16, 8, 2)
    params = dict(cases.EULER_BUMP, CFLStart=200.0, CFLEnd=200.0)
    q0 = cases.perturbed_state(m, params, seed=9, amplitude=0.4)
    from oracle.oracle import Oracle

    o = Oracle(m, params)
    o.set_state(q0)
    o.iterate(1)
    s = _solver(m, params)
    s.set_q_cells(q0)
    s.Relaxation(1)
    assert rel_err(s.get(S.PHX_Q)[:, : m.n_cell], o.q[:, : m.n_cell]) <= FP64_TOL


@pytest.mark.parametrize("blocks", ["1", "2"])
def test_levels_wider_than_grid(monkeypatch, blocks):
    """Sweep levels wider than the cooperative grid (several rounds per level)."""
    monkeypatch.setenv("PHX_LUSGS_MAX_BLOCKS", blocks)
    m = M.channel_bump(64, 32, 8)      # widest level > 64 groups of one 512-thread block
    params = cases.EULER_BUMP
    o, q0 = _oracle_case(m, params, seed=6)
    o.iterate(2)
    s = _solver(m, params)
    s.set_q_cells(q0)
    s.Relaxation(2)
    nc = m.n_cell
    assert rel_err(s.get(S.PHX_Q)[:, :nc], o.q[:, :nc]) <= FP64_TOL
