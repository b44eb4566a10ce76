"""Spalart-Allmaras (NSMB formation) coupled to the NS step on the CUDA path
(through the C ABI): SA boundary values, eddy viscosity, exact source with its
negative-nu~ branch, upwind convection, diffusion, spectral radius and face
matrices, scalar dataflow LU-SGS, and the eddy viscosity fed back into the NS
viscous terms.  Against golden vectors of the reference solver and against
the oracle.

Tolerances (norm-wise, max|a-b|/max|ref|): FP64 path 1e-12 per array after
one iteration, 1e-10 over 30 iterations; mixed path 1e-5 for the NS state
and the residual after one iteration, 1e-4 for nu~ and the eddy viscosity
(their source terms span several decades in FP32).
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
MIXED_TURB_TOL = 1e-4

SA = dict(cases.LAMINAR, viscousType=3, refReNumber=1.0e5, muoo=3.0)


def _solver(m, params, wall_dist, precision="fp64"):
    return S.NSSolverUnstruct(m, precision=precision, wall_dist=wall_dist, **params)


@pytest.mark.parametrize("name", ["sa_bump_16x8x2_step1", "sa_bump_16x8x2_lsq_step3", "sa_bump_prism_16x8x2_step2",
                                  "sa_plate_16x8x2_ausmpwp_step2"])
def test_fp64_sa_matches_reference_golden(golden, name):
    d = golden(name)
    m = d["mesh_obj"]
    nc = m.n_cell
    s = _solver(m, d["params_dict"], d["walldist"])
    s.set_q_cells(d["state_in"][:5, :nc])
    s.set_qt_cells(d["state_in"][5, :nc])
    hist = s.Relaxation(int(d["nsteps"]))
    assert rel_err(hist, d["res_hist"]) <= FP64_TOL
    assert rel_err(s.get(S.PHX_Q)[:, :nc], d["q"][:, :nc]) <= FP64_TOL
    assert rel_err(s.get(S.PHX_RES)[:, :nc], d["res"][:, :nc]) <= FP64_TOL
    assert rel_err(s.get(S.PHX_Q_TURB)[:nc], d["q_turb"][:nc]) <= FP64_TOL
    assert rel_err(s.get(S.PHX_VIST), d["vist"]) <= FP64_TOL
    assert rel_err(s.get(S.PHX_RES_TURB)[:nc], d["res_turb"][:nc]) <= FP64_TOL
    assert rel_err(s.get(S.PHX_VISSPEC), d["visSpectralRadius"]) <= FP64_TOL
    assert rel_err(s.AirForceCoef()["sums"], d["forces"]) <= FP64_TOL


@pytest.mark.parametrize("name", ["sa_bump_16x8x2_step30", "sa_plate_16x8x2_ausmpwp_step20"])
def test_fp64_sa_history_matches_reference_golden(golden, name):
    d = golden(name)
    m = d["mesh_obj"]
    nc = m.n_cell
    s = _solver(m, d["params_dict"], d["walldist"])
    hist = s.Relaxation(int(d["nsteps"]))
    assert rel_err(hist, d["res_hist"]) <= 1e-10
    assert rel_err(s.get(S.PHX_Q)[:, :nc], d["q"][:, :nc]) <= 1e-10
    assert rel_err(s.get(S.PHX_Q_TURB)[:nc], d["q_turb"][:nc]) <= 1e-10


def _oracle(m, params, wd, seed):
    from oracle.oracle import Oracle

    o = Oracle(m, params, wall_dist=wd)
    q0 = cases.perturbed_state(m, params, seed=seed)
    rng = np.random.default_rng(seed)
    qt0 = params["muoo"] * (0.2 + 1.5 * rng.random(m.n_cell))
    qt0[rng.random(m.n_cell) < 0.05] *= -0.1
    o.set_state(q0, qt0)
    return o, q0, qt0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_sa_single_iteration_vs_oracle(precision):
    """8,192-hex bump, SA, perturbed flow and nu~ (a few negative cells)."""
    m = M.channel_bump(64, 32, 4)
    wd = M.wall_distance(m)
    o, q0, qt0 = _oracle(m, SA, wd, seed=3)
    o.iterate(1)
    s = _solver(m, SA, wd, precision)
    s.set_q_cells(q0)
    s.set_qt_cells(qt0)
    s.Relaxation(1)
    nc = m.n_cell
    tol = FP64_TOL if precision == "fp64" else MIXED_TOL
    ttol = FP64_TOL if precision == "fp64" else MIXED_TURB_TOL
    assert rel_err(s.get(S.PHX_RES)[:, :nc], o.work("res")[:, :nc]) <= tol
    assert rel_err(s.get(S.PHX_Q)[:, :nc], o.q[:, :nc]) <= tol
    assert rel_err(s.get(S.PHX_RES_TURB)[:nc], o.work("res_t")[:nc]) <= ttol
    assert rel_err(s.get(S.PHX_VIST)[:nc], o.work("vist")[:nc]) <= ttol
    assert rel_err(s.get(S.PHX_Q_TURB)[:nc], o.work("qt")[:nc]) <= ttol


def test_sa_phase_entry_points_equal_relaxation():
    m = M.channel_bump(16, 8, 2)
    wd = M.wall_distance(m)
    q0 = cases.perturbed_state(m, SA, seed=4)
    a = _solver(m, SA, wd)
    a.set_q_cells(q0)
    a.Relaxation(2)
    b = _solver(m, SA, wd)
    b.set_q_cells(q0)
    for step in (1, 2):
        b.step = step
        b.Boundary()
        b.ComputeGradientAndLimiter()
        b.UpdateResiduals()
        b.LUSGS()
        b.UpdateFlowField()
        b.TurbUpdateResiduals()
        b.TurbLUSGS()
        b.TurbUpdateFlowField()
    assert np.array_equal(a.get(S.PHX_Q), b.get(S.PHX_Q))
    assert np.array_equal(a.get(S.PHX_Q_TURB), b.get(S.PHX_Q_TURB))


def test_sa_residual_history_100_steps_vs_oracle():
    from oracle.oracle import Oracle

    m = M.channel_bump(32, 16, 4)
    wd = M.wall_distance(m)
    o = Oracle(m, SA, wall_dist=wd)
    ho = o.iterate(100)
    s = _solver(m, SA, wd)
    hs = s.Relaxation(100)
    assert rel_err(hs, ho) <= 1e-9
    assert rel_err(s.get(S.PHX_Q_TURB)[: m.n_cell], o.work("qt")[: m.n_cell]) <= 1e-9


def test_mixed_sa_from_free_stream_matches_fp64():
    """Transonic bump parameters (M 0.8, Re 1e7) from the uniform free stream,
    where the vorticity is exactly zero and the source's implicit part forms
    products of order 1e48 that overflow FP32: the mixed path keeps nu~ and
    the eddy viscosity finite and within 1e-3 of the FP64 path after five
    iterations."""
    m = M.channel_bump(32, 16, 4, thickness=0.08, wall_spacing=0.001, prism_layers=4)
    wd = M.wall_distance(m)
    nc = m.n_cell
    a = _solver(m, cases.SA_BUMP, wd, "fp64")
    b = _solver(m, cases.SA_BUMP, wd, "mixed")
    a.Relaxation(5)
    b.Relaxation(5)
    qa, qb = a.get(S.PHX_Q_TURB)[:nc], b.get(S.PHX_Q_TURB)[:nc]
    assert np.all(np.isfinite(qb))
    assert rel_err(qb, qa) <= 1e-3
    assert rel_err(b.get(S.PHX_VIST)[:nc], a.get(S.PHX_VIST)[:nc]) <= 1e-3
    assert np.max(b.get(S.PHX_VIST)[:nc]) > 0.0


def test_sa_requires_wall_distance():
    m = M.channel_bump(16, 8, 2)
    with pytest.raises(S.PhxError):
        S.NSSolverUnstruct(m, **SA)


@pytest.mark.parametrize("precision,tol,turb_tol", [("fp64", FP64_TOL, FP64_TOL), ("mixed", MIXED_TOL, MIXED_TURB_TOL)])
def test_plate_vs_oracle(precision, tol, turb_tol):
    """The SA flat plate flow (SA, AUSMPW+, M 0.2, Re 5e6, CFL 50) on a 32x12x2 flat
    plate, perturbed flow and nu~: one iteration, then 30 more."""
    m = M.flat_plate(32, 12, 2, first_spacing=1e-4)
    wd = M.wall_distance(m)
    params = cases.SA_PLATE
    o, q0, qt0 = _oracle(m, params, wd, seed=13)
    s = _solver(m, params, wd, precision)
    s.set_q_cells(q0)
    s.set_qt_cells(qt0)
    nc = m.n_cell
    o.iterate(1)
    s.Relaxation(1)
    assert rel_err(s.get(S.PHX_RES)[:, :nc], o.work("res")[:, :nc]) <= tol
    assert rel_err(s.get(S.PHX_Q)[:, :nc], o.q[:, :nc]) <= tol
    assert rel_err(s.get(S.PHX_Q_TURB)[:nc], o.work("qt")[:nc]) <= turb_tol
    ho = o.iterate(30)
    hs = s.Relaxation(30)
    assert rel_err(hs, ho) <= (1e-10 if precision == "fp64" else 1e-3)
    assert rel_err(s.AirForceCoef()["sums"], o.forces()) <= (1e-10 if precision == "fp64" else 1e-3)
