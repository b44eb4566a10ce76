"""GG-node gradient (the reference's default gradientName) on the CUDA path
(through the C ABI): node values with the boundary-type priorities and
1/distance weights, face values from the face's nodes, the temperature node
values of the previous state, and with Spalart-Allmaras the node values of
nu~ from the turbulence PostSolve, against golden vectors of the reference
solver and against the oracle.

Tolerances (norm-wise, max|a-b|/max|ref|): FP64 path 1e-12 per array after
one to three iterations, 1e-10 over 20; the z gradients of the quasi-2-D
16x8x2 bump are round-off (1e-16) and are bounded against the gradient's
scale instead.  Mixed path 1e-5 for the state and residual, 5e-5 for the
gradients (the node sums and face averages add FP32 operations ahead of
the cancelling face differences).
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


@pytest.mark.parametrize("name", ["euler_bump_16x8x2_ggnode_step1", "laminar_bump_16x8x2_ggnode_step1",
                                  "euler_tetcube_4_ggnode_step3"])
def test_fp64_ggnode_matches_reference_golden(golden, name):
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
    assert rel_err(s.get(S.PHX_GRADX)[:, :nc], d["gradPrimtiveVarX"][:, :nc]) <= FP64_TOL
    assert rel_err(s.get(S.PHX_GRADY)[:, :nc], d["gradPrimtiveVarY"][:, :nc]) <= FP64_TOL
    scale = max(np.abs(d[k][:, :nc]).max() for k in ("gradPrimtiveVarX", "gradPrimtiveVarY", "gradPrimtiveVarZ"))
    assert np.abs(s.get(S.PHX_GRADZ)[:, :nc] - d["gradPrimtiveVarZ"][:, :nc]).max() <= FP64_TOL * scale
    assert rel_err(s.AirForceCoef()["sums"], d["forces"]) <= FP64_TOL


def test_fp64_ggnode_history_matches_reference_golden(golden):
    """Twenty iterations: the temperature node values lag one state behind."""
    d = golden("laminar_bump_16x8x2_ggnode_step20")
    m = d["mesh_obj"]
    s = _solver(m, d["params_dict"])
    hist = s.Relaxation(int(d["nsteps"]))
    assert rel_err(hist, d["res_hist"]) <= 1e-10
    assert rel_err(s.get(S.PHX_Q)[:, : m.n_cell], d["q"][:, : m.n_cell]) <= 1e-11


@pytest.mark.parametrize("precision,tol,gtol", [("fp64", FP64_TOL, FP64_TOL), ("mixed", MIXED_TOL, 5e-5)])
def test_ggnode_single_iteration_vs_oracle(precision, tol, gtol):
    """8,192-hex bump with wall, far-field and symmetry nodes, perturbed state."""
    from oracle.oracle import Oracle

    m = M.channel_bump(64, 32, 4)
    params = dict(cases.LAMINAR, gradientName="ggnode")
    o = Oracle(m, params)
    q0 = cases.perturbed_state(m, params, seed=3)
    o.set_state(q0)
    o.iterate(1)
    s = _solver(m, params, precision)
    s.set_q_cells(q0)
    s.Relaxation(1)
    nc = m.n_cell
    assert rel_err(s.get(S.PHX_GRADX)[:, :nc], o.work("dqdx")[:, :nc]) <= gtol
    assert rel_err(s.get(S.PHX_GRADZ)[:, :nc], o.work("dqdz")[:, :nc]) <= gtol
    assert rel_err(s.get(S.PHX_RES)[:, :nc], o.work("res")[:, :nc]) <= tol
    assert rel_err(s.get(S.PHX_Q)[:, :nc], o.q[:, :nc]) <= tol


def test_ggnode_history_vs_oracle():
    from oracle.oracle import Oracle

    m = M.channel_bump(32, 16, 4)
    params = dict(cases.LAMINAR, gradientName="ggnode")
    o = Oracle(m, params)
    ho = o.iterate(60)
    s = _solver(m, params)
    hs = s.Relaxation(60)
    assert rel_err(hs, ho) <= 1e-9


@pytest.mark.parametrize("name", ["sa_bump_16x8x2_ggnode_step1", "sa_bump_16x8x2_ggnode_step20"])
def test_fp64_sa_ggnode_matches_reference_golden(golden, name):
    """GG-node with Spalart-Allmaras: the nu~ gradient from the node values the
    turbulence PostSolve forms (face-based sums over a running face-to-node
    position, symmetry / far-field / wall nodes rebuilt from those faces)."""
    d = golden(name)
    m = d["mesh_obj"]
    nc = m.n_cell
    nsteps = int(d["nsteps"])
    tol = FP64_TOL if nsteps == 1 else 1e-10
    s = S.NSSolverUnstruct(m, wall_dist=d["walldist"], **d["params_dict"])
    if "state_in" in d:
        s.set_q_cells(d["state_in"][:5, :nc])
        s.set_qt_cells(d["state_in"][5, :nc])
    hist = s.Relaxation(nsteps)
    assert rel_err(hist, d["res_hist"]) <= tol
    assert rel_err(s.get(S.PHX_Q)[:, :nc], d["q"][:, :nc]) <= tol
    assert rel_err(s.get(S.PHX_Q_TURB)[:nc], d["q_turb"][:nc]) <= tol
    assert rel_err(s.get(S.PHX_RES_TURB)[:nc], d["res_turb"][:nc]) <= tol
    assert rel_err(s.get(S.PHX_GRAD_TURB)[0, :nc], d["gradTurbulenceX"][:nc]) <= tol
    assert rel_err(s.AirForceCoef()["sums"], d["forces"]) <= tol
