"""Failure detection on the GPU without a GPU fault.

* A dependency wait that nothing satisfies: the forward LU-SGS result of one
  cell is held back (phx_fault_hold_cell), the wait on it runs out after a
  short limit (phx_set_wait_limit), the step returns PHX_ERR_TIMEOUT, and the
  context stays usable: after the hold is lifted and the state uploaded again,
  the next step matches the oracle.
* A non-finite state from the host: a NaN pressure in one cell.  The first
  step's residual stays finite (as the oracle's does), its LU-SGS sweep
  spreads the NaN, the second step's residual monitor is NaN and the run
  returns PHX_ERR_NUMERIC (the reference aborts on a diverged residual,
  API/Physics/src/Residual.cpp:218-222); the context again recovers with a
  new state.

The waits are bounded and end in an error status; nothing traps, faults or
hangs.
"""
import numpy as np
import pytest

from phenlei_b200 import cases
from phenlei_b200 import mesh as M
from phenlei_b200 import solver as S
from tests.conftest import rel_err

pytestmark = pytest.mark.gpu


def _oracle_step(m, params, q0):
    from oracle.oracle import Oracle

    o = Oracle(m, params)
    o.set_state(q0)
    o.iterate(1)
    return o.q[:, : m.n_cell].copy()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_wait_that_runs_out_returns_timeout_and_context_recovers(precision):
    m = M.channel_bump(32, 16, 2)
    params = cases.EULER_BUMP
    q0 = cases.perturbed_state(m, params, seed=11)
    s = S.NSSolverUnstruct(m, precision=precision, **params)
    s.set_q_cells(q0)
    s.set_wait_limit(100_000)
    s.fault_hold_cell(m.n_cell // 2)
    with pytest.raises(S.PhxError, match="PHX_ERR_TIMEOUT"):
        s.Relaxation(1)
    # lift the hold, start again from the same state
    s.fault_hold_cell(-1)
    s.step = 0
    s.set_q_cells(q0)
    s.Relaxation(1)
    tol = 1e-12 if precision == "fp64" else 1e-5
    assert rel_err(s.get(S.PHX_Q)[:, : m.n_cell], _oracle_step(m, params, q0)) <= tol


def test_non_finite_state_returns_numeric_error_and_context_recovers():
    m = M.channel_bump(32, 16, 2)
    params = cases.EULER_BUMP
    q0 = cases.perturbed_state(m, params, seed=12)
    bad = q0.copy()
    bad[4, m.n_cell // 3] = np.nan
    s = S.NSSolverUnstruct(m, precision="fp64", **params)
    s.set_q_cells(bad)
    with pytest.raises(S.PhxError, match="PHX_ERR_NUMERIC"):
        s.Relaxation(2)
    s.step = 0
    s.set_q_cells(q0)
    s.Relaxation(1)
    assert rel_err(s.get(S.PHX_Q)[:, : m.n_cell], _oracle_step(m, params, q0)) <= 1e-12
