"""Restart files (phx_write_restart / phx_read_restart): the content of the
reference's restart (NSSolverUnstruct::DumpRestartH5 and
TurbSolverUnstr::DumpRestartH5: outnstep, q, q_turb, visturb) plus the
learned-source model.  A run that writes a restart and goes on, and a fresh
context that reads it and runs the same iterations, end in the same state bit
for bit.
"""
import numpy as np
import pytest

from phenlei_b200 import mesh as M
from phenlei_b200 import solver as S
from tests.test_partition import _case

pytestmark = pytest.mark.gpu


def _sa_solver(m, wd, precision, **kw):
    return S.NSSolverUnstruct(m, precision=precision, wall_dist=wd, **dict(_case("sa"), **kw))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_restart_continues_bit_for_bit(tmp_path, precision):
    m = M.channel_bump(16, 8, 2)
    wd = M.wall_distance(m)
    a = _sa_solver(m, wd, precision)
    a.Relaxation(6)
    path = str(tmp_path / "run.phxrst")
    a.DumpRestart(path)
    ha = a.Relaxation(5)
    b = _sa_solver(m, wd, precision)
    b.ReadRestart(path)
    assert b.step == 6
    hb = b.Relaxation(5)
    assert np.array_equal(a.get(S.PHX_Q), b.get(S.PHX_Q))
    assert np.array_equal(a.get(S.PHX_Q_TURB), b.get(S.PHX_Q_TURB))
    assert np.array_equal(a.get(S.PHX_VIST), b.get(S.PHX_VIST))
    # the residual monitor sums with atomics: equal up to the order of the sum
    assert np.max(np.abs(ha - hb) / np.abs(ha)) <= 1e-13


def test_restart_carries_the_learned_source(tmp_path):
    m = M.channel_bump(16, 8, 2)
    wd = M.wall_distance(m)
    t = _sa_solver(m, wd, "fp64")
    t.Relaxation(5)
    f, y, _, _ = t.capture_sa_samples()
    t.train_sa_mlp(f, y, epochs=2, batch=256, seed=1)
    blob = t.mlp_blob()
    a = _sa_solver(m, wd, "mixed", sa_source="mlp_fallback")
    a.set_mlp_blob(blob)
    a.Relaxation(4)
    path = str(tmp_path / "mlp.phxrst")
    a.DumpRestart(path)
    a.Relaxation(3)
    b = _sa_solver(m, wd, "mixed", sa_source="mlp_fallback")
    b.ReadRestart(path)   # the model comes with the file
    b.Relaxation(3)
    assert np.array_equal(b.mlp_blob(), blob)
    assert np.array_equal(a.get(S.PHX_Q), b.get(S.PHX_Q))
    assert np.array_equal(a.get(S.PHX_Q_TURB), b.get(S.PHX_Q_TURB))


def test_restart_of_another_grid_is_rejected(tmp_path):
    m = M.channel_bump(16, 8, 2)
    a = S.NSSolverUnstruct(m, **_case("laminar"))
    a.Relaxation(2)
    path = str(tmp_path / "lam.phxrst")
    a.DumpRestart(path)
    other = S.NSSolverUnstruct(M.channel_bump(16, 8, 4), **_case("laminar"))
    with pytest.raises(S.PhxError, match="PHX_ERR_ARG"):
        other.ReadRestart(path)
    with pytest.raises(S.PhxError, match="PHX_ERR_ARG"):
        other.ReadRestart(str(tmp_path / "missing.phxrst"))


def test_zones_restart_continues_bit_for_bit(tmp_path):
    """A partitioned run (three zones, SA) writes one restart file per zone,
    goes on, and a fresh zone set of the same partition reads them and runs
    the same iterations: the same state bit for bit."""
    from phenlei_b200 import cases
    from phenlei_b200.zones import ZoneSet

    m = M.channel_bump(16, 8, 2)
    wd = M.wall_distance(m)
    params = _case("sa")
    a = ZoneSet(m, params, 3, wall_dist=wd)
    a.set_state(cases.perturbed_state(m, params, seed=6))
    a.iterate(4)
    prefix = str(tmp_path / "zones.phxrst")
    a.DumpRestart(prefix)
    ha = a.iterate(3)
    b = ZoneSet(m, params, 3, wall_dist=wd)
    b.ReadRestart(prefix)
    assert {z.step for z in b.zones} == {4}
    hb = b.iterate(3)
    assert np.array_equal(a.gather(S.PHX_Q), b.gather(S.PHX_Q))
    assert np.array_equal(a.gather(S.PHX_Q_TURB), b.gather(S.PHX_Q_TURB))
    assert np.max(np.abs(ha - hb) / np.abs(ha)) <= 1e-13
    a.close()
    b.close()
