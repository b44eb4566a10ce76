"""The CUDA solver on a partitioned grid (phenlei_b200.zones): one context per
zone on one GPU, joined by interface faces (PHENGLEI::INTERFACE), stepped
phase by phase with the halo rows moved between the zones by the host, against
the reference's own runs on the same zones (golden fixtures) and the oracle's
partitioned run (oracle/partitioned.py, itself pinned to those fixtures) on
seeded inputs, meshes and partitions.  No kernel waits on another zone.

Tolerances (norm-wise, max|a-b|/max|ref|): FP64 1e-12 per array after one
iteration and 1e-10 over ten-iteration histories; mixed precision 1e-5 after
one iteration.
"""
import os

import numpy as np
import pytest

from phenlei_b200 import mesh as M
from phenlei_b200 import solver as S
from tests.conftest import rel_err
from tests.test_partition import MESHES, _case, _free_port

pytestmark = pytest.mark.gpu


def _inputs(params, kind="bump", seed=3):
    from phenlei_b200 import cases

    m = MESHES[kind]()
    q0 = cases.perturbed_state(m, params, seed=seed)
    sa = params.get("viscousType", 0) == 3
    wd = M.wall_distance(m) if sa else None
    qt0 = None
    if sa:   # nu~ around its free-stream value, some cells negative
        rng = np.random.default_rng(seed)
        qt0 = params.get("muoo", 3.0) * (1.0 + 1.5 * rng.standard_normal(m.n_cell))
    return m, q0, qt0, wd


def _pair(case, nparts, precision="fp64", kind="bump"):
    from oracle.partitioned import PartitionedOracle
    from phenlei_b200.zones import ZoneSet

    params = _case(case)
    m, q0, qt0, wd = _inputs(params, kind)
    po = PartitionedOracle(m, params, nparts, wall_dist=wd)
    po.set_state(q0, qt0)
    zs = ZoneSet(m, params, nparts, owner=po.owner, wall_dist=wd, precision=precision)
    zs.set_state(q0, qt0)
    return m, po, zs


ALL = ["euler", "euler_lsq", "laminar", "laminar_lsq", "euler_barth", "euler_ktmax", "sa", "sa_lsq"]


@pytest.mark.parametrize("case", ALL)
@pytest.mark.parametrize("nparts", [2, 3])
def test_fp64_zones_match_the_partitioned_oracle(case, nparts):
    """One iteration: every explicit quantity and the block-Jacobi sweep's
    result of every zone equal the oracle's zones."""
    m, po, zs = _pair(case, nparts)
    h_o = po.iterate(1)
    h_z = zs.iterate(1)
    nc = m.n_cell
    assert rel_err(h_z, h_o) <= 1e-12
    assert rel_err(zs.gather(S.PHX_Q), po.gather("q")) <= 1e-12
    assert rel_err(zs.gather(S.PHX_RES), po.gather("res")) <= 1e-12
    assert rel_err(zs.gather(S.PHX_LIMIT), po.gather("limit")) <= 1e-12
    assert rel_err(zs.gather(S.PHX_DT), po.gather("dt")) <= 1e-12
    grad = np.stack([zs.gather(k) for k in (S.PHX_GRADX, S.PHX_GRADY, S.PHX_GRADZ)])
    assert rel_err(grad, np.stack([po.gather(k) for k in ("dqdx", "dqdy", "dqdz")])) <= 1e-12
    assert rel_err(zs.gather(S.PHX_DQ), po.gather("dq")) <= 1e-12
    if _case(case).get("viscousType", 0) == 3:
        assert rel_err(zs.gather(S.PHX_Q_TURB), po.gather("qt")) <= 1e-12
        assert rel_err(zs.gather(S.PHX_VIST), po.gather("vist")) <= 1e-12
    assert nc == zs.n_cell_total


@pytest.mark.parametrize("case", ["laminar", "sa"])
def test_fp64_zone_histories_match_the_partitioned_oracle(case):
    m, po, zs = _pair(case, 3)
    h_o = po.iterate(10)
    h_z = zs.iterate(10)
    assert rel_err(h_z, h_o) <= 1e-10
    assert rel_err(zs.gather(S.PHX_Q), po.gather("q")) <= 1e-10
    if case == "sa":
        assert rel_err(zs.gather(S.PHX_Q_TURB), po.gather("qt")) <= 1e-10
    sums_o = po_forces(po)
    assert rel_err(zs.forces(), sums_o) <= 1e-10


def po_forces(po):
    """The wall force sums of the oracle's zones, added."""
    import ctypes as C

    from oracle.oracle import _p, lib

    tot = np.zeros(16)
    for o in po.o:
        out = np.zeros(16)
        lib().ox_forces(C.byref(o.g), C.byref(o.m), C.byref(o.p), _p(o.q), C.byref(o.w), _p(out))
        tot += out
    return tot


@pytest.mark.parametrize("case", ["euler", "laminar_lsq", "sa"])
def test_mixed_zones_match_the_partitioned_oracle(case):
    m, po, zs = _pair(case, 2, precision="mixed")
    h_o = po.iterate(1)
    h_z = zs.iterate(1)
    assert rel_err(h_z, h_o) <= 1e-5
    assert rel_err(zs.gather(S.PHX_Q), po.gather("q")) <= 1e-5
    if case == "sa":
        assert rel_err(zs.gather(S.PHX_Q_TURB), po.gather("qt")) <= 1e-5


def test_tetrahedral_zones_match_the_partitioned_oracle():
    from oracle.partitioned import PartitionedOracle
    from phenlei_b200 import cases
    from phenlei_b200.zones import ZoneSet

    params = dict(cases.LAMINAR, gradientName="lsq")
    m = MESHES["tets"]()
    q0 = cases.perturbed_state(m, params, seed=5)
    po = PartitionedOracle(m, params, 3)
    po.set_state(q0)
    zs = ZoneSet(m, params, 3, owner=po.owner)
    zs.set_state(q0)
    assert rel_err(zs.iterate(3), po.iterate(3)) <= 1e-11
    assert rel_err(zs.gather(S.PHX_Q), po.gather("q")) <= 1e-11


def test_one_zone_is_the_plain_solver():
    """A single zone (no interface faces) runs the same kernels as the fused
    driver: the same state bit for bit."""
    from phenlei_b200.zones import ZoneSet

    params = _case("sa")
    m, q0, qt0, wd = _inputs(params)
    zs = ZoneSet(m, params, 1, wall_dist=wd)
    zs.set_state(q0, qt0)
    s = S.NSSolverUnstruct(m, wall_dist=wd, **params)
    s.set_q_cells(q0)
    s.set_qt_cells(qt0)
    h1 = s.Relaxation(4)
    h2 = zs.iterate(4)
    assert rel_err(h2, h1) <= 1e-14
    assert np.array_equal(zs.gather(S.PHX_Q), s.get(S.PHX_Q)[:, : m.n_cell])
    assert np.array_equal(zs.gather(S.PHX_Q_TURB), s.get(S.PHX_Q_TURB)[: m.n_cell])


def test_fused_calls_refuse_a_zone():
    """A context with interface faces runs only phase by phase with the
    exchanges: the fused driver and the fused sweeps return PHX_ERR_STATE."""
    from phenlei_b200.zones import ZoneSet

    params = _case("laminar")
    m, q0, _, _ = _inputs(params)
    zs = ZoneSet(m, params, 2)
    z = zs.zones[0]
    with pytest.raises(S.PhxError, match="PHX_ERR_STATE"):
        z.Relaxation(1)
    z.step = z.step + 1
    z.Boundary()
    z.ComputeGradientAndLimiter()
    z.UpdateResiduals()
    with pytest.raises(S.PhxError, match="PHX_ERR_STATE"):
        z.LUSGS()
    with pytest.raises(S.PhxError, match="PHX_ERR_STATE"):
        zs.zones[1].LUSGSBackward()   # no forward sweep yet


def _zone_rank_main(rank, world, port, case, out):
    import datetime

    import torch
    import torch.distributed as dist

    from phenlei_b200.zones import DistributedZone

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        params = _case(case)
        m, q0, qt0, wd = _inputs(params)
        dz = DistributedZone(m, params, wall_dist=wd)
        dz.set_state(q0, qt0)
        hist = dz.iterate(3)
        z = dz.zones[0]
        nc = z.mesh.n_cell
        np.savez(os.path.join(out, f"rank{rank}.npz"), hist=hist, cells=dz.local_cells(),
                 q=z.get(S.PHX_Q)[:, :nc], forces=dz.forces())
        dz.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case", ["laminar", "sa"])
def test_distributed_zones_world_size_2_equal_the_zone_set(tmp_path, case):
    """Two processes, one zone each, halo rows through torch.distributed
    (gloo, staged through host memory) and the sums by all_reduce: the same
    history and state as the in-process zone set, bit for bit.  Both processes
    use the one GPU; neither waits on the other's kernels."""
    import torch.multiprocessing as mp

    from phenlei_b200.zones import ZoneSet

    mp.spawn(_zone_rank_main, args=(2, _free_port(), case, str(tmp_path)), nprocs=2, join=True)
    params = _case(case)
    m, q0, qt0, wd = _inputs(params)
    zs = ZoneSet(m, params, 2, wall_dist=wd)
    zs.set_state(q0, qt0)
    h = zs.iterate(3)
    f = zs.forces()
    for r in range(2):
        d = np.load(tmp_path / f"rank{r}.npz")
        assert np.array_equal(d["hist"], h)
        assert np.array_equal(d["q"], zs.zones[r].get(S.PHX_Q)[:, : zs.zones[r].mesh.n_cell])
        assert rel_err(d["forces"], f) <= 1e-14


@pytest.mark.parametrize("name", ["zones2_euler_bump_16x8x2_step10", "zones3_laminar_bump_16x8x2_lsq_step10",
                                  "zones2_euler_bump_16x8x2_barth_ktmax_step10", "zones2_sa_bump_16x8x2_step10",
                                  "zones3_sa_bump_16x8x2_prism_step5"])
def test_fp64_zones_match_reference_golden(golden, name):
    """The CUDA zones against the reference's own run on the same zones
    (tests/golden/make_golden.py, zone_fixture): residual history, state,
    residual, time step, limiter, gradient and wall forces after 5-10
    iterations."""
    from phenlei_b200.zones import ZoneSet

    d = golden(name)
    m = d["mesh_obj"]
    params = d["params_dict"]
    sa = params.get("viscousType", 0) == 3
    zs = ZoneSet(m, params, int(d["nparts"]), owner=d["owner"], wall_dist=d["walldist"] if sa else None)
    st = d["state_in"]
    zs.set_state(st[:5], st[5] if sa else None)
    hist = zs.iterate(int(d["nsteps"]))
    assert rel_err(hist, d["res_hist"]) <= 1e-10
    assert rel_err(zs.gather(S.PHX_Q), d["q"]) <= 1e-10
    assert rel_err(zs.gather(S.PHX_RES), d["res"]) <= 1e-10
    assert rel_err(zs.gather(S.PHX_DT), d["dt"]) <= 1e-10
    assert rel_err(zs.gather(S.PHX_LIMIT), d["limit"]) <= 1e-10
    assert rel_err(zs.gather(S.PHX_GRADX), d["gradPrimtiveVarX"]) <= 1e-10
    assert rel_err(zs.forces(), d["forces"]) <= 1e-10
    if sa:
        assert rel_err(zs.gather(S.PHX_Q_TURB), d["q_turb"]) <= 1e-10
        assert rel_err(zs.gather(S.PHX_VIST), d["vist"]) <= 1e-10


@pytest.mark.parametrize("name", ["zones2_euler_bump_16x8x2_step10", "zones2_sa_bump_16x8x2_step10"])
def test_mixed_zones_follow_reference_golden(golden, name):
    """The mixed-precision zones against the reference's own multi-zone run:
    the residual history and the state over 10 iterations within 1e-4."""
    from phenlei_b200.zones import ZoneSet

    d = golden(name)
    m = d["mesh_obj"]
    params = d["params_dict"]
    sa = params.get("viscousType", 0) == 3
    zs = ZoneSet(m, params, int(d["nparts"]), owner=d["owner"], wall_dist=d["walldist"] if sa else None,
                 precision="mixed")
    st = d["state_in"]
    zs.set_state(st[:5], st[5] if sa else None)
    hist = zs.iterate(int(d["nsteps"]))
    assert rel_err(hist, d["res_hist"]) <= 1e-4
    assert rel_err(zs.gather(S.PHX_Q), d["q"]) <= 1e-4
    if sa:
        assert rel_err(zs.gather(S.PHX_Q_TURB), d["q_turb"]) <= 1e-4


@pytest.mark.parametrize("case", ["laminar", "sa"])
def test_zones_built_from_interface_lists_equal_the_split(case):
    """Zones as a grid file gives them (meshes and interface lists, read by
    phenlei_b200.fts.zone_parts) step bit for bit as the same split built
    from the whole mesh."""
    from oracle import refrun
    from phenlei_b200 import fts
    from phenlei_b200 import partition as P
    from phenlei_b200.zones import ZoneSet

    params = _case(case)
    m, q0, qt0, wd = _inputs(params)
    owner = P.slab_owner(m, 3)
    split = P.split(m, owner)
    zones = [fts.FtsZone(index=p.rank, proc=p.rank, mesh=p.mesh, ndim=3, interface=itf)
             for p, itf in zip(split, refrun.interface_arrays(split))]
    gnum = np.concatenate([p.cells for p in split])
    a = ZoneSet(m, params, 3, owner=owner, wall_dist=wd)
    a.set_state(q0, qt0)
    ha = a.iterate(4)
    b = ZoneSet(None, params, parts=fts.zone_parts(zones), wall_dist=None if wd is None else wd[gnum])
    b.set_state(q0[:, gnum], None if qt0 is None else qt0[gnum])
    hb = b.iterate(4)
    assert np.array_equal(a.gather(S.PHX_Q)[:, gnum], b.gather(S.PHX_Q))
    if qt0 is not None:
        assert np.array_equal(a.gather(S.PHX_Q_TURB)[gnum], b.gather(S.PHX_Q_TURB))
    # the residual monitor sums with FP64 atomics: equal up to the order of the sums
    assert rel_err(hb, ha) <= 1e-13
    a.close()
    b.close()


def test_a_zone_one_cell_thick_sends_more_rows_than_it_has_cells():
    """A slab zone one cell thick between two others sends each cell across
    both cuts, so its halo lists more send rows than cells; it runs as the
    partitioned oracle runs (FP64 1e-12 after one iteration)."""
    from oracle.partitioned import PartitionedOracle
    from phenlei_b200 import partition as P
    from phenlei_b200.zones import ZoneSet

    params = _case("laminar")
    m, q0, _, _ = _inputs(params)
    cx = P.cell_centroids(m)[:, 0]
    order = np.lexsort((np.arange(m.n_cell), cx))
    column = np.empty(m.n_cell, np.int64)
    column[order] = np.arange(m.n_cell) * 16 // m.n_cell     # 16 columns of cells along x
    owner = np.where(column < 7, 0, np.where(column == 7, 1, 2)).astype(np.int32)
    po = PartitionedOracle(m, params, 3, owner=owner)
    po.set_state(q0)
    zs = ZoneSet(m, params, 3, owner=owner)
    zs.set_state(q0)
    thin = zs.parts[1]
    assert thin.halo.n_send() == 2 * thin.mesh.n_cell
    h_o, h_z = po.iterate(1), zs.iterate(1)
    assert rel_err(h_z, h_o) <= 1e-12
    assert rel_err(zs.gather(S.PHX_Q), po.gather("q")) <= 1e-12
    assert rel_err(zs.gather(S.PHX_DQ), po.gather("dq")) <= 1e-12
    zs.close()
