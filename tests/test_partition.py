"""Domain decomposition host logic (phenlei_b200.partition): cell partitions,
interface faces (boundary faces of type INTERFACE whose ghost is the
neighbouring part's cell, Geo_UnstructGrid.cpp:10806-10990), halo maps, and
the halo exchange over torch.distributed with world_size-2 gloo ranks.  CPU
only."""
import os
import socket

import numpy as np
import pytest

from oracle.oracle import Oracle
from phenlei_b200 import mesh as M
from phenlei_b200 import partition as P
from tests.conftest import rel_err

MESHES = {"bump": lambda: M.channel_bump(16, 8, 2), "tets": lambda: M.tet_cube(4, jitter=0.15, seed=3),
          "prism": lambda: M.channel_bump(16, 8, 2, prism_layers=3)}


def _field(nc_global):
    """A distinct value per global cell and variable: [5][nc]."""
    return np.arange(5)[:, None] * 1000.0 + np.arange(nc_global)[None, :] + 0.5


@pytest.mark.parametrize("kind", sorted(MESHES))
@pytest.mark.parametrize("nparts", [2, 3, 5])
def test_parts_cover_the_mesh_once(kind, nparts):
    m = MESHES[kind]()
    parts = P.split(m, P.slab_owner(m, nparts))
    assert len(parts) == nparts
    cells = np.concatenate([p.cells for p in parts])
    assert np.array_equal(np.sort(cells), np.arange(m.n_cell))
    count = np.zeros(m.n_face, int)
    for p in parts:
        np.add.at(count, p.faces, 1)
        # boundary faces first, the interface faces contiguous after the original ones
        assert p.mesh.n_bface == p.iface_first + p.n_iface
        assert np.all(p.mesh.right[: p.mesh.n_bface] == -1) and np.all(p.mesh.right[p.mesh.n_bface:] >= 0)
        rtype, _ = p.mesh.solver_regions()
        assert (P.BC_INTERFACE in rtype) == (p.n_iface > 0)
    cut = np.zeros(m.n_face, bool)
    for p in parts:
        cut[p.faces[p.iface_first:p.iface_first + p.n_iface]] = True
    # original boundary and uncut interior faces once; cut faces once in each of their two parts
    assert np.all(count[~cut] == 1) and np.all(count[cut] == 2)


@pytest.mark.parametrize("kind", sorted(MESHES))
def test_part_geometry_matches_the_global_mesh(kind):
    """Cell volumes and centres, and face areas and centres, as the oracle's
    metrics (UnstructGrid::ComputeMetrics) form them: the same in the part as
    in the whole mesh; a flipped interface face has the opposite normal."""
    m = MESHES[kind]()
    g = Oracle(m, {"refMachNumber": 0.5}).geo
    for p in P.split(m, P.slab_owner(m, 3)):
        lg = Oracle(p.mesh, {"refMachNumber": 0.5}).geo
        nc = p.mesh.n_cell
        for k in ("vol", "xcc", "ycc", "zcc"):
            assert rel_err(lg[k][:nc], g[k][p.cells]) <= 1e-14, k
        for k in ("area", "xfc", "yfc", "zfc"):
            assert rel_err(lg[k], g[k][p.faces]) <= 1e-14, k
        sgn = np.where(p.flipped, -1.0, 1.0)
        for k in ("xfn", "yfn", "zfn"):
            assert rel_err(lg[k], sgn * g[k][p.faces]) <= 1e-14, k


def _simulated_exchange(parts, values):
    """Fill every part's interface ghosts from the halo maps alone (no
    communication): what `exchange` moves between ranks."""
    for p, part in enumerate(parts):
        for q in part.halo.neighbors:
            src = parts[q].halo.send[p]
            values[p][:, part.halo.recv[q]] = values[q][:, src]


@pytest.mark.parametrize("kind", sorted(MESHES))
@pytest.mark.parametrize("nparts", [2, 4])
def test_halo_maps_fill_ghosts_with_the_neighbour_cells(kind, nparts):
    m = MESHES[kind]()
    f = _field(m.n_cell)
    parts = P.split(m, P.slab_owner(m, nparts))
    vals = []
    for p in parts:
        v = np.full((5, p.mesh.n_cell + p.mesh.n_bface), np.nan)
        v[:, : p.mesh.n_cell] = f[:, p.cells]
        vals.append(v)
    _simulated_exchange(parts, vals)
    left, right = np.asarray(m.left), np.asarray(m.right)
    for p, part in enumerate(parts):
        sl = slice(part.iface_first, part.iface_first + part.n_iface)
        gf = part.faces[sl]
        nbr = np.where(part.flipped[sl], left[gf], right[gf])
        ghosts = vals[p][:, part.mesh.n_cell + part.iface_first + np.arange(part.n_iface)]
        assert np.array_equal(ghosts, f[:, nbr])
        # the part's own side of each interface face is its owner (left) cell
        own = np.where(part.flipped[sl], right[gf], left[gf])
        assert np.array_equal(part.cells[part.mesh.left[sl]], own)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, kind, out):
    import torch
    import torch.distributed as dist
    import datetime

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        m = MESHES[kind]()
        part = P.split(m, P.slab_owner(m, world))[rank]
        f = _field(m.n_cell)
        nt = part.mesh.n_cell + part.mesh.n_bface
        field = torch.full((5, nt), float("nan"), dtype=torch.float64)
        field[:, : part.mesh.n_cell] = torch.from_numpy(f[:, part.cells])
        P.exchange(part.halo, field)
        sl = slice(part.iface_first, part.iface_first + part.n_iface)
        gf = part.faces[sl]
        nbr = np.where(part.flipped[sl], np.asarray(m.left)[gf], np.asarray(m.right)[gf])
        got = field[:, part.mesh.n_cell + part.iface_first + np.arange(part.n_iface)].numpy()
        ok = bool(np.array_equal(got, f[:, nbr])) and part.n_iface > 0
        np.save(os.path.join(out, f"rank{rank}.npy"), np.array([ok]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind", ["bump", "tets"])
def test_gloo_exchange_world_size_2(tmp_path, kind):
    import torch.multiprocessing as mp

    mp.spawn(_rank_main, args=(2, _free_port(), kind, str(tmp_path)), nprocs=2, join=True)
    assert all(np.load(tmp_path / f"rank{r}.npy")[0] for r in range(2))


# --- the oracle on a partitioned grid (oracle/partitioned.py) --------------------------------------

def _global_and_parts(params, nparts, kind="bump", seed=3):
    from phenlei_b200 import cases
    from oracle.partitioned import PartitionedOracle

    m = MESHES[kind]()
    q0 = cases.perturbed_state(m, params, seed=seed)
    sa = params.get("viscousType", 0) == 3
    wd = M.wall_distance(m) if sa else None
    qt0 = None
    if sa:   # nu~ around its free-stream value, some cells negative
        rng = np.random.default_rng(seed)
        qt0 = params.get("muoo", 3.0) * (1.0 + 1.5 * rng.standard_normal(m.n_cell))
    o = Oracle(m, params, wall_dist=wd)
    o.set_state(q0, qt0)
    po = PartitionedOracle(m, params, nparts, wall_dist=wd)
    po.set_state(q0, qt0)
    return m, o, po


def _case(name):
    from phenlei_b200 import cases

    return {"euler": cases.EULER_BUMP, "euler_lsq": dict(cases.EULER_BUMP, gradientName="lsq"),
            "laminar": cases.LAMINAR, "laminar_lsq": dict(cases.LAMINAR, gradientName="lsq"),
            "euler_barth": dict(cases.EULER_BUMP, uns_limiter_name="barth"),
            "euler_ktmax": dict(cases.EULER_BUMP, ktmax=1.5),
            "sa": dict(cases.SA_BUMP, refReNumber=1.0e5), "sa_lsq": dict(cases.SA_BUMP, refReNumber=1.0e5,
                                                                          gradientName="lsq")}[name]


@pytest.mark.parametrize("case", ["laminar", "sa"])
def test_one_part_is_the_whole_mesh(case):
    m, o, po = _global_and_parts(_case(case), 1)
    h0, h1 = o.iterate(3), po.iterate(3)
    assert np.array_equal(h0, h1)
    assert np.array_equal(po.gather("q"), o.q[:, : m.n_cell])
    if case == "sa":
        assert np.array_equal(po.gather("qt"), o.work("qt")[: m.n_cell])


@pytest.mark.parametrize("case", ["euler", "euler_lsq", "laminar", "laminar_lsq", "euler_barth", "euler_ktmax", "sa",
                                  "sa_lsq"])
@pytest.mark.parametrize("nparts", [2, 3])
def test_partitioned_explicit_operator_equals_the_whole_mesh(case, nparts):
    """With the interface ghosts filled as the reference fills them, every
    explicit quantity of an iteration (gradients, limiter, residual, spectral
    radius, time step) is the whole mesh's, to rounding: only the LU-SGS
    sweep (block-Jacobi across parts) differs."""
    m, o, po = _global_and_parts(_case(case), nparts)
    o.iterate(1)
    po.iterate(1)
    nc = m.n_cell
    # the three gradient components together: on the quasi-2-D bump d/dz is round-off
    grad = ("dqdx", "dqdy", "dqdz")
    assert rel_err(np.stack([po.gather(k) for k in grad]), np.stack([o.work(k)[:, :nc] for k in grad])) <= 1e-12
    for k in ("limit", "res", "inv_spec", "dt"):
        assert rel_err(po.gather(k), o.work(k)[..., :nc]) <= 1e-12, k
    if _case(case).get("viscousType", 0):
        for k in ("dtdx", "dtdy", "vis_spec"):
            assert rel_err(po.gather(k), o.work(k)[..., :nc]) <= 1e-12, k


def test_block_jacobi_sweep_stays_close_to_the_whole_mesh():
    """The partitioned LU-SGS couples the parts only through the forward dq
    of the interface ghosts, so dq differs from the whole mesh's near the cut,
    and the residual history follows the whole mesh's."""
    m, o, po = _global_and_parts(_case("euler"), 2)
    h0, h1 = o.iterate(10), po.iterate(10)
    assert np.all(np.abs(h1 / h0 - 1.0) < 0.05)
    assert not np.array_equal(po.gather("dq"), o.work("dq")[:, : m.n_cell])


@pytest.mark.parametrize("case", ["laminar", "sa"])
def test_partitioned_history_follows_the_whole_mesh(case):
    m, o, po = _global_and_parts(_case(case), 3)
    h0, h1 = o.iterate(10), po.iterate(10)
    assert np.all(np.abs(h1 / h0 - 1.0) < 0.05)
    if case == "sa":
        assert rel_err(po.gather("qt"), o.work("qt")[: m.n_cell]) < 0.05


def _oracle_rank_main(rank, world, port, case, out):
    import datetime

    import torch.distributed as dist

    from oracle.partitioned import DistributedOracle
    from phenlei_b200 import cases

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        params = _case(case)
        m = MESHES["bump"]()
        q0 = cases.perturbed_state(m, params, seed=3)
        sa = params.get("viscousType", 0) == 3
        wd = M.wall_distance(m) if sa else None
        qt0 = params.get("muoo", 3.0) * (1.0 + 1.5 * np.random.default_rng(3).standard_normal(m.n_cell)) if sa else None
        do = DistributedOracle(m, params, rank, world, wall_dist=wd)
        do.set_state(q0, qt0)
        hist = do.iterate(3)
        np.savez(os.path.join(out, f"rank{rank}.npz"), hist=hist, cells=do.local_cells(), q=do.gather("q"),
                 qt=do.gather("qt") if sa else np.zeros(1))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case", ["laminar", "sa"])
def test_distributed_oracle_world_size_2_equals_in_process(tmp_path, case):
    """The partitioned oracle as two gloo ranks, each with its own part, halos
    moved by partition.exchange and sums by all_reduce: the same residual
    history and state as the in-process partitioned run, bit for bit."""
    import torch.multiprocessing as mp

    mp.spawn(_oracle_rank_main, args=(2, _free_port(), case, str(tmp_path)), nprocs=2, join=True)
    m, _, po = _global_and_parts(_case(case), 2)
    h = po.iterate(3)
    q = po.gather("q")
    for r in range(2):
        d = np.load(tmp_path / f"rank{r}.npz")
        assert np.array_equal(d["hist"], h)
        cells = d["cells"]
        assert np.array_equal(d["q"][:, cells], q[:, cells])
        if case == "sa":
            assert np.array_equal(d["qt"][cells], po.gather("qt")[cells])


# --- zones built alone (phenlei_b200.zones.channel_zone) ------------------------------------------

@pytest.mark.parametrize("prism", [0, 3])
@pytest.mark.parametrize("world", [2, 3])
def test_channel_zones_built_alone_equal_the_split_channel(prism, world):
    """Zone r of a channel built alone holds the cells that slab_owner + split
    give part r of the whole channel, and each interface ghost's halo source is
    the neighbouring zone's cell across that face (the face's nodes are the
    cell's nodes)."""
    from phenlei_b200.zones import channel_zone

    kw = dict(nx=12 * world, ny=6, nz=2, length=1.5 * world, dz=0.125, prism_layers=prism)
    whole = M.channel_bump(**kw)
    parts = P.split(whole, P.slab_owner(whole, world))
    zones = [channel_zone(r, world, **kw) for r in range(world)]
    for r, (z, p) in enumerate(zip(zones, parts)):
        a = P.cell_centroids(z.mesh)
        b = P.cell_centroids(p.mesh)
        assert a.shape == b.shape
        assert np.allclose(a[np.lexsort(a.T)], b[np.lexsort(b.T)], rtol=0, atol=1e-12)
        assert z.n_iface == p.n_iface and z.halo.neighbors == p.halo.neighbors
        assert z.mesh.solver_regions()[0].tolist().count(P.BC_INTERFACE) == (1 if world > 1 else 0)
    xyz = [np.stack([z.mesh.x, z.mesh.y, z.mesh.z], 1) for z in zones]
    for r, z in enumerate(zones):
        m = z.mesh
        foff = m.face_offsets()
        for q in z.halo.neighbors:
            nq = zones[q].mesh
            coff = np.zeros(nq.n_cell + 1, np.int64)
            np.cumsum(nq.cell_nnode, out=coff[1:])
            src = zones[q].halo.send[r]
            assert len(src) == len(z.halo.recv[q])
            for ghost, c in zip(z.halo.recv[q], src):
                f = int(ghost) - m.n_cell
                fpts = xyz[r][np.asarray(m.face2node)[foff[f]:foff[f + 1]]]
                cpts = xyz[q][np.asarray(nq.cell2node)[coff[c]:coff[c + 1]]]
                d = np.min(np.abs(fpts[:, None, :] - cpts[None, :, :]).sum(-1), axis=1)
                assert np.all(d < 1e-12)


def test_a_zone_one_cell_thick_sends_each_cell_across_both_cuts():
    """A slab one cell thick between two zones: each of its cells is sent
    across both cuts (twice as many send rows as cells), and the partitioned
    oracle steps it."""
    from oracle.partitioned import PartitionedOracle
    from phenlei_b200 import cases

    m = MESHES["bump"]()
    cx = P.cell_centroids(m)[:, 0]
    order = np.lexsort((np.arange(m.n_cell), cx))
    column = np.empty(m.n_cell, np.int64)
    column[order] = np.arange(m.n_cell) * 16 // m.n_cell
    owner = np.where(column < 7, 0, np.where(column == 7, 1, 2)).astype(np.int32)
    parts = P.split(m, owner)
    assert [p.halo.neighbors for p in parts] == [[1], [0, 2], [1]]
    assert parts[1].halo.n_send() == 2 * parts[1].mesh.n_cell == parts[1].n_iface
    params = _case("laminar")
    po = PartitionedOracle(m, params, 3, owner=owner)
    po.set_state(cases.perturbed_state(m, params, seed=3))
    assert np.isfinite(po.iterate(2)).all()


@pytest.mark.parametrize("nparts", [1, 2, 3, 7, 8, 16])
def test_recursive_bisection_balances_parts_and_cuts_fewer_faces(nparts):
    """rcb_owner: every part non-empty, sizes within one cell per level of
    cuts, a valid split; from 7 parts on the jittered-tet cube it cuts fewer
    faces than slabs."""
    m = MESHES["tets"]() if nparts < 7 else M.tet_cube(12, jitter=0.15, seed=1)
    owner = P.rcb_owner(m, nparts)
    cnt = np.bincount(owner, minlength=nparts)
    assert cnt.size == nparts and cnt.min() > 0
    assert cnt.max() - cnt.min() <= int(np.ceil(np.log2(nparts))) if nparts > 1 else cnt[0] == m.n_cell
    assert np.array_equal(P.rcb_owner(m, nparts), owner)     # deterministic
    parts = P.split(m, owner)
    assert sum(p.mesh.n_cell for p in parts) == m.n_cell
    if nparts >= 7:
        cut = lambda o: sum(p.n_iface for p in P.split(m, o)) // 2  # noqa: E731
        assert cut(owner) < cut(P.slab_owner(m, nparts)) / 2


def test_recursive_bisection_parts_step_in_the_partitioned_oracle():
    from oracle.partitioned import PartitionedOracle
    from phenlei_b200 import cases

    m = MESHES["bump"]()
    params = _case("laminar")
    po = PartitionedOracle(m, params, 4, owner=P.rcb_owner(m, 4))
    po.set_state(cases.perturbed_state(m, params, seed=3))
    assert np.isfinite(po.iterate(2)).all()
