"""The .fts grid reader (phenlei_b200.fts over phenlei_b200.h5lite), on the CPU.

Pinned on the reference's own example grid, rae2822_hybrid2d__4.fts (the
RAE 2822 aerofoil, hybrid triangles and quadrilaterals, four zones: the grid
of the reference's cfd_para_transonic.hypara), against the Fluent case
rae2822_hybrid2d.cas it was converted from, parsed independently
(tests/fluent_cas.py): the zones hold exactly the case's nodes, faces and
cells, each face with its two cells on the same sides and each boundary face
with the matching boundary condition.  The interface lists of the zones
point back at each other and join faces with the same nodes, and the halo
plans made from them give the file's lists back.

The example grid is two-dimensional, which the solver path does not take;
`zone_parts` is checked on three-dimensional zones by rebuilding the parts of
a split channel from their interface lists alone: the partitioned oracle then
steps bit for bit as on the split itself.
"""
import numpy as np
import pytest

from oracle import refrun
from oracle.partitioned import PartitionedOracle
from phenlei_b200 import cases, fts
from phenlei_b200 import mesh as M
from phenlei_b200 import partition as P
from phenlei_b200.h5lite import H5Error, H5File
from tests.conftest import reference_file
from tests.fluent_cas import FLUENT_PRESSURE_FAR_FIELD, FLUENT_WALL, read_cas

EXAMPLE = "PHengLEI/examples/grid/rae2822_hybrid2d__4_0.fts"
CASE = "PHengLEI/examples/grid/rae2822_hybrid2d.cas"

needs_example = pytest.mark.skipif(reference_file(EXAMPLE) is None or reference_file(CASE) is None,
                                   reason="the reference project's example grid is not on this machine")


@pytest.fixture(scope="module")
def grid():
    path = reference_file(EXAMPLE)
    # the grid is named without the file number, as the parameter file names it
    return fts.read_fts(path.replace("__4_0.fts", "__4.fts"))


@pytest.fixture(scope="module")
def case():
    return read_cas(reference_file(CASE))


@needs_example
def test_reads_every_zone_of_the_example_grid(grid):
    assert grid.version == 2.0
    assert len(grid.files) == 1 and grid.files[0].endswith("__4_0.fts")
    assert [z.index for z in grid.zones] == [0, 1, 2, 3]
    assert [z.proc for z in grid.zones] == [0, 1, 2, 3]
    assert [z.mesh.n_cell for z in grid.zones] == [9009, 9010, 9008, 9009]
    for z in grid.zones:
        m = z.mesh
        assert z.ndim == 2
        assert m.n_node == np.unique(m.face2node).size
        assert m.left.min() >= 0 and m.right[m.n_bface:].min() >= 0 and (m.right[: m.n_bface] == -1).all()
        kinds = {t for t, _ in m.regions}
        assert M.BC_INTERFACE in kinds and len(z.interface[0]) == int(
            (np.array([m.regions[r][0] for r in m.bface_region]) == M.BC_INTERFACE).sum())


@needs_example
def test_zones_hold_the_fluent_case_they_were_converted_from(grid, case):
    xyz = case["xyz"]
    node_of = {(float(a), float(b)): i for i, (a, b) in enumerate(xyz)}
    assert len(node_of) == xyz.shape[0]
    cas_face = {}
    cell_nodes = [set() for _ in range(case["n_cell"])]
    for zone, bc, nodes, c0, c1 in case["faces"]:
        cas_face[frozenset(nodes)] = (zone, bc, nodes, c0, c1)
        for c in (c0, c1):
            if c >= 0:
                cell_nodes[c].update(nodes)
    cell_of = {frozenset(s): c for c, s in enumerate(cell_nodes)}
    assert len(cell_of) == case["n_cell"]

    seen_cells = np.zeros(case["n_cell"], np.int64)
    face_uses = {}
    bc_of = {4: FLUENT_PRESSURE_FAR_FIELD, 2: FLUENT_WALL}
    for z in grid.zones:
        m = z.mesh
        gnode = np.array([node_of[(float(a), float(b))] for a, b in zip(m.x, m.y)])
        assert (m.z == 0.0).all()
        coff = m.cell_offsets()
        gcell = np.array([cell_of[frozenset(gnode[m.cell2node[coff[c]:coff[c + 1]]].tolist())]
                          for c in range(m.n_cell)])
        seen_cells[gcell] += 1
        foff = m.face_offsets()
        for f in range(m.n_face):
            nodes = tuple(gnode[m.face2node[foff[f]:foff[f + 1]]].tolist())
            zone, bc, cnodes, c0, c1 = cas_face[frozenset(nodes)]
            face_uses[frozenset(nodes)] = face_uses.get(frozenset(nodes), 0) + 1
            left = gcell[m.left[f]]
            if f < m.n_bface:
                t, name = m.regions[m.bface_region[f]]
                if t == M.BC_INTERFACE:
                    assert bc == 2 and left in (c0, c1)        # an interior face of the case, cut
                    continue
                # the boundary type, and the region name of the case's face zone
                assert bc == bc_of[t] and name == case["zone_names"][zone][0]
                right = -1
            else:
                right = gcell[m.right[f]]
            # the same face with the same cells on the same sides: the node
            # order of the case with its c0 on the left, or reversed with c1
            assert (nodes == cnodes and (left, right) == (c0, c1)) or \
                   (nodes == cnodes[::-1] and (left, right) == (c1, c0))
    assert (seen_cells == 1).all()
    assert len(face_uses) == len(case["faces"])
    # interior faces cut by the partition appear in two zones, all others in one
    n_itf = sum(len(z.interface[0]) for z in grid.zones)
    assert sum(face_uses.values()) == len(case["faces"]) + n_itf // 2


@needs_example
def test_interface_lists_point_back_and_join_the_same_faces(grid):
    zones = grid.zones
    for i, z in enumerate(zones):
        zid, iid, bf = z.interface
        m = z.mesh
        foff = m.face_offsets()
        for k in range(len(zid)):
            o = zones[zid[k]]
            j = iid[k]
            assert o.interface[0][j] == i and o.interface[1][j] == k
            f, g = bf[k], o.interface[2][j]
            a = {(float(m.x[n]), float(m.y[n])) for n in m.face2node[foff[f]:foff[f + 1]]}
            ofo = o.mesh.face_offsets()
            b = {(float(o.mesh.x[n]), float(o.mesh.y[n])) for n in o.mesh.face2node[ofo[g]:ofo[g + 1]]}
            assert a == b


@needs_example
def test_halo_plans_give_the_file_interface_lists_back(grid):
    parts = fts.zone_parts(grid.zones)
    for z, p, (zid, iid, bf) in zip(grid.zones, parts, refrun.interface_arrays(parts)):
        assert np.array_equal(zid, z.interface[0])
        assert np.array_equal(iid, z.interface[1])
        assert np.array_equal(bf, z.interface[2])
        assert p.halo.neighbors == sorted(set(z.interface[0].tolist()))
    assert parts[2].halo.send[3].size == parts[3].halo.recv[2].size == 127


@needs_example
def test_stored_wall_distances(grid):
    """The example's .wdt file: one distance per cell of every zone.  In the
    two zones away from the aerofoil (triangles only) every value is the
    distance from the cell's node mean to the nearest wall segment, to
    rounding; near the wall (zones 2 and 3, with quadrilaterals) the
    reference's search takes other centres, so those are held to 25 %."""
    wd = fts.read_wall_distance(grid)
    assert [d.size for d in wd] == [z.mesh.n_cell for z in grid.zones]
    seg = []
    for z in grid.zones:
        m = z.mesh
        off = m.face_offsets()
        for f in range(m.n_bface):
            if m.regions[m.bface_region[f]][0] == M.BC_SOLID_SURFACE:
                a, b = m.face2node[off[f]:off[f + 1]]
                seg.append((m.x[a], m.y[a], m.x[b], m.y[b]))
    x0, y0, x1, y1 = (np.array(seg)[:, k][None, :] for k in range(4))
    for z, d in zip(grid.zones, wd):
        m = z.mesh
        cnn = np.asarray(m.cell_nnode)
        cell = np.repeat(np.arange(m.n_cell), cnn)
        px = (np.bincount(cell, m.x[m.cell2node]) / cnn)[:, None]
        py = (np.bincount(cell, m.y[m.cell2node]) / cnn)[:, None]
        dx, dy = x1 - x0, y1 - y0
        t = np.clip(((px - x0) * dx + (py - y0) * dy) / (dx * dx + dy * dy), 0.0, 1.0)
        exact = np.sqrt((px - x0 - t * dx) ** 2 + (py - y0 - t * dy) ** 2).min(axis=1)
        rel = np.abs(exact - d) / d
        assert (d > 0).all()
        if int(cnn.max()) == 3:
            assert np.median(rel) <= 1e-13 and rel.max() <= 1e-5
        else:
            assert rel.max() <= 0.25


@needs_example
def test_two_dimensional_zones_are_refused_by_the_path(grid):
    from oracle.oracle import Oracle

    with pytest.raises(ValueError, match="two-dimensional"):
        Oracle(grid.zones[0].mesh, dict(cases.EULER_BUMP))


@needs_example
def test_reader_names_what_it_does_not_read(grid):
    f = H5File(grid.files[0])
    with pytest.raises(H5Error, match="not a group"):
        f.keys("/Grid-0/iDimensions")
    with pytest.raises(H5Error, match="not a dataset"):
        f.read("/Grid-0/FaceTopology")
    with pytest.raises(KeyError):
        f.read("/Grid-9/iDimensions")


def test_not_an_hdf5_file(tmp_path):
    p = tmp_path / "x.fts"
    p.write_bytes(b"not hdf5" * 100)
    with pytest.raises(H5Error, match="signature"):
        H5File(str(p))
    with pytest.raises(FileNotFoundError):
        fts.read_fts(str(tmp_path / "missing.fts"))


@pytest.mark.parametrize("case_name,nparts", [("laminar", 3), ("sa", 2)])
def test_zone_parts_from_interface_lists_step_like_the_split(case_name, nparts):
    m = M.channel_bump(16, 8, 2)
    params = dict(cases.LAMINAR if case_name == "laminar" else cases.SA_BUMP)
    wd = M.wall_distance(m) if case_name == "sa" else None
    owner = P.slab_owner(m, nparts)
    split = P.split(m, owner)
    # the zones as a grid file holds them: their meshes and interface lists only
    zones = [fts.FtsZone(index=p.rank, proc=p.rank, mesh=p.mesh, ndim=3, interface=itf)
             for p, itf in zip(split, refrun.interface_arrays(split))]
    parts = fts.zone_parts(zones)
    for a, b in zip(split, parts):
        assert a.halo.neighbors == b.halo.neighbors
        for q in a.halo.neighbors:
            assert np.array_equal(a.halo.send[q], b.halo.send[q])
            assert np.array_equal(a.halo.recv[q], b.halo.recv[q])
    # the global cell numbers of the rebuilt parts follow the zones; the split's are the mesh's
    gnum = np.concatenate([p.cells for p in split])
    q0 = cases.perturbed_state(m, params, seed=5)
    ref = PartitionedOracle(m, params, owner=owner, wall_dist=wd)
    ref.set_state(q0)
    h_ref = ref.iterate(3)
    got = PartitionedOracle(None, params, parts=parts, wall_dist=None if wd is None else wd[gnum])
    got.set_state(q0[:, gnum])
    h_got = got.iterate(3)
    assert np.array_equal(h_ref, h_got)
    assert np.array_equal(ref.gather("q")[:, gnum], got.gather("q"))


def _fts_tree(parts, itfs, turned=()):
    """A grid file's groups for the zones `parts` in the reference's layout
    (IO_HDF5Read, Pre_HDF5File.cpp:1270-1990).  Boundary faces listed in
    `turned` are stored the other way round (no left cell, nodes reversed),
    which the reader must undo."""
    n = len(parts)
    tree = {"Version": {"VersionData": np.array([2.0])},
            "Information": {"nBlocks": np.array([n], np.int32), "block_idx": np.arange(n, dtype=np.int32),
                            "block_proc": np.zeros(n, np.int32), "block_type": np.zeros(n, np.int32)}}
    for p, (zid, iid, bf) in zip(parts, itfs):
        m = p.mesh
        nb = m.n_bface
        left = np.asarray(m.left, np.int32).copy()
        right = np.asarray(m.right, np.int32).copy()
        f2n = np.asarray(m.face2node, np.int32).copy()
        off = m.face_offsets()
        for f in turned:
            if f < nb:
                f2n[off[f]:off[f + 1]] = f2n[off[f]:off[f + 1]][::-1].copy()
                left[f], right[f] = -1, left[f]
        btype = np.array([m.regions[r][0] for r in m.bface_region], np.int32)
        names = b"".join(m.regions[r][1].encode() + b"\0" for r in m.bface_region)
        tree[f"Grid-{p.rank}"] = {
            "iDimensions": np.array([m.n_node, m.n_face, m.n_cell], np.int32),
            "GridCoordinates": {"CoordinateX": m.x, "CoordinateY": m.y, "CoordinateZ": m.z},
            "FaceTopology": {"nodeNumberOfEachFace": np.asarray(m.face_nnode, np.int32), "face2Node": f2n,
                             "leftCellOfFace": left, "rightCellOfFace": right,
                             "nBoundFace": np.array([nb], np.int32), "BcType": btype},
            "CellTopology": {"nodeNumberOfEachCell": np.asarray(m.cell_nnode, np.int32),
                             "cell2Node": np.asarray(m.cell2node, np.int32)},
            "BCName": {"BCName": np.frombuffer(names, np.int8)},
            "InterfaceInfo": {"nIFace": np.array([len(zid)], np.int32), "interFace2ZoneID": zid,
                              "interFace2InterFaceID": iid, "interFace2BoundaryFace": bf},
        }
    return tree


def test_a_three_dimensional_grid_file_reads_back_and_steps_like_the_split(tmp_path):
    """Zones of a split hex/prism channel written as a grid file (numbered
    files, some boundary faces stored the other way round) come back as the
    same meshes and interface lists, and step bit for bit as the split."""
    from tests.h5write import write_h5

    m = M.channel_bump(16, 8, 2, prism_layers=2)
    params = dict(cases.LAMINAR)
    owner = P.slab_owner(m, 3)
    split = P.split(m, owner)
    itfs = refrun.interface_arrays(split)
    tree = _fts_tree(split, itfs, turned=(0, 3, 5))
    # the reference's writer names the files of a grid name_0, name_1, ...:
    # two files here, zones 0 and 1 in the first, zone 2 in the second
    # (each file's /Information lists its own zones)
    info = lambda idx: {"nBlocks": np.array([len(idx)], np.int32), "block_idx": np.array(idx, np.int32),  # noqa: E731
                        "block_proc": np.array(idx, np.int32), "block_type": np.zeros(len(idx), np.int32)}
    first = {k: v for k, v in tree.items() if k != "Grid-2"}
    first["Information"] = info([0, 1])
    second = {"Version": tree["Version"], "Grid-2": tree["Grid-2"], "Information": info([2])}
    write_h5(str(tmp_path / "chan__3_0.fts"), first)
    write_h5(str(tmp_path / "chan__3_1.fts"), second)
    grid = fts.read_fts(str(tmp_path / "chan__3.fts"))
    assert len(grid.files) == 2 and [z.index for z in grid.zones] == [0, 1, 2]
    assert [z.proc for z in grid.zones] == [0, 1, 2]
    for z, p, itf in zip(grid.zones, split, itfs):
        a, b = z.mesh, p.mesh
        assert z.ndim == 3
        for k in ("x", "y", "z", "face_nnode", "face2node", "left", "right", "cell_nnode", "cell2node"):
            assert np.array_equal(getattr(a, k), getattr(b, k)), k
        assert a.n_bface == b.n_bface
        assert [a.regions[r] for r in a.bface_region] == [b.regions[r] for r in b.bface_region]
        for x, y in zip(z.interface, itf):
            assert np.array_equal(x, y)
    gnum = np.concatenate([p.cells for p in split])
    q0 = cases.perturbed_state(m, params, seed=9)
    ref = PartitionedOracle(m, params, owner=owner)
    ref.set_state(q0)
    got = PartitionedOracle(None, params, parts=fts.zone_parts(grid.zones))
    got.set_state(q0[:, gnum])
    assert np.array_equal(ref.iterate(3), got.iterate(3))
    assert np.array_equal(ref.gather("q")[:, gnum], got.gather("q"))


def test_the_reference_restart_layout_reads_back(tmp_path):
    """Restart files in the layout of CFDSolver::CreateH5RestartFile and the
    DumpRestartH5 methods: the flow file's q of cells and ghosts and
    outnstep, the turbulence file's q_turb and visturb; a restart of
    another grid is refused."""
    from tests.h5write import write_h5

    nc, nb = 40, 12
    nt = nc + nb
    rng = np.random.default_rng(4)
    q = rng.standard_normal((5, nt))
    write_h5(str(tmp_path / "flow.dat"), {
        "Version": np.array([1], np.int32), "outnstep": np.array([1234], np.int32),
        "Group3": {"q": q, "t": rng.standard_normal((1, nt)), "nTotalCell": np.array([nc], np.int32)}})
    qt, vt = rng.standard_normal((1, nt)), rng.standard_normal((1, nt))
    write_h5(str(tmp_path / "turb.dat"), {
        "Version": np.array([1], np.int32), "outnstep": np.array([1234], np.int32),
        "Group3": {"q_turb": qt, "visturb": vt, "nTotalCell": np.array([nc], np.int32)}})
    r = fts.read_restart_h5(str(tmp_path / "flow.dat"), 3, nc, nb, str(tmp_path / "turb.dat"))
    assert r["outnstep"] == 1234
    assert np.array_equal(r["q"], q)
    assert np.array_equal(r["q_turb"], qt[0]) and np.array_equal(r["vist"], vt[0])
    with pytest.raises(ValueError, match="cells"):
        fts.read_restart_h5(str(tmp_path / "flow.dat"), 3, nc + 1, nb)
    with pytest.raises(ValueError, match="Group0"):
        fts.read_restart_h5(str(tmp_path / "flow.dat"), 0, nc, nb)


def _file_rank_main(rank, world, port, path, out):
    import datetime
    import os

    import torch.distributed as dist

    from oracle.partitioned import DistributedOracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        grid = fts.read_fts(path)
        params = dict(cases.LAMINAR)
        do = DistributedOracle(None, params, rank, world, parts=fts.zone_parts(grid.zones))
        n = sum(z.mesh.n_cell for z in grid.zones)
        q0 = cases.perturbed_state(M.channel_bump(16, 8, 2), params, seed=2)[:, :n]
        do.set_state(q0)
        hist = do.iterate(3)
        np.savez(os.path.join(out, f"rank{rank}.npz"), hist=hist, cells=do.local_cells(), q=do.gather("q"))
    finally:
        dist.destroy_process_group()


def test_grid_file_zones_on_two_gloo_ranks_equal_in_process(tmp_path):
    """Each of two ranks reads the grid file and steps its own zone, halos
    over gloo: the same history and state as all zones in one process."""
    import torch.multiprocessing as mp

    from tests.h5write import write_h5
    from tests.test_partition import _free_port

    m = M.channel_bump(16, 8, 2)
    split = P.split(m, P.slab_owner(m, 2))
    path = str(tmp_path / "two.fts")
    write_h5(path, _fts_tree(split, refrun.interface_arrays(split)))
    mp.spawn(_file_rank_main, args=(2, _free_port(), path, str(tmp_path)), nprocs=2, join=True)
    grid = fts.read_fts(path)
    params = dict(cases.LAMINAR)
    po = PartitionedOracle(None, params, parts=fts.zone_parts(grid.zones))
    n = sum(z.mesh.n_cell for z in grid.zones)
    po.set_state(cases.perturbed_state(m, params, seed=2)[:, :n])
    h = po.iterate(3)
    q = po.gather("q")
    for r in range(2):
        d = np.load(tmp_path / f"rank{r}.npz")
        assert np.array_equal(d["hist"], h)
        assert np.array_equal(d["q"][:, d["cells"]], q[:, d["cells"]])


@pytest.mark.parametrize("version", [0, 1])
def test_superblock_versions_and_damaged_files(tmp_path, version):
    """Both superblock versions the library writes with default settings
    read; a file cut short raises H5Error instead of misreading."""
    from tests.h5write import write_h5

    a = np.arange(1000, dtype=np.float64)
    path = tmp_path / "x.h5"
    write_h5(str(path), {"g": {"a": a, "n": np.array([7], np.int32)}}, superblock_version=version)
    f = H5File(str(path))
    assert np.array_equal(f.read("/g/a"), a) and int(f.read("/g/n")[0]) == 7
    data = path.read_bytes()
    cut = tmp_path / "cut.h5"
    cut.write_bytes(data[: len(data) // 3])
    with pytest.raises(H5Error):
        g = H5File(str(cut))
        g.read("/g/a")
        g.read("/g/n")
