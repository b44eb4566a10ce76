"""PHengLEI's unstructured grid files (.fts, HDF5), read into this package's
Mesh layout without an HDF5 library (phenlei_b200.h5lite reads the file).

The reference reads them with IO_HDF5Read (API/PreProcess/src/Pre_HDF5File.cpp):

* a grid named `name.fts` is stored as the files `name_0.fts`, `name_1.fts`,
  ... (IO_HDF5Read::CheckNumberofFiles, :819-860, AddSymbolToFileName);
* each file lists its zones in /Information (nBlocks, block_idx, block_proc,
  block_type) and holds zone i in the group /Grid-i (ReadEachGrid, :1270-1316);
* ReadUnstructGrid (:1753-1797) reads iDimensions (nodes, faces, cells),
  GridCoordinates, FaceTopology, InterfaceInfo, CellTopology, BCName and
  InterpointInfo;
* the stored wall distances sit beside each grid file in `name_i.wdt`
  (ReadWallDist, :910-1024).

ReadFaceTopology (:1799-1847) reverses the node list of every face whose left
cell is negative and swaps its two cells, so that every face has a cell on its
left; boundary faces come first (nBoundFace of them).  ReadUnstrBCName
(:1867-1940) gives every boundary face its BcType and its region name (the
BCName dataset: one NUL-terminated name per boundary face).  Interface faces
(BcType PHENGLEI::INTERFACE, -1) join the zones: face k of zone i's interface
list is boundary face interFace2BoundaryFace[k] and is face
interFace2InterFaceID[k] of zone interFace2ZoneID[k]'s list
(ReadInterfaceInfo, :1366-1405).

`read_fts` returns the zones; `zone_parts` turns them into the parts that
phenlei_b200.zones (CUDA) and oracle.partitioned (CPU) step, their halo plans
made from the interface lists.  The solver path is three-dimensional; zones of
a two-dimensional grid (faces of two nodes) are read but not accepted by it.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np

from . import partition as P
from .h5lite import H5File
from .mesh import BC_INTERFACE, Mesh

UNSTRUCTGRID = 0   # block_type of an unstructured zone (PHSPACE::UNSTRUCTGRID)


@dataclass
class FtsZone:
    index: int              # the zone's global index (block_idx)
    proc: int               # the processor the file assigns it to (block_proc)
    mesh: Mesh
    ndim: int               # 2 when every face has two nodes, else 3
    interface: tuple        # (interFace2ZoneID, interFace2InterFaceID, interFace2BoundaryFace), int32
    interpoint: dict = field(default_factory=dict)   # the InterpointInfo arrays as stored


@dataclass
class FtsGrid:
    version: float
    files: list
    zones: list             # FtsZone, ascending global index


def grid_files(path: str) -> list:
    """The files of the grid `path`: the file itself if it exists, else
    `stem_0.ext`, `stem_1.ext`, ... for as long as they exist."""
    if os.path.exists(path):
        return [path]
    stem, ext = os.path.splitext(path)
    out = []
    while os.path.exists(f"{stem}_{len(out)}{ext}"):
        out.append(f"{stem}_{len(out)}{ext}")
    if not out:
        raise FileNotFoundError(path)
    return out


def _ints(f: H5File, path: str) -> np.ndarray:
    return np.asarray(f.read(path), np.int64).reshape(-1)


def _zone(f: H5File, g: str, index: int, proc: int) -> FtsZone:
    nn, nf, nc = (int(v) for v in _ints(f, g + "/iDimensions")[:3])
    x = np.asarray(f.read(g + "/GridCoordinates/CoordinateX"), np.float64).reshape(-1)
    y = np.asarray(f.read(g + "/GridCoordinates/CoordinateY"), np.float64).reshape(-1)
    z = np.asarray(f.read(g + "/GridCoordinates/CoordinateZ"), np.float64).reshape(-1)
    ft = g + "/FaceTopology"
    fnn = _ints(f, ft + "/nodeNumberOfEachFace")
    f2n = _ints(f, ft + "/face2Node")
    left = _ints(f, ft + "/leftCellOfFace")
    right = _ints(f, ft + "/rightCellOfFace")
    nb = int(_ints(f, ft + "/nBoundFace")[0])
    if not (x.size == y.size == z.size == nn and fnn.size == left.size == right.size == nf
            and f2n.size == int(fnn.sum()) and 0 <= nb <= nf):
        raise ValueError(f"{g}: array sizes disagree with iDimensions")
    # ReadFaceTopology: a face with no left cell is turned round
    flip = left < 0
    if flip.any():
        off = np.zeros(nf + 1, np.int64)
        np.cumsum(fnn, out=off[1:])
        pos = np.arange(f2n.size) - np.repeat(off[:-1], fnn)          # position within the face
        rev = np.repeat(off[:-1], fnn) + (np.repeat(fnn, fnn) - 1 - pos)
        f2n = np.where(np.repeat(flip, fnn), f2n[rev], f2n)
        left, right = np.where(flip, right, left), np.where(flip, left, right)
    right = right.copy()
    right[:nb] = -1                        # SpecifyRightCellofBC: the ghost cell nCell + face
    if (left < 0).any() or (left >= nc).any() or (right[nb:] < 0).any() or (right[nb:] >= nc).any():
        raise ValueError(f"{g}: a face without a valid cell on each side")
    if (f2n < 0).any() or (f2n >= nn).any():
        raise ValueError(f"{g}: a face node out of range")
    ct = g + "/CellTopology"
    cnn = _ints(f, ct + "/nodeNumberOfEachCell")
    c2n = _ints(f, ct + "/cell2Node")
    if cnn.size != nc or c2n.size != int(cnn.sum()):
        raise ValueError(f"{g}: cell topology sizes disagree with iDimensions")
    # ReadUnstrBCName: one BcType and one NUL-terminated name per boundary face
    btype = _ints(f, ft + "/BcType")[:nb]
    raw = bytes(np.asarray(f.read(g + "/BCName/BCName")).astype(np.uint8))
    names = [s.decode() for s in raw.split(b"\0")[:nb]]
    if btype.size != nb or len(names) != nb:
        raise ValueError(f"{g}: {nb} boundary faces, {btype.size} types, {len(names)} names")
    regions, rid, bregion = [], {}, np.empty(nb, np.int32)
    for i, key in enumerate(zip(btype.tolist(), names)):
        if key not in rid:
            rid[key] = len(regions)
            regions.append(key)
        bregion[i] = rid[key]
    it = g + "/InterfaceInfo"
    n_if = int(_ints(f, it + "/nIFace")[0]) if f.exists(it + "/nIFace") else 0
    if n_if:
        itf = tuple(_ints(f, f"{it}/{k}").astype(np.int32)
                    for k in ("interFace2ZoneID", "interFace2InterFaceID", "interFace2BoundaryFace"))
    else:
        itf = tuple(np.zeros(0, np.int32) for _ in range(3))
    if n_if and not np.array_equal(np.sort(itf[2]), np.flatnonzero(btype == BC_INTERFACE)):
        raise ValueError(f"{g}: the interface list and the INTERFACE boundary faces differ")
    ip = {}
    if f.exists(g + "/InterpointInfo"):
        for k in f.keys(g + "/InterpointInfo"):
            ip[k] = np.asarray(f.read(f"{g}/InterpointInfo/{k}"))
    mesh = Mesh(x=x, y=y, z=z, face_nnode=fnn.astype(np.int32), face2node=f2n.astype(np.int32),
                left=left.astype(np.int32), right=right.astype(np.int32), cell_nnode=cnn.astype(np.int32),
                cell2node=c2n.astype(np.int32), n_bface=nb, bface_region=bregion, regions=regions)
    ndim = 2 if nf and int(fnn.max()) == 2 else 3
    return FtsZone(index=index, proc=proc, mesh=mesh, ndim=ndim, interface=itf, interpoint=ip)


def read_fts(path: str) -> FtsGrid:
    """Every zone of the grid `path` (one file, or the numbered files of a
    grid written in parts)."""
    files = grid_files(path)
    zones, version = [], None
    for fn in files:
        f = H5File(fn)
        if f.exists("/Version/VersionData"):
            version = float(np.asarray(f.read("/Version/VersionData")).reshape(-1)[0])
        n = int(_ints(f, "/Information/nBlocks")[0])
        idx = _ints(f, "/Information/block_idx")
        proc = _ints(f, "/Information/block_proc")
        btype = _ints(f, "/Information/block_type")
        if min(idx.size, proc.size, btype.size) < n:
            raise ValueError(f"{fn}: /Information lists fewer than nBlocks zones")
        for i in range(n):
            # ReadTotalInfo / ReadEachGrid (:1149-1203, :1270-1316): the file's
            # i-th entries give the zone's global index, its processor and its
            # type; the zone is the group Grid-<global index>
            gi = int(idx[i])
            if int(btype[i]) != UNSTRUCTGRID:
                raise ValueError(f"zone {gi} is a structured zone; only unstructured zones are read")
            zones.append(_zone(f, f"/Grid-{gi}", gi, int(proc[i])))
    zones.sort(key=lambda z: z.index)
    if [z.index for z in zones] != list(range(len(zones))):
        raise ValueError("the zone indices are not 0..n-1")
    return FtsGrid(version=version, files=files, zones=zones)


def read_wall_distance(grid: FtsGrid) -> list:
    """The wall distance of every cell of every zone from the grid's `.wdt`
    files, the reference's stored wall distances (IO_HDF5Read::ReadWallDist,
    API/PreProcess/src/Pre_HDF5File.cpp:910-1024): beside each grid file
    `name_i.fts` the file `name_i.wdt` holds one dataset Grid-<zone> of n_cell
    values per zone.  Returns a list in zone order, or None where the files
    are missing (the reference then computes the distances itself)."""
    per_zone = {}
    for fn in grid.files:
        wdt = os.path.splitext(fn)[0] + ".wdt"
        if not os.path.exists(wdt):
            return None
        f = H5File(wdt)
        for k in f.keys("/"):
            if k.startswith("Grid-") and k[5:].isdigit():
                per_zone[int(k[5:])] = np.asarray(f.read("/" + k), np.float64).reshape(-1)
    out = []
    for z in grid.zones:
        d = per_zone.get(z.index)
        if d is None or d.size != z.mesh.n_cell:
            raise ValueError(f"zone {z.index}: the wall distance file does not hold one value per cell")
        out.append(d)
    return out


def read_restart_h5(path: str, zone: int, n_cell: int, n_bface: int, turb_path: str | None = None) -> dict:
    """The reference's HDF5 restart of one zone, as NSSolverUnstruct::ReadRestartH5
    (CFD/NSSolver/src/NSSolverUnstruct.cpp:1400-1440) and
    TurbSolverUnstr::ReadRestartH5 (CFD/TurbSolver/src/TurbSolverUnstr.cpp:638-693)
    read it.  The flow file holds `outnstep` and, in the group Group<zone>
    (CFDSolver::CreateH5RestartFile, CFD/Solver/src/CFDSolver.cpp:2345-2522),
    `nTotalCell` and `q` [nEquation][nTotalCell + nBoundFace] of FP64
    primitive variables of the cells and their ghosts (and `t`); the
    turbulence file holds `q_turb` [nTurbulenceEquation][...] and `visturb`.
    A restart of another grid (its nTotalCell differs) is refused, as the
    reference refuses it.  Returns outnstep, q [5][nTotal] and, with
    `turb_path`, q_turb [nTotal] and vist [nTotal] (None where the file has
    no visturb, which the reference then leaves as it was)."""
    nt = n_cell + n_bface
    g = f"/Group{zone}"

    def zone_group(f: H5File, what: str):
        if not f.exists(g):
            raise ValueError(f"the {what} restart has no group {g[1:]}")
        n = int(np.asarray(f.read(g + "/nTotalCell")).reshape(-1)[0])
        if n != n_cell:
            raise ValueError(f"the {what} restart holds {n} cells, the grid {n_cell}")

    def rows(a: np.ndarray, nrow: int) -> np.ndarray:
        a = np.asarray(a, np.float64).reshape(-1)
        if a.size < nrow * nt or a.size % nrow:
            raise ValueError(f"{a.size} values cannot hold {nrow} rows of {nt}")
        return a.reshape(nrow, -1)[:, :nt].copy()

    f = H5File(path)
    zone_group(f, "flow")
    out = {"outnstep": int(np.asarray(f.read("/outnstep")).reshape(-1)[0]),
           "q": rows(f.read(g + "/q"), 5)}
    if turb_path is not None:
        ft = H5File(turb_path)
        zone_group(ft, "turbulence")
        out["q_turb"] = rows(ft.read(g + "/q_turb"), 1)[0]
        out["vist"] = rows(ft.read(g + "/visturb"), 1)[0] if ft.exists(g + "/visturb") else None
    return out


def zone_parts(zones: list) -> list:
    """The parts (phenlei_b200.partition.Part) of the zones, for
    phenlei_b200.zones and oracle.partitioned: zone i is part i, its cells
    numbered globally after those of the zones before it.  Interface face k
    of zone i receives the cell on the left of face interFace2InterFaceID[k]
    of zone interFace2ZoneID[k], which in turn sends it.  Each zone's
    interface faces must be its last boundary faces, in their list's order
    (as the reference's partitioner writes them)."""
    n = len(zones)
    starts = np.cumsum([0] + [z.mesh.n_cell for z in zones])
    fstarts = np.cumsum([0] + [z.mesh.n_face for z in zones])
    parts = []
    for i, zn in enumerate(zones):
        m = zn.mesh
        zid, iid, bf = (np.asarray(a, np.int64) for a in zn.interface)
        first = m.n_bface - bf.size
        if not np.array_equal(bf, np.arange(first, m.n_bface)):
            raise ValueError(f"zone {i}: the interface faces are not the last boundary faces in list order")
        if ((zid < 0) | (zid >= n) | (zid == i)).any():
            raise ValueError(f"zone {i}: an interface face names no other zone")
        parts.append(P.Part(rank=i, mesh=m, cells=starts[i] + np.arange(m.n_cell), faces=fstarts[i] + np.arange(m.n_face),
                            flipped=np.zeros(m.n_face, bool), nodes=np.arange(m.n_node), iface_first=int(first),
                            n_iface=int(bf.size), halo=P.Halo(neighbors=[], send={}, recv={})))
    for i, (zn, part) in enumerate(zip(zones, parts)):
        zid, iid, bf = (np.asarray(a, np.int64) for a in zn.interface)
        for q in np.unique(zid):
            sel = np.flatnonzero(zid == q)
            other = zones[int(q)]
            ozid, oiid, obf = (np.asarray(a, np.int64) for a in other.interface)
            k = iid[sel]
            if (k < 0).any() or (k >= ozid.size).any() or (ozid[k] != i).any() or (oiid[k] != sel).any():
                raise ValueError(f"zones {i} and {int(q)}: the interface lists do not point back at each other")
            part.halo.recv[int(q)] = part.mesh.n_cell + bf[sel]
            parts[int(q)].halo.send[i] = np.asarray(other.mesh.left, np.int64)[obf[k]]
            # both zones name the face pair by one number: the lower zone's global face
            if i < int(q):
                parts[int(q)].faces[obf[k]] = part.faces[bf[sel]]
    for part in parts:
        part.halo.neighbors = sorted(part.halo.recv)
        if sorted(part.halo.send) != part.halo.neighbors:
            raise ValueError(f"zone {part.rank}: its send and receive partners differ")
    return parts
