"""Synthetic unstructured grids in the reference's face-based layout.

The layout is the one `UnstructGrid` holds after reading a grid file
(API/PreProcess/src/Pre_HDF5File.cpp:1799-1847, API/Geometry/src/Geo_UnstructGrid.cpp):

* nodes `x, y, z`;
* faces as node lists (`face_nnode`, `face2node`), boundary faces first;
  the node order makes the right-hand-rule normal point from the left cell to
  the right cell (outward for boundary faces, whose right cell is -1 here and
  becomes the ghost index nTotalCell + iFace in the solver);
* `cell2node` as the sorted set of each cell's nodes (the reference's
  `ComputeCell2Node`, Geo_UnstructGrid.cpp:954-1024, builds it this way);
* boundary regions: one (bcType, name) per region and a region index per
  boundary face.

Generators, all seeded and deterministic:

* `channel_bump`  hexahedral 3-D channel with a circular-arc bump on the lower
  wall, y tanh-stretched (the Euler bump and the transonic bump cases);
* `flat_plate`    hexahedral flat-plate boundary-layer box with an inviscid
  lead-in section;
* `tet_cube`      unit cube, n^3 hexes split into 6 tetrahedra each, interior
  nodes jittered.
"""
from __future__ import annotations

import dataclasses
import struct

import numpy as np

# Boundary-condition codes of the reference (API/Geometry/include/Geo_SimpleBC.h:32-39).
BC_SOLID_SURFACE = 2
BC_SYMMETRY = 3
BC_FARFIELD = 4
BC_INFLOW = 5
BC_OUTFLOW = 6
BC_INTERFACE = -1   # PHENGLEI::INTERFACE: a face cut by a partition (ghost = the neighbouring zone's cell)


@dataclasses.dataclass
class Mesh:
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    face_nnode: np.ndarray     # int32 [nFace]
    face2node: np.ndarray      # int32 [sum(face_nnode)]
    left: np.ndarray           # int32 [nFace]
    right: np.ndarray          # int32 [nFace], -1 on boundary faces
    cell_nnode: np.ndarray     # int32 [nCell]
    cell2node: np.ndarray      # int32 [sum(cell_nnode)]
    n_bface: int
    bface_region: np.ndarray   # int32 [nBFace]
    regions: list              # [(bcType, name)]

    def solver_regions(self):
        """Boundary regions in the order the reference solver numbers them
        (by name, as the std::set<string> of ReadUnstrBCName orders them,
        Pre_HDF5File.cpp:1753-1940): their bcTypes, and each boundary face's
        region in that numbering."""
        order = sorted(range(len(self.regions)), key=lambda r: self.regions[r][1])
        rank = np.empty(len(self.regions), np.int32)
        rank[order] = np.arange(len(order), dtype=np.int32)
        rtype = np.array([self.regions[r][0] for r in order], np.int32)
        return rtype, rank[np.asarray(self.bface_region, np.int64)].astype(np.int32)

    @property
    def n_node(self) -> int:
        return int(self.x.size)

    @property
    def n_face(self) -> int:
        return int(self.face_nnode.size)

    @property
    def n_cell(self) -> int:
        return int(self.cell_nnode.size)

    def face_offsets(self) -> np.ndarray:
        off = np.zeros(self.n_face + 1, dtype=np.int64)
        np.cumsum(self.face_nnode, out=off[1:])
        return off

    def cell_offsets(self) -> np.ndarray:
        off = np.zeros(self.n_cell + 1, dtype=np.int64)
        np.cumsum(self.cell_nnode, out=off[1:])
        return off


def wall_distance(m: Mesh) -> np.ndarray:
    """Distance of each cell's node-average centre to the nearest node-average
    centre of a solid-wall face (k-d tree).  A stand-in for the reference's
    wall-distance preprocessing (Pre_WalldistCompute) for generated meshes; the
    SA path takes the wall distance as an input, and parity tests give both
    sides the reference's own values."""
    from scipy.spatial import cKDTree

    fo = m.face_offsets()
    walls = np.array([t == BC_SOLID_SURFACE for t, _ in m.regions])
    wf = np.flatnonzero(walls[m.bface_region[: m.n_bface]])
    if wf.size == 0:
        raise ValueError("the mesh has no solid-wall faces")
    xyz = np.stack([m.x, m.y, m.z], axis=1)
    nb_end = int(fo[m.n_bface])
    bsum = np.add.reduceat(xyz[m.face2node[:nb_end]], fo[: m.n_bface], axis=0)
    fc = (bsum / m.face_nnode[: m.n_bface, None])[wf]
    co = m.cell_offsets()
    csum = np.add.reduceat(xyz[m.cell2node[: co[-1]]], co[:-1], axis=0)
    cc = csum / m.cell_nnode[:, None]
    d, _ = cKDTree(fc).query(cc, workers=-1)
    return d


def write_mesh(path: str, m: Mesh) -> None:
    """Raw little-endian file read by the oracle's reference harness."""
    with open(path, "wb") as f:
        f.write(b"PHXMESH1")
        f.write(struct.pack("<7q", m.n_node, m.n_face, m.n_cell, m.n_bface,
                            m.face2node.size, m.cell2node.size, len(m.regions)))
        for a in (m.x, m.y, m.z):
            f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())
        for a in (m.face_nnode, m.face2node, m.left, m.right, m.cell_nnode,
                  m.cell2node, m.bface_region):
            f.write(np.ascontiguousarray(a, dtype="<i4").tobytes())
        for t, name in m.regions:
            nb = name.encode()
            f.write(struct.pack("<ii", t, len(nb)))
            f.write(nb)


# ----------------------------------------------------------------------------
# structured hexahedral block -> unstructured faces
# ----------------------------------------------------------------------------

def _hex_block(X: np.ndarray, side_region: dict, regions: list) -> Mesh:
    """Unstructured form of a structured block of hexahedra.

    X has shape (ni+1, nj+1, nk+1, 3).  Cells are numbered i fastest, then j,
    then k.  side_region maps "imin/imax/jmin/jmax/kmin/kmax" to a region
    index, or to a callable (face-centre coordinates -> region index array).
    """
    ni, nj, nk = (s - 1 for s in X.shape[:3])
    nid = np.arange((ni + 1) * (nj + 1) * (nk + 1), dtype=np.int64).reshape(
        (nk + 1, nj + 1, ni + 1)).transpose(2, 1, 0)  # nid[i,j,k]
    cid = np.arange(ni * nj * nk, dtype=np.int64).reshape((nk, nj, ni)).transpose(2, 1, 0)

    def quad(a, b, c, d):
        return np.stack([a.ravel(), b.ravel(), c.ravel(), d.ravel()], axis=1)

    # Faces normal to +i: nodes (j,k),(j+1,k),(j+1,k+1),(j,k+1).
    def ifaces(i):
        return quad(nid[i, :-1, :-1], nid[i, 1:, :-1], nid[i, 1:, 1:], nid[i, :-1, 1:])

    def jfaces(j):
        return quad(nid[:-1, j, :-1], nid[:-1, j, 1:], nid[1:, j, 1:], nid[1:, j, :-1])

    def kfaces(k):
        return quad(nid[:-1, :-1, k], nid[1:, :-1, k], nid[1:, 1:, k], nid[:-1, 1:, k])

    bnd_nodes, bnd_left, bnd_side = [], [], []
    for side, (nodes, cells, flip) in {
        "imin": (ifaces(0), cid[0, :, :], True),
        "imax": (ifaces(ni), cid[ni - 1, :, :], False),
        "jmin": (jfaces(0), cid[:, 0, :], True),
        "jmax": (jfaces(nj), cid[:, nj - 1, :], False),
        "kmin": (kfaces(0), cid[:, :, 0], True),
        "kmax": (kfaces(nk), cid[:, :, nk - 1], False),
    }.items():
        if flip:
            nodes = nodes[:, ::-1]
        bnd_nodes.append(nodes)
        bnd_left.append(cells.ravel())
        bnd_side.append(side)

    xyz = X.transpose(2, 1, 0, 3).reshape(-1, 3)  # node id = i + (ni+1)*(j + (nj+1)*k)
    # Region per boundary face.
    regs = []
    for nodes, side in zip(bnd_nodes, bnd_side):
        r = side_region[side]
        if callable(r):
            fc = xyz[nodes].mean(axis=1)
            regs.append(np.asarray(r(fc), dtype=np.int32))
        else:
            regs.append(np.full(nodes.shape[0], r, dtype=np.int32))
    bnodes = np.concatenate(bnd_nodes)
    bleft = np.concatenate(bnd_left)
    breg = np.concatenate(regs)
    # Boundary faces grouped by region (stable), then interior faces.
    order = np.argsort(breg, kind="stable")
    bnodes, bleft, breg = bnodes[order], bleft[order], breg[order]

    inodes, ileft, iright = [], [], []
    for i in range(1, ni):
        inodes.append(ifaces(i)); ileft.append(cid[i - 1].ravel()); iright.append(cid[i].ravel())
    for j in range(1, nj):
        inodes.append(jfaces(j)); ileft.append(cid[:, j - 1].ravel()); iright.append(cid[:, j].ravel())
    for k in range(1, nk):
        inodes.append(kfaces(k)); ileft.append(cid[:, :, k - 1].ravel()); iright.append(cid[:, :, k].ravel())
    inodes = np.concatenate(inodes) if inodes else np.zeros((0, 4), np.int64)
    ileft = np.concatenate(ileft) if ileft else np.zeros(0, np.int64)
    iright = np.concatenate(iright) if iright else np.zeros(0, np.int64)

    faces = np.concatenate([bnodes, inodes])
    left = np.concatenate([bleft, ileft])
    right = np.concatenate([np.full(bleft.size, -1), iright])

    cnodes = np.stack([nid[:-1, :-1, :-1], nid[1:, :-1, :-1], nid[:-1, 1:, :-1], nid[1:, 1:, :-1],
                       nid[:-1, :-1, 1:], nid[1:, :-1, 1:], nid[:-1, 1:, 1:], nid[1:, 1:, 1:]],
                      axis=-1).transpose(2, 1, 0, 3).reshape(-1, 8)
    cnodes = np.sort(cnodes, axis=1)
    return Mesh(
        x=np.ascontiguousarray(xyz[:, 0]), y=np.ascontiguousarray(xyz[:, 1]),
        z=np.ascontiguousarray(xyz[:, 2]),
        face_nnode=np.full(faces.shape[0], 4, np.int32),
        face2node=faces.astype(np.int32).ravel(),
        left=left.astype(np.int32), right=right.astype(np.int32),
        cell_nnode=np.full(cnodes.shape[0], 8, np.int32),
        cell2node=cnodes.astype(np.int32).ravel(),
        n_bface=int(bnodes.shape[0]), bface_region=breg.astype(np.int32), regions=regions)


def _hex_prism_block(X: np.ndarray, jp: int, side_region: dict, regions: list) -> Mesh:
    """Structured block with its first `jp` j-layers split into prisms.

    Each hexahedron (i, j, k) with j < jp becomes two prisms with triangles
    (i,k)(i+1,k)(i+1,k+1) [A] and (i,k)(i+1,k+1)(i,k+1) [B] in the x-z plane,
    extruded in j.  The hexahedra of layer jp see the prism layer's top as two
    triangular faces (7 faces per cell).  Cells are numbered k slowest, then j,
    then i (prism pairs A, B adjacent); boundary faces come first, grouped by
    region, then interior faces ordered by (left, right).  Faces are oriented
    from the left cell to the right cell (outward on the boundary).
    """
    ni, nj, nk = (s_ - 1 for s_ in X.shape[:3])
    jp = max(0, min(jp, nj))
    xyz = X.transpose(2, 1, 0, 3).reshape(-1, 3)

    def nid(i, j, k):
        return (i + (ni + 1) * (j + (nj + 1) * k)).astype(np.int64)

    S = jp * 2 * ni + (nj - jp) * ni

    def cA(i, j, k):
        return k * S + j * 2 * ni + 2 * i

    def cH(i, j, k):
        return k * S + jp * 2 * ni + (j - jp) * ni + i

    def grid(*shape_ranges):
        return np.meshgrid(*[np.arange(a, b, dtype=np.int64) for a, b in shape_ranges], indexing="ij")

    F, L, R, SIDE = [], [], [], []   # face node arrays, left, right (-1 boundary), boundary side

    def add(nodes, left, right, side=None):
        F.append(nodes); L.append(left.ravel()); R.append(right.ravel())
        SIDE.append(np.full(left.size, -1 if side is None else side, np.int8))

    sides = ["imin", "imax", "jmin", "jmax", "kmin", "kmax"]
    # i-faces
    for lo_j, hi_j, prism in ((0, jp, True), (jp, nj, False)):
        if hi_j <= lo_j:
            continue
        ii, j, k = grid((0, ni + 1), (lo_j, hi_j), (0, nk))
        q = np.stack([nid(ii, j, k), nid(ii, j + 1, k), nid(ii, j + 1, k + 1), nid(ii, j, k + 1)], -1).reshape(-1, 4)
        minus = (cA(ii - 1, j, k) if prism else cH(ii - 1, j, k)).ravel()       # A has the +x side
        plus = (cA(ii, j, k) + 1 if prism else cH(ii, j, k)).ravel()           # B has the -x side
        iiv = ii.ravel()
        inner = (iiv > 0) & (iiv < ni)
        add(q[inner], minus[inner], plus[inner])
        add(q[iiv == 0], plus[iiv == 0], np.full(int((iiv == 0).sum()), -1), 0)
        add(q[iiv == ni], minus[iiv == ni], np.full(int((iiv == ni).sum()), -1), 1)
    # k-faces
    for lo_j, hi_j, prism in ((0, jp, True), (jp, nj, False)):
        if hi_j <= lo_j:
            continue
        i, j, kk = grid((0, ni), (lo_j, hi_j), (0, nk + 1))
        q = np.stack([nid(i, j, kk), nid(i + 1, j, kk), nid(i + 1, j + 1, kk), nid(i, j + 1, kk)], -1).reshape(-1, 4)
        minus = (cA(i, j, kk - 1) + 1 if prism else cH(i, j, kk - 1)).ravel()  # B has the +z side
        plus = (cA(i, j, kk) if prism else cH(i, j, kk)).ravel()               # A has the -z side
        kv = kk.ravel()
        inner = (kv > 0) & (kv < nk)
        add(q[inner], minus[inner], plus[inner])
        add(q[kv == 0], plus[kv == 0], np.full(int((kv == 0).sum()), -1), 4)
        add(q[kv == nk], minus[kv == nk], np.full(int((kv == nk).sum()), -1), 5)
    # j-faces: triangles up to and including the interface jp, quads above
    if jp > 0:
        i, jj, k = grid((0, ni), (0, jp + 1), (0, nk))
        n00, n10, n11, n01 = nid(i, jj, k), nid(i + 1, jj, k), nid(i + 1, jj, k + 1), nid(i, jj, k + 1)
        for tri, off in ((np.stack([n00, n10, n11], -1), 0), (np.stack([n00, n11, n01], -1), 1)):
            t = tri.reshape(-1, 3)
            jv = jj.ravel()
            below = (cA(i, jj - 1, k) + off).ravel()
            above = np.where(jj < jp, cA(i, jj, k) + off, cH(i, np.minimum(jj, nj - 1), k) if jp < nj else -1).ravel()
            inner = (jv > 0) & ((jv < jp) | ((jv == jp) & (jp < nj)))
            add(t[inner], below[inner], above[inner])
            add(t[jv == 0], above[jv == 0], np.full(int((jv == 0).sum()), -1), 2)
            if jp == nj:
                add(t[jv == nj], below[jv == nj], np.full(int((jv == nj).sum()), -1), 3)
    if jp < nj:
        i, jj, k = grid((0, ni), (jp if jp > 0 else 0, nj + 1), (0, nk))
        q = np.stack([nid(i, jj, k), nid(i, jj, k + 1), nid(i + 1, jj, k + 1), nid(i + 1, jj, k)], -1).reshape(-1, 4)
        jv = jj.ravel()
        below = cH(i, np.maximum(jj - 1, jp), k).ravel()
        above = cH(i, np.minimum(jj, nj - 1), k).ravel()
        inner = (jv > jp) & (jv < nj)
        add(q[inner], below[inner], above[inner])
        if jp == 0:
            add(q[jv == 0], above[jv == 0], np.full(int((jv == 0).sum()), -1), 2)
        add(q[jv == nj], below[jv == nj], np.full(int((jv == nj).sum()), -1), 3)
    # diagonal faces inside the prism pairs
    if jp > 0:
        i, j, k = grid((0, ni), (0, jp), (0, nk))
        q = np.stack([nid(i, j, k), nid(i + 1, j, k + 1), nid(i + 1, j + 1, k + 1), nid(i, j + 1, k)], -1).reshape(-1, 4)
        add(q, cA(i, j, k).ravel(), (cA(i, j, k) + 1).ravel())
    # cells
    cells = []
    if jp > 0:
        i, j, k = grid((0, ni), (0, jp), (0, nk))
        a = np.stack([nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j, k + 1),
                      nid(i, j + 1, k), nid(i + 1, j + 1, k), nid(i + 1, j + 1, k + 1)], -1)
        b = np.stack([nid(i, j, k), nid(i + 1, j, k + 1), nid(i, j, k + 1),
                      nid(i, j + 1, k), nid(i + 1, j + 1, k + 1), nid(i, j + 1, k + 1)], -1)
        cells.append((cA(i, j, k).ravel(), a.reshape(-1, 6)))
        cells.append(((cA(i, j, k) + 1).ravel(), b.reshape(-1, 6)))
    if jp < nj:
        i, j, k = grid((0, ni), (jp, nj), (0, nk))
        h = np.stack([nid(i, j, k), nid(i + 1, j, k), nid(i, j + 1, k), nid(i + 1, j + 1, k),
                      nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i, j + 1, k + 1), nid(i + 1, j + 1, k + 1)], -1)
        cells.append((cH(i, j, k).ravel(), h.reshape(-1, 8)))
    ncell = sum(c.size for c, _ in cells)
    cnn = np.zeros(ncell, np.int32)
    for ids, nodes in cells:
        cnn[ids] = nodes.shape[1]
    coff = np.zeros(ncell + 1, np.int64)
    np.cumsum(cnn, out=coff[1:])
    c2n = np.zeros(int(coff[-1]), np.int64)
    cen = np.zeros((ncell, 3))
    for ids, nodes in cells:
        w = nodes.shape[1]
        c2n[(coff[ids][:, None] + np.arange(w)[None, :]).ravel()] = np.sort(nodes, axis=1).ravel()
        cen[ids] = xyz[nodes].mean(axis=1)
    # orient faces left -> right (outward on the boundary), order, flatten
    out_nodes, out_left, out_right, out_side = [], [], [], []
    for nodes, le, re, sd in zip(F, L, R, SIDE):
        if nodes.shape[0] == 0:
            continue
        p = xyz[nodes]
        if nodes.shape[1] == 4:
            nrm = np.cross(p[:, 2] - p[:, 0], p[:, 3] - p[:, 1])
        else:
            nrm = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
        tgt = np.where((re >= 0)[:, None], cen[np.maximum(re, 0)], p.mean(axis=1)) - cen[le]
        flip = np.einsum("ij,ij->i", nrm, tgt) < 0.0
        nodes = nodes.copy()
        nodes[flip] = nodes[flip][:, ::-1]
        out_nodes.append(nodes); out_left.append(le); out_right.append(re); out_side.append(sd)
    left = np.concatenate(out_left)
    right = np.concatenate(out_right)
    side = np.concatenate(out_side)
    nnode = np.concatenate([np.full(n.shape[0], n.shape[1], np.int32) for n in out_nodes])
    # region of each boundary face
    breg = np.full(left.size, -1, np.int64)
    fcen = np.concatenate([xyz[n].mean(axis=1) for n in out_nodes])
    for sidx, name in enumerate(sides):
        m_ = side == sidx
        if not m_.any():
            continue
        r = side_region[name]
        breg[m_] = np.asarray(r(fcen[m_]), np.int64) if callable(r) else r
    bnd = right < 0
    bidx = np.flatnonzero(bnd)
    bidx = bidx[np.lexsort((left[bidx], breg[bidx]))]
    iidx = np.flatnonzero(~bnd)
    iidx = iidx[np.lexsort((right[iidx], left[iidx]))]
    order = np.concatenate([bidx, iidx])
    # flatten face2node in the new order
    offs = np.zeros(nnode.size + 1, np.int64)
    np.cumsum(nnode, out=offs[1:])
    flat = np.concatenate([n.ravel() for n in out_nodes])
    nn_o = nnode[order]
    starts = offs[order]
    idx = np.repeat(starts, nn_o) + (np.arange(int(nn_o.sum())) - np.repeat(np.cumsum(nn_o) - nn_o, nn_o))
    f2n = flat[idx]
    return Mesh(
        x=np.ascontiguousarray(xyz[:, 0]), y=np.ascontiguousarray(xyz[:, 1]), z=np.ascontiguousarray(xyz[:, 2]),
        face_nnode=nn_o.astype(np.int32), face2node=f2n.astype(np.int32),
        left=left[order].astype(np.int32), right=np.where(bnd[order], -1, right[order]).astype(np.int32),
        cell_nnode=cnn, cell2node=c2n.astype(np.int32),
        n_bface=int(bidx.size), bface_region=breg[bidx].astype(np.int32), regions=regions)


def tanh_one_sided(n: int, first: float) -> np.ndarray:
    """n+1 points on [0,1] clustered at 0 with first spacing `first` (tanh law)."""
    if first * n >= 1.0:
        return np.linspace(0.0, 1.0, n + 1)
    eta = np.linspace(0.0, 1.0, n + 1)

    def s(beta):
        return 1.0 + np.tanh(beta * (eta - 1.0)) / np.tanh(beta)

    lo, hi = 1e-6, 50.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if s(mid)[1] > first:
            lo = mid
        else:
            hi = mid
    out = s(0.5 * (lo + hi))
    out[0], out[-1] = 0.0, 1.0
    return out


def channel_bump(nx=64, ny=32, nz=4, thickness=0.10, length=3.0, height=1.0,
                 wall_spacing=0.01, dz=None, lower_region="Wall", upper_region="Wall", prism_layers=0,
                 zone=None) -> Mesh:
    """3-D channel with a circular-arc bump of chord 1 on x in [1,2] of the lower wall.

    x and z are uniform (dz defaults to dx), y is tanh-stretched from the lower
    wall with first spacing wall_spacing*height.  Regions: lower and upper walls
    (solid surface), inlet/outlet (far field), z planes (symmetry).

    zone=(r, n): the r-th of n equal slabs in x of this channel (i in
    [r nx/n, (r+1) nx/n]); a cut side belongs to a fifth region "Interface" of
    type BC_INTERFACE.
    """
    x = np.linspace(0.0, length, nx + 1)
    t = thickness
    r = (0.25 + t * t) / (2.0 * t)
    yw = np.where((x >= 1.0) & (x <= 2.0), np.sqrt(np.maximum(r * r - (x - 1.5) ** 2, 0.0)) - (r - t), 0.0)
    yw = np.maximum(yw, 0.0)
    s = tanh_one_sided(ny, wall_spacing)
    dz = length / nx if dz is None else dz
    zz = np.arange(nz + 1) * dz
    X = np.empty((nx + 1, ny + 1, nz + 1, 3))
    X[..., 0] = x[:, None, None]
    X[..., 1] = (yw[:, None] + (height - yw[:, None]) * s[None, :])[:, :, None]
    X[..., 2] = zz[None, None, :]
    regions = [(BC_SOLID_SURFACE, "LowerWall"), (BC_SOLID_SURFACE, "UpperWall"),
               (BC_FARFIELD, "Farfield"), (BC_SYMMETRY, "Symmetry")]
    side = {"jmin": 0, "jmax": 1, "imin": 2, "imax": 2, "kmin": 3, "kmax": 3}
    if zone is not None:
        r, n = zone
        if nx % n or not 0 <= r < n:
            raise ValueError("zone (r, n) needs 0 <= r < n and n dividing nx")
        w = nx // n
        X = X[r * w:(r + 1) * w + 1]
        if n > 1:
            regions = regions + [(BC_INTERFACE, "Interface")]
            if r > 0:
                side["imin"] = 4
            if r < n - 1:
                side["imax"] = 4
    if prism_layers > 0:
        return _hex_prism_block(X, prism_layers, side, regions)
    return _hex_block(X, side, regions)


def flat_plate(nx=512, ny=192, nz=32, lead=0.33, plate=2.0, height=1.0, width=0.5,
               first_spacing=5.4e-6) -> Mesh:
    """Flat-plate boundary-layer box: x in [-lead, plate], plate (no-slip) on
    x >= 0 of the lower boundary, symmetry on the lead-in, far field on inlet,
    top and outlet, symmetry on the z planes.  x clusters at the leading edge."""
    n_lead = max(2, int(round(nx * lead / (lead + plate) * 0.6)))
    n_plate = nx - n_lead
    xp = plate * tanh_one_sided(n_plate, 0.25 / n_plate)
    xl = -lead * tanh_one_sided(n_lead, (xp[1] - xp[0]) / lead)[::-1]
    x = np.concatenate([xl[:-1], xp])
    y = height * tanh_one_sided(ny, first_spacing / height)
    zz = np.linspace(0.0, width, nz + 1)
    X = np.empty((nx + 1, ny + 1, nz + 1, 3))
    X[..., 0] = x[:, None, None]
    X[..., 1] = y[None, :, None]
    X[..., 2] = zz[None, None, :]
    regions = [(BC_SOLID_SURFACE, "Plate"), (BC_SYMMETRY, "LeadIn"), (BC_FARFIELD, "Farfield"),
               (BC_SYMMETRY, "Symmetry")]

    def lower(fc):
        return np.where(fc[:, 0] > 0.0, 0, 1)

    side = {"jmin": lower, "jmax": 2, "imin": 2, "imax": 2, "kmin": 3, "kmax": 3}
    return _hex_block(X, side, regions)


# ----------------------------------------------------------------------------
# tetrahedral cube
# ----------------------------------------------------------------------------

# Six tetrahedra per hex sharing the main diagonal (local hex nodes: bit0=i, bit1=j, bit2=k).
_HEX_TETS = np.array([[0, 1, 3, 7], [0, 3, 2, 7], [0, 2, 6, 7],
                      [0, 6, 4, 7], [0, 4, 5, 7], [0, 5, 1, 7]], dtype=np.int64)


def tet_cube(n=100, jitter=0.15, seed=0) -> Mesh:
    """Unit cube of n^3 hexes, each split into 6 tetrahedra; interior nodes
    jittered uniformly by +-jitter*h (seeded).  All six sides are far field."""
    rng = np.random.default_rng(seed)
    h = 1.0 / n
    g = np.linspace(0.0, 1.0, n + 1)
    X = np.stack(np.meshgrid(g, g, g, indexing="ij"), axis=-1)  # [i,j,k,3]
    inner = (slice(1, n), slice(1, n), slice(1, n))
    X[inner] += rng.uniform(-jitter * h, jitter * h, size=X[inner].shape)
    nid = np.arange((n + 1) ** 3, dtype=np.int64).reshape((n + 1,) * 3)  # nid[i,j,k] = (i*(n+1)+j)*(n+1)+k
    loc = np.stack([nid[:-1, :-1, :-1], nid[1:, :-1, :-1], nid[:-1, 1:, :-1], nid[1:, 1:, :-1],
                    nid[:-1, :-1, 1:], nid[1:, :-1, 1:], nid[:-1, 1:, 1:], nid[1:, 1:, 1:]], axis=-1)
    loc = loc.transpose(2, 1, 0, 3).reshape(-1, 8)  # hex order: i fastest
    tets = loc[:, _HEX_TETS].reshape(-1, 4)
    xyz = X.reshape(-1, 3)
    return _from_tets(xyz, tets)


def _from_tets(xyz: np.ndarray, tets: np.ndarray) -> Mesh:
    nt = tets.shape[0]
    # Four faces per tet: opposite node d, face (a,b,c).
    lf = np.array([[1, 2, 3, 0], [0, 3, 2, 1], [0, 1, 3, 2], [0, 2, 1, 3]])
    fa = tets[:, lf[:, :3]].reshape(-1, 3)
    opp = tets[:, lf[:, 3]].reshape(-1)
    owner = np.repeat(np.arange(nt, dtype=np.int64), 4)
    # Orient each face outward from its owner.
    p0, p1, p2, pd = xyz[fa[:, 0]], xyz[fa[:, 1]], xyz[fa[:, 2]], xyz[opp]
    nrm = np.cross(p1 - p0, p2 - p0)
    inward = np.einsum("ij,ij->i", nrm, pd - p0) > 0.0
    fa[inward] = fa[inward][:, ::-1]
    key = np.sort(fa, axis=1)
    order = np.lexsort((key[:, 2], key[:, 1], key[:, 0]))
    ks = key[order]
    same = np.all(ks[1:] == ks[:-1], axis=1)
    first = np.ones(ks.shape[0], bool)
    first[1:] = ~same
    grp = np.cumsum(first) - 1
    ngrp = int(grp[-1]) + 1
    cnt = np.bincount(grp, minlength=ngrp)
    # Each group: one (boundary) or two (interior) entries.
    start = np.flatnonzero(first)
    e0 = order[start]
    e1 = np.where(cnt == 2, order[np.minimum(start + 1, order.size - 1)], -1)
    bmask = cnt == 1
    # Interior: left = lower cell index, face oriented outward from left.
    i0, i1 = e0[~bmask], e1[~bmask]
    c0, c1 = owner[i0], owner[i1]
    swap = c0 > c1
    le = np.where(swap, c1, c0)
    re = np.where(swap, c0, c1)
    ent = np.where(swap, i1, i0)
    inodes = fa[ent]
    # Interior faces ordered by (left, right).
    io = np.lexsort((re, le))
    inodes, le, re = inodes[io], le[io], re[io]
    bent = e0[bmask]
    bnodes = fa[bent]
    bleft = owner[bent]
    bo = np.argsort(bleft, kind="stable")
    bnodes, bleft = bnodes[bo], bleft[bo]
    faces = np.concatenate([bnodes, inodes])
    cnodes = np.sort(tets, axis=1)
    return Mesh(
        x=np.ascontiguousarray(xyz[:, 0]), y=np.ascontiguousarray(xyz[:, 1]),
        z=np.ascontiguousarray(xyz[:, 2]),
        face_nnode=np.full(faces.shape[0], 3, np.int32),
        face2node=faces.astype(np.int32).ravel(),
        left=np.concatenate([bleft, le]).astype(np.int32),
        right=np.concatenate([np.full(bleft.size, -1), re]).astype(np.int32),
        cell_nnode=np.full(nt, 4, np.int32), cell2node=cnodes.astype(np.int32).ravel(),
        n_bface=int(bnodes.shape[0]), bface_region=np.zeros(bnodes.shape[0], np.int32),
        regions=[(BC_FARFIELD, "Farfield")])
