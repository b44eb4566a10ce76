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
                 wall_spacing=0.01, dz=None, lower_region="Wall", upper_region="Wall") -> Mesh:
    """3-D channel with a circular-arc bump of chord 1 on x in [1,2] of the lower wall.

    x and z are uniform (dz defaults to dx), y is tanh-stretched from the lower
    wall with first spacing wall_spacing*height.  Regions: lower and upper walls
    (solid surface), inlet/outlet (far field), z planes (symmetry).
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
