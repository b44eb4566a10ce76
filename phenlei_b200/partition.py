"""Domain decomposition for one process per GPU: cell partitions, the
interface faces between them, and the halo exchange of interface ghosts.

The reference runs a partitioned grid as zones whose cut faces are boundary
faces of type INTERFACE (PHENGLEI::INTERFACE = -1,
API/Geometry/include/Geo_SimpleBC.h:32).  The first ghost layer of an
interface face holds the neighbouring zone's cell across that face
(UploadInterfaceValue / DownloadInterfaceValue,
API/Geometry/src/Geo_UnstructGrid.cpp:10806-10990), and the solver refreshes
those ghosts at fixed points of each iteration:

* q and T after the update (NSSolver::PostSolve, CFD/NSSolver/src/NSSolver.cpp:139-142);
* the gradients after ComputeGradient (Controller.cpp:1288);
* the limiter after ComputeLimiter (Controller.cpp:1321);
* dq between the forward and backward LU-SGS sweeps (Controller.cpp:1917-1924).

Here a part is a self-contained Mesh.  Its interface faces form one extra
boundary region, typed BC_INTERFACE.  Each interface face is oriented out of
the part's own cell: a face whose global left cell lies in another part is
flipped.  `Halo` lists, for every neighbouring part, the local cells to send
and the ghost slots (n_cell + boundary face) to fill, in matching order.
`exchange` moves those values with torch.distributed point-to-point calls:
gloo on the host, NCCL between GPUs.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .mesh import BC_INTERFACE, Mesh   # noqa: F401  (BC_INTERFACE: PHENGLEI::INTERFACE)


@dataclass
class Halo:
    neighbors: list      # neighbouring parts, ascending
    send: dict           # part q -> local cells whose values q receives, in q's receive order
    recv: dict           # part q -> local ghost slots (n_cell + boundary face) filled from q

    def n_send(self) -> int:
        return int(sum(len(v) for v in self.send.values()))

    def index_tensors(self, device):
        """{q: (send, recv)} as int64 tensors on `device`, made once per device."""
        import torch

        cache = self.__dict__.setdefault("_index", {})
        key = str(device)
        if key not in cache:
            cache[key] = {q: (torch.as_tensor(self.send[q], dtype=torch.int64, device=device),
                              torch.as_tensor(self.recv[q], dtype=torch.int64, device=device))
                          for q in self.neighbors}
        return cache[key]


@dataclass
class Part:
    rank: int
    mesh: Mesh
    cells: np.ndarray        # local cell -> global cell
    faces: np.ndarray        # local face -> global face
    flipped: np.ndarray      # bool per local face: orientation reversed against the global face
    nodes: np.ndarray        # local node -> global node
    iface_first: int         # local index of the first interface face (they are contiguous)
    n_iface: int
    halo: Halo


def cell_centroids(m: Mesh) -> np.ndarray:
    """Mean of each cell's nodes, [n_cell, 3] (for ordering cells only)."""
    off = np.zeros(m.n_cell + 1, dtype=np.int64)
    np.cumsum(m.cell_nnode, out=off[1:])
    xyz = np.stack([m.x, m.y, m.z], axis=1)[np.asarray(m.cell2node, np.int64)]
    sums = np.add.reduceat(xyz, off[:-1], axis=0)
    return sums / np.asarray(m.cell_nnode, np.float64)[:, None]


def slab_owner(m: Mesh, nparts: int, axis: int | None = None) -> np.ndarray:
    """Part of every cell: equal-count slabs along `axis` (default: the axis
    the mesh is longest in), cells ordered by centroid then by index."""
    if nparts < 1:
        raise ValueError("nparts must be >= 1")
    c = cell_centroids(m)
    if axis is None:
        axis = int(np.argmax(c.max(axis=0) - c.min(axis=0)))
    order = np.lexsort((np.arange(m.n_cell), c[:, axis]))
    owner = np.empty(m.n_cell, dtype=np.int32)
    owner[order] = (np.arange(m.n_cell, dtype=np.int64) * nparts // m.n_cell).astype(np.int32)
    return owner


def rcb_owner(m: Mesh, nparts: int) -> np.ndarray:
    """Part of every cell by recursive coordinate bisection of the cell
    centroids: a set of cells bound for k parts is cut across its longest
    extent at the floor(k/2)/k quantile (ties broken by cell number), and the
    two sides go on with floor(k/2) and k - floor(k/2) parts.  Part sizes
    differ by at most one cell per level of cuts, and the cuts follow the
    mesh's shape instead of one axis, so for many parts the interface faces
    (the halo volume) stay fewer than with slabs."""
    if nparts < 1:
        raise ValueError("nparts must be >= 1")
    c = cell_centroids(m)
    owner = np.empty(m.n_cell, dtype=np.int32)
    stack = [(np.arange(m.n_cell), 0, nparts)]
    while stack:
        cells, first, k = stack.pop()
        if k == 1 or cells.size == 0:
            owner[cells] = first
            continue
        pts = c[cells]
        axis = int(np.argmax(pts.max(axis=0) - pts.min(axis=0)))
        order = cells[np.lexsort((cells, pts[:, axis]))]
        kl = k // 2
        nl = (cells.size * kl) // k
        stack.append((order[:nl], first, kl))
        stack.append((order[nl:], first + kl, k - kl))
    return owner


def _ranks(counts: np.ndarray) -> np.ndarray:
    """0, 1, .., n-1 for each run length n in `counts`, concatenated."""
    counts = np.asarray(counts, np.int64)
    if counts.size == 0:
        return np.zeros(0, np.int64)
    starts = np.repeat(np.cumsum(counts) - counts, counts)
    return np.arange(int(counts.sum()), dtype=np.int64) - starts


def split(m: Mesh, owner: np.ndarray) -> list:
    """The parts of `m` for the cell-to-part map `owner` (values 0..P-1)."""
    owner = np.asarray(owner, np.int32)
    if owner.shape != (m.n_cell,) or owner.min() < 0:
        raise ValueError("owner must give a part >= 0 for every cell")
    nparts = int(owner.max()) + 1
    nb = m.n_bface
    left = np.asarray(m.left, np.int64)
    right = np.asarray(m.right, np.int64)
    foff = m.face_offsets()
    coff = np.zeros(m.n_cell + 1, dtype=np.int64)
    np.cumsum(m.cell_nnode, out=coff[1:])
    fidx = np.arange(m.n_face)
    interior = fidx >= nb
    lp = owner[left]
    rp = np.where(interior, owner[np.where(interior, right, 0)], -1)
    cut = interior & (lp != rp)
    # local cell numbering of every global cell inside its own part
    local_of = np.empty(m.n_cell, dtype=np.int64)
    for p in range(nparts):
        cells = np.flatnonzero(owner == p)
        local_of[cells] = np.arange(cells.size)
    parts = []
    for p in range(nparts):
        cells = np.flatnonzero(owner == p)
        bfaces = np.flatnonzero((fidx < nb) & (lp == p))
        # interface faces in global face order; flipped where the global left cell is elsewhere
        ifaces = np.flatnonzero(cut & ((lp == p) | (rp == p)))
        iflip = rp[ifaces] == p
        ifaces_in = np.flatnonzero(interior & ~cut & (lp == p))
        faces = np.concatenate([bfaces, ifaces, ifaces_in])
        flipped = np.concatenate([np.zeros(bfaces.size, bool), iflip, np.zeros(ifaces_in.size, bool)])
        own = np.where(flipped, right[faces], left[faces])
        other = np.where(flipped, left[faces], right[faces])
        nbl = bfaces.size + ifaces.size
        # face nodes: a flipped face keeps its first node and reverses the rest
        fnn = np.asarray(m.face_nnode, np.int64)[faces]
        j = _ranks(fnn)                                   # position of each entry within its face
        nn = np.repeat(fnn, fnn)
        j = np.where(np.repeat(flipped, fnn) & (j > 0), nn - j, j)
        f2n = np.asarray(m.face2node)[np.repeat(foff[faces], fnn) + j]
        cnn = np.asarray(m.cell_nnode, np.int64)[cells]
        c2n = np.asarray(m.cell2node)[np.repeat(coff[cells], cnn) + _ranks(cnn)]
        nodes = np.unique(np.concatenate([f2n, c2n]))
        node_local = np.full(m.n_node, -1, dtype=np.int64)
        node_local[nodes] = np.arange(nodes.size)
        regions = list(m.regions)
        bregion = np.asarray(m.bface_region, np.int32)[bfaces]
        if ifaces.size:
            regions.append((BC_INTERFACE, "Interface"))
            bregion = np.concatenate([bregion, np.full(ifaces.size, len(regions) - 1, np.int32)])
        lright = np.full(faces.size, -1, dtype=np.int64)
        lright[nbl:] = local_of[other[nbl:]]
        pm = Mesh(x=m.x[nodes].copy(), y=m.y[nodes].copy(), z=m.z[nodes].copy(),
                  face_nnode=fnn.astype(np.int32), face2node=node_local[f2n].astype(np.int32),
                  left=local_of[own].astype(np.int32), right=lright.astype(np.int32),
                  cell_nnode=np.asarray(m.cell_nnode, np.int32)[cells].copy(),
                  cell2node=node_local[c2n].astype(np.int32), n_bface=int(nbl), bface_region=bregion,
                  regions=regions)
        parts.append(Part(rank=p, mesh=pm, cells=cells, faces=faces, flipped=flipped, nodes=nodes,
                          iface_first=int(bfaces.size), n_iface=int(ifaces.size),
                          halo=Halo(neighbors=[], send={}, recv={})))
    # halo maps: part p's interface ghost k is filled from the neighbour's cell across the face
    for p, part in enumerate(parts):
        g = part.faces[part.iface_first:part.iface_first + part.n_iface]
        nbr_cell = np.where(part.flipped[part.iface_first:part.iface_first + part.n_iface], left[g], right[g])
        nbr_part = owner[nbr_cell]
        slots = part.mesh.n_cell + part.iface_first + np.arange(part.n_iface)
        for q in np.unique(nbr_part):
            sel = nbr_part == q
            part.halo.recv[int(q)] = slots[sel].astype(np.int64)
            parts[int(q)].halo.send[p] = local_of[nbr_cell[sel]].astype(np.int64)
    for part in parts:
        part.halo.neighbors = sorted(part.halo.recv)
        if sorted(part.halo.send) != part.halo.neighbors:
            raise AssertionError("halo send and receive partners differ")
    return parts


def exchange(halo: Halo, field, group=None) -> None:
    """Fill the interface ghosts of `field` ([nvar, n_total] torch tensor, this
    rank's part) from the neighbouring ranks, which call this in the same
    step.  One send and one receive per neighbour, posted together
    (torch.distributed.batch_isend_irecv): gloo for host tensors, NCCL for
    device tensors.  Part q is the rank q of `group` (default: the default
    group); the peers are passed to torch.distributed as global ranks."""
    import torch
    import torch.distributed as dist

    if not halo.neighbors:
        return
    ops, bufs = [], []
    index = halo.index_tensors(field.device)
    for q in halo.neighbors:
        peer = q if group is None else dist.get_global_rank(group, q)
        out = field.index_select(1, index[q][0]).contiguous()
        inb = torch.empty((field.shape[0], len(halo.recv[q])), dtype=field.dtype, device=field.device)
        ops.append(dist.P2POp(dist.isend, out, peer, group))
        ops.append(dist.P2POp(dist.irecv, inb, peer, group))
        bufs.append((q, inb, out))
    for r in dist.batch_isend_irecv(ops):
        r.wait()
    for q, inb, _ in bufs:
        field[:, index[q][1]] = inb
