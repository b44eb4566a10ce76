"""Partitioned runs of the CUDA solver: one phx context per zone (a part of
phenlei_b200.partition.split), stepped phase by phase with the reference's
interface exchanges between the phases.

The reference runs a partitioned grid as zones joined by INTERFACE faces
(PHENGLEI::INTERFACE, API/Geometry/include/Geo_SimpleBC.h:32).  One outer
iteration of Controller::Relaxation (CFD/Solver/src/Controller.cpp:549-587)
then exchanges, through Controller::CommunicationInterfaceData (:3389):

* the gradients and the limiter after ComputeGradient / ComputeLimiter
  (:1288, :1321);
* the minimum local time step over all zones before the ktmax clamp
  (Controller::GetGlobalMinTimeStep, :720-751);
* dq between the forward and the backward LU-SGS sweep (Controller::LUSGS,
  :1917-1924, CommunicationDQ :2874), for the NS solver and when swapDq is
  set (the reference's parameter file sets it);
* the residual sums (PH_AllReduce);
* q after the update (NSSolver::PostSolve, CFD/NSSolver/src/NSSolver.cpp:139-142);
* with Spalart-Allmaras, nu~ with the eddy viscosity after its update
  (TurbSolverUnstr::UploadInterfaceValue,
  CFD/TurbSolver/src/TurbSolverUnstr.cpp:7130-7145); the SA dq is not
  exchanged between its sweeps (CommunicationDQ serves the NS solver only).
  The reference also exchanges the gradient of nu~; here only a cell's own
  gradient is ever read, so that exchange moves nothing anyone reads and is
  left out.

The set-up follows Region::SwapGeometry (API/Physics/src/Region.cpp:3257-3268):
the interface ghosts take the neighbouring cells' centres and volumes and the
least-squares weights are formed again; the Venkatakrishnan threshold uses
the average cell volume over all zones (Region::ComputeGlobalGridSize,
:2655-2734).

`ZoneSet` drives all zones in one process on one device: the halo rows move
as device-to-device copies.  `DistributedZone` is one rank's zone: the rows
move with torch.distributed point-to-point calls (NCCL between GPUs; with
gloo they are staged through host memory), the time-step minimum and the
residual and force sums with all_reduce.  Every rank calls the same steps.
No kernel of one zone ever waits on another zone: every exchange is a host
step between two launches.
"""
from __future__ import annotations

import numpy as np

from . import partition as P
from .solver import (PHX_HALO_DQ, PHX_HALO_GRADIENT, PHX_HALO_Q, PHX_HALO_TURB, NSSolverUnstruct, PhxError,
                     force_coefficients)


def channel_zone(rank: int, world: int, **channel_kw) -> P.Part:
    """Zone `rank` of `world` equal slabs in x of mesh.channel_bump(**channel_kw),
    built alone (no process holds the whole channel), with its halo plan.  The
    cut sides are interface faces; across a cut, the faces of both zones list
    the same (k, j) rows in the order of their own cells' numbers, so zone r
    sends the cells behind its upper cut in that order and zone r + 1 fills
    the ghosts of its lower cut in that order.  Global cell numbers are
    r n_cell + local number."""
    from . import mesh as M

    m = M.channel_bump(zone=(rank, world), **channel_kw)
    nb, nc = m.n_bface, m.n_cell
    breg = np.asarray(m.bface_region, np.int64)
    itf = np.flatnonzero(breg == len(m.regions) - 1) if world > 1 else np.zeros(0, np.int64)
    foff = m.face_offsets()
    f2n = np.asarray(m.face2node, np.int64)
    xs = np.asarray(m.x)
    fx = np.array([xs[f2n[foff[f]:foff[f + 1]]].mean() for f in itf]) if itf.size else np.zeros(0)
    lo = itf[np.abs(fx - xs.min()) < np.abs(fx - xs.max())]
    hi = np.setdiff1d(itf, lo)
    left = np.asarray(m.left, np.int64)
    halo = P.Halo(neighbors=[], send={}, recv={})
    for q, faces in ((rank - 1, lo), (rank + 1, hi)):
        if 0 <= q < world:
            faces = faces[np.argsort(left[faces], kind="stable")]
            halo.recv[q] = nc + faces
            halo.send[q] = left[faces]
            halo.neighbors.append(q)
    first = int(itf[0]) if itf.size else nb
    if itf.size and not np.array_equal(itf, np.arange(first, nb)):
        raise AssertionError("interface faces are not the last boundary faces")
    return P.Part(rank=rank, mesh=m, cells=rank * nc + np.arange(nc), faces=np.zeros(0, np.int64),
                  flipped=np.zeros(0, bool), nodes=np.zeros(0, np.int64), iface_first=first,
                  n_iface=int(itf.size), halo=halo)


def _wall_of(wall_dist, own=False):
    """Per-part wall distances: the whole mesh's values at the part's cells,
    or (own) the values given, which are already the part's."""
    if wall_dist is None:
        return None
    wd = np.asarray(wall_dist)
    return (lambda p: wd) if own else (lambda p: wd[p.cells])


def _plan(part):
    """Concatenated send cells and receiving boundary faces of a part, and
    per neighbour the (offset, count) of its rows in each list."""
    h = part.halo
    send = [np.asarray(h.send[q], np.int64) for q in h.neighbors]
    recv = [np.asarray(h.recv[q], np.int64) - part.mesh.n_cell for q in h.neighbors]
    soff, roff, s0, r0 = {}, {}, 0, 0
    for q, s, r in zip(h.neighbors, send, recv):
        soff[q] = (s0, len(s))
        roff[q] = (r0, len(r))
        s0 += len(s)
        r0 += len(r)
    cat = lambda a: np.concatenate(a) if a else np.zeros(0, np.int64)  # noqa: E731
    return cat(send), cat(recv), soff, roff


class _Zones:
    """The phase sequence of one partitioned outer iteration over the zones
    this process drives; subclasses move the halo rows and form the sums."""

    FIELDS = (PHX_HALO_Q, PHX_HALO_GRADIENT, PHX_HALO_DQ, PHX_HALO_TURB)

    def _setup(self, mesh, parts, params, precision, wall_of):
        """wall_of(part): the part's wall distances, or None."""
        import torch

        if params.get("gradientName", "ggcell") in ("ggnode", 2):
            raise ValueError("GG-node across zones needs the interpoint exchange; not built")
        self.mesh = mesh
        self.sa = params.get("viscousType", 0) == 3
        self.swap_dq = int(params.get("swapDq", 1)) != 0
        if self.sa and wall_of is None:
            raise ValueError("the SA model needs the wall distance of every cell")
        self.zones = [NSSolverUnstruct(p.mesh, precision=precision, wall_dist=None if wall_of is None else wall_of(p),
                                       **params) for p in self.parts]
        self.plans = [_plan(p) for p in self.parts]
        # zones without interface faces (a single zone) take part in the sums only
        self.linked = [p.n_iface > 0 for p in self.parts]
        for z, (send, recv, _, _), k in zip(self.zones, self.plans, self.linked):
            if k:
                z.set_halo(send, recv)
        dev = torch.device("cuda", torch.cuda.current_device())
        self.bufs = []
        for z, (send, recv, _, _) in zip(self.zones, self.plans):
            b = {}
            for f in self.FIELDS:
                if f == PHX_HALO_TURB and not self.sa:
                    continue
                w = z.halo_row_bytes(f)
                b[f] = (torch.empty(max(len(send), 1) * w, dtype=torch.uint8, device=dev),
                        torch.empty(max(len(recv), 1) * w, dtype=torch.uint8, device=dev), w)
            self.bufs.append(b)
        # SwapGeometry: every interface ghost takes the centre and volume of
        # the neighbouring zone's cell behind it
        cents = self._centres([np.stack([z.geometry(k) for k in ("xcc", "ycc", "zcc", "vol")])
                               for z in self.zones])
        vsum, n = 0.0, 0
        for z in self.zones:
            nc = z.mesh.n_cell
            vsum += float(np.cumsum(z.geometry("vol")[:nc])[-1]) if nc else 0.0   # sequential, as the reference
            n += nc
        vsum, n = self._allsum2(vsum, n)
        for z, (_, recv, _, _), c, k in zip(self.zones, self.plans, cents, self.linked):
            if k:
                z.SwapGeometry(recv, c[0], c[1], c[2], c[3], vsum / n)
        self.n_cell_total = n
        self._exchange_state()

    # -- exchanges ------------------------------------------------------------
    def _exchange(self, field):
        for z, b, k in zip(self.zones, self.bufs, self.linked):
            if k:
                z.halo_pack(field, b[field][0].data_ptr())
        self._move(field)
        for z, b, k in zip(self.zones, self.bufs, self.linked):
            if k:
                z.halo_unpack(field, b[field][1].data_ptr())

    def _exchange_state(self):
        """The interface data of the PostSolve steps: q, and with SA nu~ and the
        eddy viscosity."""
        self._exchange(PHX_HALO_Q)
        if self.sa:
            self._exchange(PHX_HALO_TURB)

    # -- state ----------------------------------------------------------------
    def set_state(self, q_cells, qt_cells=None):
        """The global cell state [5][n_cell] (global cell numbers), and nu~."""
        q_cells = np.asarray(q_cells)
        for part, z in zip(self.parts, self.zones):
            z.set_q_cells(q_cells[:, part.cells])
            if qt_cells is not None:
                z.set_qt_cells(np.asarray(qt_cells)[part.cells])
        self._exchange_state()

    # -- one outer iteration -----------------------------------------------------
    def iterate(self, nsteps: int = 1, timer: dict | None = None) -> np.ndarray:
        """`nsteps` outer iterations; returns the global residual monitor
        sqrt(sum res_rho^2 / nCell) of each.  With `timer` (a dict), CUDA
        events bracket every phase's kernels on the current stream, the
        exchanges between them left out: timer[phase] lists (start, end)
        pairs."""
        hist = []
        zs = self.zones

        def phase(name, fn):
            if timer is None:
                for z in zs:
                    fn(z)
                return
            import torch

            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for z in zs:
                fn(z)
            b.record()
            timer.setdefault(name, []).append((a, b))

        for _ in range(nsteps):
            for z in zs:
                z.step = z.step + 1   # Simulation::UpdateOuterIterationStep
            phase("boundary", lambda z: z.Boundary())
            phase("gradient_limiter", lambda z: z.ComputeGradientAndLimiter())
            self._exchange(PHX_HALO_GRADIENT)
            phase("residual", lambda z: z.UpdateResiduals())
            mindt = self._allmin(min(z.min_timestep() for z in zs))
            for z in zs:
                z.set_min_timestep(mindt)
            phase("lusgs", lambda z: z.LUSGSForward())
            if self.swap_dq:
                self._exchange(PHX_HALO_DQ)
            phase("lusgs", lambda z: z.LUSGSBackward())
            s = 0.0
            for z in zs:
                r = z.GetResidual()[0]
                s += r * r * z.mesh.n_cell
            s = self._allsum(s)
            h = float(np.sqrt(s / self.n_cell_total))
            phase("update", lambda z: z.UpdateFlowField())
            self._exchange(PHX_HALO_Q)
            if self.sa:
                phase("sa_residual", lambda z: z.TurbUpdateResiduals())
                phase("sa_lusgs", lambda z: z.TurbLUSGSForward())
                phase("sa_lusgs", lambda z: z.TurbLUSGSBackward())
                phase("sa_update", lambda z: z.TurbUpdateFlowField())
                self._exchange(PHX_HALO_TURB)
            for z in zs:
                z.status()
            if not np.isfinite(h):
                raise PhxError("residual is not finite (divergence): PHX_ERR_NUMERIC")
            hist.append(h)
        return np.array(hist)

    def forces(self) -> np.ndarray:
        """The wall force sums of AirForceCoefParts over all zones."""
        from .solver import lib

        tot = np.zeros(16)
        for z in self.zones:
            out = np.zeros(16)
            z._check(lib().phx_forces(z.h, out.ctypes.data), "phx_forces")
            tot += out
        return self._allsum_vec(tot)

    def AirForceCoef(self, reference_area: float = 1.0) -> dict:
        p = self.zones[0].params
        return force_coefficients(self.forces(), p.attackd, p.angleSlide, reference_area)

    # -- restart ----------------------------------------------------------------
    def DumpRestart(self, prefix: str):
        """One restart file per zone this process drives, `prefix.zone<i>`
        (i the zone's part number), as the reference writes one group per zone
        (NSSolverUnstruct::DumpRestartH5, CFD/NSSolver/src/NSSolverUnstruct.cpp:1247)."""
        for part, z in zip(self.parts, self.zones):
            z.DumpRestart(f"{prefix}.zone{part.rank}")

    def ReadRestart(self, prefix: str):
        """Continues from DumpRestart's files of the same partition; the
        interface ghosts are refreshed from the neighbours as after an update."""
        for part, z in zip(self.parts, self.zones):
            z.ReadRestart(f"{prefix}.zone{part.rank}")
        steps = {z.step for z in self.zones}
        if len(steps) != 1:
            raise PhxError("the zones' restart files hold different steps: PHX_ERR_ARG")
        self._exchange_state()

    def close(self):
        for z in self.zones:
            z.close()


class ZoneSet(_Zones):
    """All zones of a partitioned grid in this process, on the current device."""

    def __init__(self, mesh, params: dict, nparts: int = 2, owner=None, wall_dist=None, precision="fp64",
                 parts=None):
        """The parts of `mesh` (slabs, or the cell-to-part map `owner`), or the
        parts given (e.g. phenlei_b200.fts.zone_parts of a grid file's zones;
        `mesh` is then None); wall_dist in global cell numbers."""
        if parts is None:
            self.owner = P.slab_owner(mesh, nparts) if owner is None else np.asarray(owner, np.int32)
            parts = P.split(mesh, self.owner)
        self.parts = parts
        self._setup(mesh, self.parts, params, precision, _wall_of(wall_dist))

    def _centres(self, cc):
        out = []
        for p, part in enumerate(self.parts):
            _, recv, _, roff = self.plans[p]
            c = np.zeros((4, len(recv)))
            for q in part.halo.neighbors:
                o, n = roff[q]
                c[:, o:o + n] = cc[q][:, np.asarray(self.parts[q].halo.send[p], np.int64)]
            out.append(c)
        return out

    def _move(self, field):
        for p, part in enumerate(self.parts):
            dst = self.bufs[p][field][1]
            w = self.bufs[p][field][2]
            _, _, _, roff = self.plans[p]
            for q in part.halo.neighbors:
                so, sn = self.plans[q][2][p]
                ro, rn = roff[q]
                dst[ro * w:(ro + rn) * w].copy_(self.bufs[q][field][0][so * w:(so + sn) * w])

    def _allmin(self, v):
        return v

    def _allsum(self, v):
        return v

    def _allsum2(self, a, b):
        return a, b

    def _allsum_vec(self, v):
        return v

    def gather(self, which) -> np.ndarray:
        """A per-cell field (solver.PHX_* selector) of every zone in global cell order."""
        first = self.zones[0].get(which)
        shape = first.shape[:-1]
        out = np.zeros(shape + (self.n_cell_total,))
        for part, z in zip(self.parts, self.zones):
            out[..., part.cells] = z.get(which)[..., : z.mesh.n_cell]
        return out


class DistributedZone(_Zones):
    """This rank's zone of a partitioned grid (rank r of the default
    torch.distributed group takes part r).  Every rank builds the same
    partition and calls the same steps."""

    def __init__(self, mesh, params: dict, owner=None, wall_dist=None, precision="fp64", part=None):
        """`mesh` is the whole grid, split here; or `part` is this rank's zone,
        built alone (channel_zone), with `wall_dist` then its own cells'."""
        import torch.distributed as dist

        self.rank, self.world = dist.get_rank(), dist.get_world_size()
        self._nccl = dist.get_backend() == "nccl"
        if part is not None:
            self.parts = [part]
            self._setup(None, self.parts, params, precision, _wall_of(wall_dist, own=True))
            return
        self.owner = P.slab_owner(mesh, self.world) if owner is None else np.asarray(owner, np.int32)
        parts = P.split(mesh, self.owner)
        if len(parts) != self.world:
            raise ValueError("one part per rank")
        self.parts = [parts[self.rank]]
        self._setup(mesh, self.parts, params, precision, _wall_of(wall_dist))

    @property
    def part(self):
        return self.parts[0]

    def _p2p(self, bufs_out, bufs_in):
        """One send and one receive per neighbour, posted together."""
        import torch
        import torch.distributed as dist

        h = self.part.halo
        if not h.neighbors:
            return
        ops, staged = [], []
        for q in h.neighbors:
            out, inb = bufs_out[q], bufs_in[q]
            if not self._nccl:   # gloo moves host tensors
                out = out.cpu()
                staged.append((inb, torch.empty(inb.shape, dtype=inb.dtype)))
                inb = staged[-1][1]
            ops.append(dist.P2POp(dist.isend, out, q))
            ops.append(dist.P2POp(dist.irecv, inb, q))
        for r in dist.batch_isend_irecv(ops):
            r.wait()
        for dev, host in staged:
            dev.copy_(host)

    def _centres(self, cc):
        import torch

        send, recv, soff, roff = self.plans[0]
        mine = torch.as_tensor(np.ascontiguousarray(cc[0][:, send].T))
        h = self.part.halo
        outs = {q: mine[soff[q][0]:soff[q][0] + soff[q][1]].contiguous() for q in h.neighbors}
        ins = {q: torch.empty((roff[q][1], 4), dtype=torch.float64) for q in h.neighbors}
        if self._nccl:
            outs = {q: t.cuda() for q, t in outs.items()}
            ins = {q: t.cuda() for q, t in ins.items()}
        self._p2p(outs, ins)
        c = np.zeros((4, len(recv)))
        for q in h.neighbors:
            o, n = roff[q]
            c[:, o:o + n] = ins[q].cpu().numpy().T
        return [c]

    def _move(self, field):
        send_buf, recv_buf, w = self.bufs[0][field]
        _, _, soff, roff = self.plans[0]
        h = self.part.halo
        outs = {q: send_buf[soff[q][0] * w:(soff[q][0] + soff[q][1]) * w] for q in h.neighbors}
        ins = {q: recv_buf[roff[q][0] * w:(roff[q][0] + roff[q][1]) * w] for q in h.neighbors}
        if self._nccl:
            import torch

            torch.cuda.current_stream().synchronize()   # the pack kernel ran on the context's stream
        self._p2p(outs, ins)

    def _reduce(self, vals, op):
        import torch
        import torch.distributed as dist

        t = torch.tensor(vals, dtype=torch.float64)
        if self._nccl:
            t = t.cuda()
        dist.all_reduce(t, op=op)
        return t.cpu().numpy()

    def _allmin(self, v):
        import torch.distributed as dist

        return float(self._reduce([v], dist.ReduceOp.MIN)[0])

    def _allsum(self, v):
        import torch.distributed as dist

        return float(self._reduce([v], dist.ReduceOp.SUM)[0])

    def _allsum2(self, a, b):
        import torch.distributed as dist

        r = self._reduce([a, float(b)], dist.ReduceOp.SUM)
        return float(r[0]), int(round(float(r[1])))

    def _allsum_vec(self, v):
        import torch.distributed as dist

        return self._reduce(list(v), dist.ReduceOp.SUM)

    def local_cells(self):
        return self.part.cells
