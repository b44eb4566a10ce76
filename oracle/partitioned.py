"""The oracle on a partitioned grid (test infrastructure, like the rest of
oracle/): one Oracle per part of phenlei_b200.partition.split, stepped phase
by phase with the reference's interface exchanges between the phases.

The reference runs a partitioned grid as zones joined by INTERFACE faces
(PHENGLEI::INTERFACE, API/Geometry/include/Geo_SimpleBC.h:32), and fills
their ghosts from the neighbouring zone at these points:

* set-up: the ghosts' cell centres and volumes, then the LSQ weights
  (Region::SwapGeometry, API/Physics/src/Region.cpp:3257-3268), and one
  average cell volume over all zones (Region::ComputeGlobalGridSize, :2655-2734);
* after the update and at initialisation: q (NSSolver::PostSolve,
  CFD/NSSolver/src/NSSolver.cpp:139-142);
* after the gradient: the primitive and temperature gradients
  (Controller::ComputeGradient, CFD/Solver/src/Controller.cpp:1288);
* after the limiter: limit2D (Controller.cpp:1321);
* between the forward and the backward LU-SGS sweep: dq (Controller.cpp:1917-1924),
  for the NS solver only and when swapDq is set (Controller::CommunicationDQ,
  :2874-2886; the reference's parameter file sets it).

The residual norm is a sum over all zones (PH_AllReduce).  The exchanges here
are plain array copies between the in-process parts; phenlei_b200.partition.exchange
moves the same values between ranks.

With Spalart-Allmaras the turbulence step exchanges the gradient of nu~ and,
in its PostSolve, q_turb with vist (TurbSolverUnstr::UploadInterfaceValue,
:7130-7145).  Its dq is not exchanged between the sweeps (CommunicationDQ
returns for every solver but the NS one), so an interface ghost's SA dq stays
its ghost residual, zero.  The wall distance of every part is given.

The ktmax clamp of the local time step takes the minimum over all zones
(Controller::GetGlobalMinTimeStep, Controller.cpp:720-751).

Covered: NS, inviscid, laminar and SA, GG-cell or LSQ gradient, one LU-SGS
sweep, no initialisation phase.  Not covered: GG-node (its node values need
the interpoint exchange, Controller::PostSolve :5063-5205).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from phenlei_b200 import partition as P

from .oracle import Oracle, _p, lib


class PartitionedOracle:
    def __init__(self, mesh, params: dict, nparts: int = 2, owner=None, wall_dist=None, parts=None):
        """The parts of `mesh` (slabs, or the cell-to-part map `owner`), or the
        parts given (e.g. phenlei_b200.fts.zone_parts of a grid file's zones;
        `mesh` is then None); wall_dist in global cell numbers."""
        if params.get("gradientName", "ggcell") == "ggnode":
            raise ValueError("GG-node across parts needs the interpoint exchange; not restated")
        if params.get("viscousType", 0) not in (0, 1, 3):
            raise ValueError("inviscid, laminar and SA runs only")
        self.sa = params.get("viscousType", 0) == 3
        if self.sa and wall_dist is None:
            raise ValueError("the SA model needs the wall distance of every cell")
        if params.get("flowInitStep", 100) != 0 or params.get("uns_limiter_name", "vencat") == "1st":
            raise ValueError("second order from the first step only (flowInitStep = 0)")
        if params.get("nLUSGSSweeps", 1) != 1:
            raise ValueError("one LU-SGS sweep only")
        self.mesh = mesh
        if parts is None:
            self.owner = P.slab_owner(mesh, nparts) if owner is None else np.asarray(owner, np.int32)
            parts = P.split(mesh, self.owner)
        self.n_cell_total = int(sum(p.mesh.n_cell for p in parts))
        self.parts = self._local(parts)
        self.o = [Oracle(p.mesh, params, wall_dist=None if wall_dist is None else np.asarray(wall_dist)[p.cells])
                  for p in self.parts]
        self.viscous = params.get("viscousType", 0) > 0
        self.swap_dq = int(params.get("swapDq", 1)) != 0
        self.step = 0
        # SwapGeometry: the interface ghosts take the neighbouring cells' centres
        # and volumes (UnstructGrid::TranslateCellCenter,
        # API/Geometry/src/Geo_UnstructGrid.cpp:4500-4541), and the least-squares
        # weights are formed again from them
        for k in ("xcc", "ycc", "zcc", "vol"):
            self._exchange(lambda o, k=k: o.geo[k])
        for o in self.o:
            lib().ox_lsq_weights(C.byref(o.g), C.byref(o.m))
        # Region::ComputeGlobalGridSize (API/Physics/src/Region.cpp:2655-2734): one
        # average cell volume for all zones, each zone's sum added across the
        # ranks (PH_AllReduce); the Venkatakrishnan limiter scales with it
        tot, n = 0.0, 0
        for o in self.o:
            nc = o.mesh.n_cell
            tot += float(np.cumsum(o.geo["vol"][:nc])[-1]) if nc else 0.0
            n += nc
        tot, n = self._allsum(tot, n)
        for o in self.o:
            o.m.avg_vol = tot / n
        self._exchange_state()

    def _exchange_state(self) -> None:
        """The interface data of NSSolver / TurbSolver PostSolve: q, and with SA
        q_turb and vist."""
        self._exchange(lambda o: o.q)
        if self.sa:
            self._exchange(lambda o: o.w_arrays["qt"])
            self._exchange(lambda o: o.w_arrays["vist"])

    def _local(self, parts):
        """The parts this process steps (all of them in process)."""
        return parts

    def _allsum(self, s: float, n: int):
        """The sums over all parts (PH_AllReduce); in process they are complete."""
        return s, n

    def _allmin(self, v: float) -> float:
        """The minimum over all parts (PH_CompareMaxMin)."""
        return v

    def _exchange(self, get) -> None:
        """Fill every part's interface ghosts of the array `get(oracle)`
        ([..., n_total]) from the neighbouring parts' cells."""
        arrs = [get(o) for o in self.o]
        for p, part in enumerate(self.parts):
            for q in part.halo.neighbors:
                arrs[p][..., part.halo.recv[q]] = arrs[q][..., self.parts[q].halo.send[p]]

    def set_state(self, q_cells: np.ndarray, qt_cells=None) -> None:
        """Global cell state [5][n_cell] (reference numbering), and nu~ [n_cell]."""
        for part, o in zip(self.parts, self.o):
            o.set_state(q_cells[:, part.cells], None if qt_cells is None else np.asarray(qt_cells)[part.cells])
        self._exchange_state()

    def gather(self, name_or_array) -> np.ndarray:
        """A per-cell work array (or 'q') of every part, in global cell order."""
        first = self._cells(self.o[0], name_or_array)
        out = np.zeros(first.shape[:-1] + (self.n_cell_total,))
        for part, o in zip(self.parts, self.o):
            out[..., part.cells] = self._cells(o, name_or_array)
        return out

    @staticmethod
    def _cells(o, name):
        a = o.q if name == "q" else o.work(name)
        return a[..., : o.mesh.n_cell]

    def iterate(self, nsteps: int = 1) -> np.ndarray:
        """`nsteps` outer iterations (ox_ns_iteration phase by phase); returns
        the global residual norms."""
        L = lib()
        hist = []
        for _ in range(nsteps):
            self.step += 1
            for o in self.o:
                w = o.w_arrays
                g, m, p = C.byref(o.g), C.byref(o.m), C.byref(o.p)
                L.ox_gamma_temperature(g, p, _p(o.q), _p(w["gama"]), _p(w["t"]))
                L.ox_ns_boundary(g, m, p, _p(o.q), _p(w["gama"]))
                L.ox_gamma_temperature(g, p, _p(o.q), _p(w["gama"]), _p(w["t"]))
                if self.viscous:
                    L.ox_viscosity(g, p, _p(w["t"]), _p(w["visl"]), _p(w["vist"]))
                nt = o.nt
                for k in range(5):
                    off = k * nt * 8
                    L.ox_gradient(g, m, p, C.cast(C.c_void_p(o.q.ctypes.data + off), C.POINTER(C.c_double)),
                                  *[C.cast(C.c_void_p(w[d].ctypes.data + off), C.POINTER(C.c_double))
                                    for d in ("dqdx", "dqdy", "dqdz")])
                if self.viscous:
                    L.ox_gradient(g, m, p, _p(w["t"]), _p(w["dtdx"]), _p(w["dtdy"]), _p(w["dtdz"]))
            for d in ("dqdx", "dqdy", "dqdz") + (("dtdx", "dtdy", "dtdz") if self.viscous else ()):
                self._exchange(lambda o, d=d: o.w_arrays[d])
            for o in self.o:
                w = o.w_arrays
                L.ox_limiter(C.byref(o.g), C.byref(o.m), C.byref(o.p), _p(o.q), _p(w["dqdx"]), _p(w["dqdy"]),
                             _p(w["dqdz"]), _p(w["limit"]))
            self._exchange(lambda o: o.w_arrays["limit"])
            for o in self.o:
                w = o.w_arrays
                g, m, p = C.byref(o.g), C.byref(o.m), C.byref(o.p)
                w["res"][:] = 0.0
                L.ox_inviscid_flux(g, m, p, _p(o.q), _p(w["gama"]), _p(w["dqdx"]), _p(w["dqdy"]), _p(w["dqdz"]),
                                   _p(w["limit"]), _p(w["res"]))
                if self.viscous:
                    L.ox_viscous_flux(g, m, p, _p(o.q), _p(w["t"]), _p(w["visl"]), _p(w["vist"]), _p(w["dqdx"]),
                                      _p(w["dqdy"]), _p(w["dqdz"]), _p(w["dtdx"]), _p(w["dtdy"]), _p(w["dtdz"]),
                                      _p(w["res"]))
                L.ox_spectrum(g, m, p, _p(o.q), _p(w["gama"]), _p(w["visl"]), _p(w["vist"]), _p(w["inv_spec"]),
                              _p(w["vis_spec"]))
                o._mindt = L.ox_timestep_raw(g, m, p, self.step, _p(o.q), _p(w["inv_spec"]), _p(w["vis_spec"]),
                                             _p(w["dt"]))
            mindt = self._allmin(min(o._mindt for o in self.o))
            for o in self.o:
                w = o.w_arrays
                g, m, p = C.byref(o.g), C.byref(o.m), C.byref(o.p)
                L.ox_timestep_clamp(g, m, p, C.c_double(mindt), _p(w["dt"]))
                o._dflux = np.zeros((5, o.nt))
                L.ox_lusgs_forward(g, m, p, _p(o.q), _p(w["gama"]), _p(w["visl"]), _p(w["vist"]), _p(w["res"]),
                                   _p(w["dt"]), _p(w["inv_spec"]), _p(w["vis_spec"]), _p(w["dq"]), _p(o._dflux))
            if self.swap_dq:
                self._exchange(lambda o: o.w_arrays["dq"])
            s, n = 0.0, 0
            for o in self.o:
                w = o.w_arrays
                g, m, p = C.byref(o.g), C.byref(o.m), C.byref(o.p)
                L.ox_lusgs_backward(g, m, p, _p(o.q), _p(w["gama"]), _p(w["visl"]), _p(w["vist"]), _p(w["res"]),
                                    _p(w["dt"]), _p(w["inv_spec"]), _p(w["vis_spec"]), _p(w["dq"]), _p(o._dflux))
                L.ox_update(g, m, p, _p(o.q), _p(w["gama"]), _p(w["dq"]))
                nc = o.mesh.n_cell
                r = w["res"][0, :nc]
                s += float(np.cumsum(r * r)[-1]) if nc else 0.0   # sequential, as ox_residual_norm sums
                n += nc
            s, n = self._allsum(s, n)
            hist.append(np.sqrt(s / n))
            # PostSolve: interface ghosts of the updated state, then the boundary
            self._exchange(lambda o: o.q)
            for o in self.o:
                L.ox_ns_boundary(C.byref(o.g), C.byref(o.m), C.byref(o.p), _p(o.q), _p(o.w_arrays["gama"]))
            if self.sa:
                self._sa_step()
        return np.array(hist)

    def _sa_step(self) -> None:
        """ox_sa_step phase by phase, with the turbulence solver's exchanges."""
        L = lib()
        args = [(C.byref(o.g), C.byref(o.m), C.byref(o.p), _p(o.q), C.byref(o.w)) for o in self.o]
        for a in args:
            L.ox_sa_gradient_phase(*a)
        for d in ("dntx", "dnty", "dntz"):
            self._exchange(lambda o, d=d: o.w_arrays[d])
        for o, a in zip(self.o, args):
            L.ox_sa_residual_phase(*a)
            o._dfl = np.zeros(o.nt)
            L.ox_sa_lusgs_forward(a[0], a[1], a[4], _p(o._dfl))
        for o, a in zip(self.o, args):
            L.ox_sa_lusgs_backward(a[0], a[1], a[4], _p(o._dfl))
        self._exchange(lambda o: o.w_arrays["qt"])
        self._exchange(lambda o: o.w_arrays["vist"])
        for a in args:
            L.ox_sa_post_phase(*a)


class DistributedOracle(PartitionedOracle):
    """One rank's part of a PartitionedOracle run across processes: the same
    phases, with the halos moved by phenlei_b200.partition.exchange over the
    default torch.distributed group (gloo) and the global sums by all_reduce.
    Every rank builds the same partition and calls the same steps."""

    def __init__(self, mesh, params: dict, rank: int, world: int, owner=None, wall_dist=None, parts=None):
        self._rank = rank
        self._world = world
        super().__init__(mesh, params, world, owner=owner, wall_dist=wall_dist, parts=parts)

    def _local(self, parts):
        if len(parts) != self._world:
            raise ValueError("one part per rank")
        return [parts[self._rank]]

    def _exchange(self, get) -> None:
        import torch

        a = get(self.o[0])
        # the received ghosts must land in the oracle's own array: a reshape of a
        # non-contiguous array would be a copy, and they would be lost
        if not a.flags.c_contiguous:
            raise ValueError("halo exchange needs C-contiguous work arrays")
        t = torch.from_numpy(a.reshape(-1, a.shape[-1]))
        assert np.shares_memory(a, t.numpy())
        P.exchange(self.parts[0].halo, t)

    def _allsum(self, s: float, n: int):
        import torch
        import torch.distributed as dist

        t = torch.tensor([s, float(n)], dtype=torch.float64)
        dist.all_reduce(t)
        return float(t[0]), int(round(float(t[1])))

    def _allmin(self, v: float) -> float:
        import torch
        import torch.distributed as dist

        t = torch.tensor([v], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MIN)
        return float(t[0])

    def local_cells(self):
        return self.parts[0].cells

