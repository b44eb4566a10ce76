"""Python front end of the phx C ABI (include/phx.h), mirroring the solver
plug-in surface of PHengLEI's NSSolverUnstruct (CFD/NSSolver/include/NSSolverUnstruct.h):
Boundary, ComputeGradient/ComputeLimiter, UpdateResiduals (+SpectrumRadius,
TimeStep), LUSGS, UpdateFlowField and the Controller::Relaxation sequence.

Parameters use the reference's hypara key names (cfd_para.hypara); string-valued
keys take the reference's strings ("roe", "vencat", "ggcell", ...).

The CUDA library is required: there is no CPU path.  Importing this module on
a machine without the built library raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libphx.so")

PHX_FP64, PHX_MIXED = 0, 1
PHX_Q, PHX_RES, PHX_DT, PHX_LIMIT, PHX_GRADX, PHX_GRADY, PHX_GRADZ, PHX_DQ, PHX_INVSPEC, PHX_VISSPEC = range(10)
PHX_Q_TURB, PHX_VISL, PHX_VIST, PHX_RES_TURB = 10, 11, 12, 13
PHX_SA_SRC = 15
PHX_GRAD_TURB = 16
# halo fields of a partitioned grid (include/phx.h PHX_HALO_*)
PHX_HALO_Q, PHX_HALO_GRADIENT, PHX_HALO_DQ, PHX_HALO_TURB = range(4)
ERRORS = {-1: "PHX_ERR_ARG", -2: "PHX_ERR_CUDA", -3: "PHX_ERR_TIMEOUT", -4: "PHX_ERR_NUMERIC", -5: "PHX_ERR_STATE"}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class GridDesc(C.Structure):
    _fields_ = [("n_node", C.c_int64), ("n_face", C.c_int64), ("n_cell", C.c_int64), ("n_bface", C.c_int64),
                ("x", _dp), ("y", _dp), ("z", _dp), ("face_nnode", _ip), ("face2node", _ip),
                ("left_cell", _ip), ("right_cell", _ip), ("cell_nnode", _ip), ("cell2node", _ip),
                ("n_region", C.c_int32), ("region_type", _ip), ("bface_region", _ip), ("wall_dist", _dp)]


class Params(C.Structure):
    _fields_ = [("precision", C.c_int32), ("refGama", C.c_double), ("refMachNumber", C.c_double),
                ("attackd", C.c_double), ("angleSlide", C.c_double), ("viscousType", C.c_int32),
                ("refReNumber", C.c_double), ("refDimensionalTemperature", C.c_double), ("prl", C.c_double),
                ("prt", C.c_double), ("tsuth", C.c_double), ("wallTemperature", C.c_double),
                ("gradientName", C.c_int32), ("uns_limiter_name", C.c_int32), ("ivencat", C.c_int32),
                ("venkatCoeff", C.c_double), ("reconmeth", C.c_int32), ("uns_scheme_name", C.c_int32),
                ("roeEntropyFixMethod", C.c_int32), ("roeEntropyScale", C.c_double), ("CFLStart", C.c_double),
                ("CFLEnd", C.c_double), ("CFLVaryStep", C.c_int32), ("ktmax", C.c_double),
                ("nLUSGSSweeps", C.c_int32), ("LUSGSTolerance", C.c_double), ("skewnessAngle", C.c_double),
                ("muoo", C.c_double), ("turbCFLScale", C.c_double), ("sa_source", C.c_int32),
                ("turbSkewnessAngle", C.c_double), ("freeStreamViscosity", C.c_double),
                ("AusmpwPlusLimiter", C.c_double), ("flowInitStep", C.c_int32), ("flowInitMethod", C.c_int32)]


_STRING_KEYS = {
    "gradientName": {"ggcell": 0, "lsq": 1, "ggnode": 2},
    "uns_limiter_name": {"nolim": 0, "vencat": 1, "1st": 2, "barth": 3},
    "uns_scheme_name": {"roe": 0, "ausmpw+": 1, "steger": 2, "vanleer": 3, "hlle": 4, "ausmdv": 5, "ausmpw": 6,
                        "vanleer_Rotate": 7},
    "precision": {"fp64": PHX_FP64, "mixed": PHX_MIXED},
    "sa_source": {"exact": 0, "mlp": 1, "mlp_fallback": 2},
}

_lib = None


def lib() -> C.CDLL:
    """The loaded phx library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"phx CUDA library not built: {LIB_PATH} (python -m phenlei_b200.build)")
        _lib = C.CDLL(LIB_PATH)
        _lib.phx_last_error.restype = C.c_char_p
        _lib.phx_launch_count.restype = C.c_int64
        _lib.phx_ctx_create.argtypes = [C.POINTER(GridDesc), C.POINTER(Params), C.POINTER(C.c_void_p)]
        for name in ("phx_set_state", "phx_get_state", "phx_set_state_device", "phx_get_state_device"):
            getattr(_lib, name).argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int64]
        _lib.phx_get_geometry.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p, C.c_int64]
        _lib.phx_ns_relaxation.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        _lib.phx_set_stream.argtypes = [C.c_void_p, C.c_void_p]
        for name in ("phx_ns_boundary", "phx_ns_gradient_limiter", "phx_ns_residual", "phx_ns_lusgs",
                     "phx_ns_update", "phx_ctx_destroy", "phx_launch_count", "phx_get_step", "phx_sa_boundary",
                     "phx_sa_residual", "phx_sa_lusgs", "phx_sa_update", "phx_ns_lusgs_forward",
                     "phx_ns_lusgs_backward", "phx_sa_lusgs_forward", "phx_sa_lusgs_backward", "phx_step_status"):
            getattr(_lib, name).argtypes = [C.c_void_p]
        _lib.phx_swap_geometry.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_double]
        _lib.phx_set_halo.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p]
        _lib.phx_halo_row_bytes.argtypes = [C.c_void_p, C.c_int]
        _lib.phx_halo_row_bytes.restype = C.c_int64
        _lib.phx_halo_pack.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        _lib.phx_halo_unpack.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        _lib.phx_ns_min_timestep.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        _lib.phx_ns_set_min_timestep.argtypes = [C.c_void_p, C.c_double]
        _lib.phx_set_step.argtypes = [C.c_void_p, C.c_int]
        _lib.phx_residual_norm.argtypes = [C.c_void_p, C.c_void_p]
        _lib.phx_forces.argtypes = [C.c_void_p, C.c_void_p]
        _lib.phx_sa_capture.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                        C.POINTER(C.c_int64)]
        _lib.phx_mlp_train.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_double,
                                       C.c_uint64, C.POINTER(C.c_double)]
        _lib.phx_mlp_get.argtypes = [C.c_void_p, C.c_void_p, C.c_int64]
        _lib.phx_mlp_set.argtypes = [C.c_void_p, C.c_void_p, C.c_int64]
        _lib.phx_mlp_blob_size.restype = C.c_int64
        _lib.phx_mlp_cells.argtypes = [C.c_void_p, C.POINTER(C.c_uint64)]
        _lib.phx_mlp_param_count.restype = C.c_int64
        _lib.phx_mlp_loss_grad.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                           C.POINTER(C.c_double)]
        _lib.phx_set_wait_limit.argtypes = [C.c_void_p, C.c_int64]
        _lib.phx_write_restart.argtypes = [C.c_void_p, C.c_char_p]
        _lib.phx_read_restart.argtypes = [C.c_void_p, C.c_char_p]
        _lib.phx_fault_hold_cell.argtypes = [C.c_void_p, C.c_int32]
    return _lib


class PhxError(RuntimeError):
    pass


def make_params(**keys) -> Params:
    """phx_params from hypara keys on top of the reference defaults."""
    p = Params()
    lib().phx_default_params(C.byref(p))
    for k, v in keys.items():
        if k in _STRING_KEYS and isinstance(v, str):
            v = _STRING_KEYS[k][v]
        if not hasattr(p, k):
            continue  # keys the path does not read (e.g. tscheme) are accepted and ignored
        setattr(p, k, v)
    return p


class NSSolverUnstruct:
    """One phx context: a grid, its FP64 metrics and the device-resident flow state."""

    def __init__(self, mesh, precision="fp64", wall_dist=None, **params):
        """wall_dist: distance of every cell centre to the nearest wall (reference
        order, [n_cell]); required by the SA model (viscousType 3)."""
        self.mesh = mesh
        self._keep = []
        nb, nc = mesh.n_bface, mesh.n_cell
        self.nt = nc + nb
        arr = lambda a, t: np.ascontiguousarray(a, dtype=t)  # noqa: E731
        a = dict(x=arr(mesh.x, np.float64), y=arr(mesh.y, np.float64), z=arr(mesh.z, np.float64),
                 fnn=arr(mesh.face_nnode, np.int32), f2n=arr(mesh.face2node, np.int32),
                 left=arr(mesh.left, np.int32), right=arr(mesh.right, np.int32),
                 cnn=arr(mesh.cell_nnode, np.int32), c2n=arr(mesh.cell2node, np.int32),
                 rtype=arr(mesh.solver_regions()[0], np.int32), breg=arr(mesh.solver_regions()[1], np.int32))
        self._keep.append(a)
        g = GridDesc()
        g.n_node, g.n_face, g.n_cell, g.n_bface = mesh.n_node, mesh.n_face, nc, nb
        d = lambda v: v.ctypes.data_as(_dp)  # noqa: E731
        i = lambda v: v.ctypes.data_as(_ip)  # noqa: E731
        g.x, g.y, g.z = d(a["x"]), d(a["y"]), d(a["z"])
        g.face_nnode, g.face2node, g.left_cell, g.right_cell = i(a["fnn"]), i(a["f2n"]), i(a["left"]), i(a["right"])
        g.cell_nnode, g.cell2node = i(a["cnn"]), i(a["c2n"])
        g.n_region, g.region_type, g.bface_region = len(mesh.regions), i(a["rtype"]), i(a["breg"])
        if wall_dist is not None:
            wd = np.ascontiguousarray(wall_dist, dtype=np.float64)
            if wd.shape != (nc,):
                raise ValueError("wall_dist must hold one value per cell")
            self._keep.append(wd)
            g.wall_dist = wd.ctypes.data_as(_dp)
        else:
            g.wall_dist = _dp()
        self.params = make_params(precision=precision, **params)
        h = C.c_void_p()
        rc = lib().phx_ctx_create(C.byref(g), C.byref(self.params), C.byref(h))
        if rc != 0:
            raise PhxError(f"phx_ctx_create failed: {ERRORS.get(rc, rc)}")
        self.h = h

    # -- plumbing ------------------------------------------------------------
    def _check(self, rc, what):
        if rc != 0:
            msg = lib().phx_last_error(self.h).decode()
            raise PhxError(f"{what}: {ERRORS.get(rc, rc)}: {msg}")

    def close(self):
        if getattr(self, "h", None):
            lib().phx_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_handle: int):
        self._check(lib().phx_set_stream(self.h, C.c_void_p(stream_handle)), "phx_set_stream")

    @property
    def launches(self) -> int:
        return int(lib().phx_launch_count(self.h))

    _SHAPES = {PHX_Q: 5, PHX_RES: 5, PHX_DT: 1, PHX_LIMIT: 1, PHX_GRADX: 5, PHX_GRADY: 5, PHX_GRADZ: 5,
               PHX_DQ: 5, PHX_INVSPEC: -1, PHX_VISSPEC: -1, PHX_Q_TURB: 1, PHX_VISL: 1, PHX_VIST: 1,
               PHX_RES_TURB: 1, PHX_SA_SRC: -1, PHX_GRAD_TURB: 3}

    def get(self, which) -> np.ndarray:
        rows = self._SHAPES[which]
        if rows < 0:
            out = np.empty(self.mesh.n_cell)
        else:
            out = np.empty((rows, self.nt)) if rows > 1 else np.empty(self.nt)
        self._check(lib().phx_get_state(self.h, which, out.ctypes.data, out.size), "phx_get_state")
        return out

    def set(self, which, values: np.ndarray):
        """PHX_Q, PHX_Q_TURB or PHX_VIST of cells and ghosts."""
        v = np.ascontiguousarray(values, dtype=np.float64)
        self._check(lib().phx_set_state(self.h, which, v.ctypes.data, v.size), "phx_set_state")

    def set_q_cells(self, q_cells: np.ndarray):
        """Set the primitive state of the interior cells (ghosts are set by Boundary)."""
        q = self.get(PHX_Q)
        q[:, : self.mesh.n_cell] = q_cells
        self.set(PHX_Q, q)

    def set_qt_cells(self, qt_cells: np.ndarray):
        """Set the SA variable nu~ of the interior cells (ghosts are set by the SA boundary)."""
        qt = self.get(PHX_Q_TURB)
        qt[: self.mesh.n_cell] = qt_cells
        self.set(PHX_Q_TURB, qt)

    def geometry(self, name: str) -> np.ndarray:
        n = self.mesh.n_face if name in ("xfn", "yfn", "zfn", "area", "xfc", "yfc", "zfc") else (
            self.mesh.n_cell if name in ("skew", "walldist") else self.nt)
        out = np.empty(n)
        self._check(lib().phx_get_geometry(self.h, name.encode(), out.ctypes.data, n), "phx_get_geometry")
        return out

    def DumpRestart(self, path: str):
        """The restart file (NSSolverUnstruct::DumpRestartH5 and
        TurbSolverUnstr::DumpRestartH5 content: outnstep, q, q_turb, visturb;
        plus the learned-source model)."""
        self._check(lib().phx_write_restart(self.h, os.fsencode(path)), "phx_write_restart")

    def ReadRestart(self, path: str):
        """Continues from a restart file of the same grid."""
        self._check(lib().phx_read_restart(self.h, os.fsencode(path)), "phx_read_restart")

    def ReadRestartH5(self, flow_path: str, zone: int = 0, turb_path: str | None = None):
        """Continues from the reference's own HDF5 restart files of this zone
        (phenlei_b200.fts.read_restart_h5): the step count, the state of the
        cells and ghosts and, with the turbulence file, nu~ and the eddy
        viscosity."""
        from .fts import read_restart_h5

        r = read_restart_h5(flow_path, zone, self.mesh.n_cell, self.mesh.n_bface, turb_path)
        self.set(PHX_Q, r["q"])
        if turb_path is not None:
            self.set(PHX_Q_TURB, r["q_turb"])
            if r["vist"] is not None:
                self.set(PHX_VIST, r["vist"])
        self.step = r["outnstep"]

    def set_wait_limit(self, polls: int):
        """Bound on every device-side dependency wait of the LU-SGS sweeps, in polls."""
        self._check(lib().phx_set_wait_limit(self.h, int(polls)), "phx_set_wait_limit")

    def fault_hold_cell(self, cell: int):
        """Failure-detection hook: the forward LU-SGS result of reference cell
        `cell` never comes (-1: off), so the step returns PHX_ERR_TIMEOUT."""
        self._check(lib().phx_fault_hold_cell(self.h, int(cell)), "phx_fault_hold_cell")

    @property
    def step(self) -> int:
        return int(lib().phx_get_step(self.h))

    @step.setter
    def step(self, v: int):
        self._check(lib().phx_set_step(self.h, int(v)), "phx_set_step")

    # -- the reference's solver methods ----------------------------------------
    def Boundary(self):
        self._check(lib().phx_ns_boundary(self.h), "phx_ns_boundary")

    def ComputeGradientAndLimiter(self):
        self._check(lib().phx_ns_gradient_limiter(self.h), "phx_ns_gradient_limiter")

    def UpdateResiduals(self):
        """InviscidFlux + ViscousFlux + LoadFlux, SpectrumRadius and TimeStep."""
        self._check(lib().phx_ns_residual(self.h), "phx_ns_residual")

    def LUSGS(self):
        self._check(lib().phx_ns_lusgs(self.h), "phx_ns_lusgs")

    def UpdateFlowField(self):
        self._check(lib().phx_ns_update(self.h), "phx_ns_update")

    # -- the reference's TurbSolverUnstr methods (SA) --------------------------
    def TurbBoundary(self):
        self._check(lib().phx_sa_boundary(self.h), "phx_sa_boundary")

    def TurbUpdateResiduals(self):
        """Viscosity, gradient of nu~, source, convection, diffusion, Diagonal."""
        self._check(lib().phx_sa_residual(self.h), "phx_sa_residual")

    def TurbLUSGS(self):
        self._check(lib().phx_sa_lusgs(self.h), "phx_sa_lusgs")

    def TurbUpdateFlowField(self):
        self._check(lib().phx_sa_update(self.h), "phx_sa_update")

    # -- one zone of a partitioned grid (interface faces) ----------------------
    def LUSGSForward(self):
        """SolveLUSGSForward (NSSolverUnstruct.cpp:15118); the dq exchange follows."""
        self._check(lib().phx_ns_lusgs_forward(self.h), "phx_ns_lusgs_forward")

    def LUSGSBackward(self):
        """SolveLUSGSBackward (NSSolverUnstruct.cpp:15446), after the dq exchange."""
        self._check(lib().phx_ns_lusgs_backward(self.h), "phx_ns_lusgs_backward")

    def TurbLUSGSForward(self):
        self._check(lib().phx_sa_lusgs_forward(self.h), "phx_sa_lusgs_forward")

    def TurbLUSGSBackward(self):
        self._check(lib().phx_sa_lusgs_backward(self.h), "phx_sa_lusgs_backward")

    def SwapGeometry(self, bfaces, xcc, ycc, zcc, vol, avg_vol: float = 0.0):
        """Region::SwapGeometry / ComputeGlobalGridSize: the neighbouring zones'
        cell centres and volumes behind the interface faces `bfaces`, and the
        average cell volume over all zones (0: keep this zone's)."""
        b = np.ascontiguousarray(bfaces, np.int32)
        x, y, z, v = (np.ascontiguousarray(a, np.float64) for a in (xcc, ycc, zcc, vol))
        if not (len(b) == len(x) == len(y) == len(z) == len(v)):
            raise ValueError("one centre and volume per interface face")
        self._check(lib().phx_swap_geometry(self.h, len(b), b.ctypes.data, x.ctypes.data, y.ctypes.data,
                                            z.ctypes.data, v.ctypes.data, float(avg_vol)), "phx_swap_geometry")

    def set_halo(self, send_cells, recv_bfaces):
        """The halo plan: cells whose rows this zone sends, interface faces whose
        ghosts it fills (each concatenated over the neighbours)."""
        sc = np.ascontiguousarray(send_cells, np.int32)
        rb = np.ascontiguousarray(recv_bfaces, np.int32)
        self._check(lib().phx_set_halo(self.h, len(sc), sc.ctypes.data, len(rb), rb.ctypes.data), "phx_set_halo")

    def halo_row_bytes(self, field: int) -> int:
        n = int(lib().phx_halo_row_bytes(self.h, field))
        if n < 0:
            raise PhxError(f"phx_halo_row_bytes: {ERRORS.get(n, n)}")
        return n

    def halo_pack(self, field: int, buf_ptr: int):
        self._check(lib().phx_halo_pack(self.h, field, C.c_void_p(buf_ptr)), "phx_halo_pack")

    def halo_unpack(self, field: int, buf_ptr: int):
        self._check(lib().phx_halo_unpack(self.h, field, C.c_void_p(buf_ptr)), "phx_halo_unpack")

    def min_timestep(self) -> float:
        v = C.c_double()
        self._check(lib().phx_ns_min_timestep(self.h, C.byref(v)), "phx_ns_min_timestep")
        return v.value

    def set_min_timestep(self, value: float):
        self._check(lib().phx_ns_set_min_timestep(self.h, float(value)), "phx_ns_set_min_timestep")

    def status(self):
        """Raises PhxError if a sweep's wait ran out or the repair overflowed."""
        self._check(lib().phx_step_status(self.h), "phx_step_status")

    # -- learned SA source --------------------------------------------------------
    def capture_sa_samples(self):
        """Features [n, 6], targets [n], reference cell numbers [n], scales [n] of
        every cell with nu~ > 0, from the last SA residual."""
        nc = self.mesh.n_cell
        f = np.empty((nc, 6), np.float32)
        t = np.empty(nc, np.float32)
        cells = np.empty(nc, np.int32)
        sc = np.empty(nc, np.float32)
        n = C.c_int64()
        self._check(lib().phx_sa_capture(self.h, f.ctypes.data, t.ctypes.data, cells.ctypes.data, sc.ctypes.data,
                                         nc, C.byref(n)), "phx_sa_capture")
        k = n.value
        # the device fills the arrays in the order its threads finish: sort by
        # cell so that a capture (and a model trained on it) is reproducible
        o = np.argsort(cells[:k], kind="stable")
        return f[:k][o], t[:k][o], cells[:k][o], sc[:k][o]

    def train_sa_mlp(self, features, targets, epochs=20, batch=8192, lr=1e-3, seed=0) -> float:
        f = np.ascontiguousarray(features, np.float32)
        t = np.ascontiguousarray(targets, np.float32)
        loss = C.c_double()
        self._check(lib().phx_mlp_train(self.h, f.ctypes.data, t.ctypes.data, len(t), epochs, batch, lr, seed,
                                        C.byref(loss)), "phx_mlp_train")
        return loss.value

    def mlp_blob(self) -> np.ndarray:
        b = np.empty(int(lib().phx_mlp_blob_size()), np.float32)
        self._check(lib().phx_mlp_get(self.h, b.ctypes.data, b.size), "phx_mlp_get")
        return b

    def set_mlp_blob(self, blob):
        b = np.ascontiguousarray(blob, np.float32)
        self._check(lib().phx_mlp_set(self.h, b.ctypes.data, b.size), "phx_mlp_set")

    def mlp_cells(self) -> int:
        n = C.c_uint64()
        self._check(lib().phx_mlp_cells(self.h, C.byref(n)), "phx_mlp_cells")
        return int(n.value)

    def Relaxation(self, nsteps: int = 1) -> np.ndarray:
        """nsteps outer iterations; returns the residual monitor per step."""
        hist = np.zeros(max(nsteps, 1))
        self._check(lib().phx_ns_relaxation(self.h, nsteps, hist.ctypes.data), "phx_ns_relaxation")
        return hist[:nsteps]

    def AirForceCoef(self, reference_area: float = 1.0) -> dict:
        """Wall force sums (AirForceCoefParts) and CL / CD (Force.cpp:441-536)."""
        out = np.zeros(16)
        self._check(lib().phx_forces(self.h, out.ctypes.data), "phx_forces")
        return force_coefficients(out, self.params.attackd, self.params.angleSlide, reference_area)

    def GetResidual(self) -> np.ndarray:
        out = np.zeros(5)
        self._check(lib().phx_residual_norm(self.h, out.ctypes.data), "phx_residual_norm")
        return out


def force_coefficients(sums, attackd: float = 0.0, angleSlide: float = 0.0, reference_area: float = 1.0) -> dict:
    """CL and CD from the 16 wall force sums of AirForceCoefParts
    (CA_f CA_p CN_f CN_p CZ_f CZ_p ...): the body-axis force coefficients scaled
    by 1 / forceReferenceArea and rotated by the angles of attack and sideslip
    (degrees), as Force.cpp:441-536 does."""
    import math

    out = np.asarray(sums, dtype=np.float64)
    a = math.radians(attackd)
    b = math.radians(angleSlide)
    cf = (out[0:6:2] + out[1:6:2]) / reference_area
    cl = -math.sin(a) * cf[0] + math.cos(a) * cf[1]
    cd = math.cos(a) * math.cos(b) * cf[0] + math.sin(a) * math.cos(b) * cf[1] + math.sin(b) * cf[2]
    return {"sums": out, "CL": cl, "CD": cd}


def mlp_loss_grad(params, x, y):
    """Mean squared error of one batch and its gradient with respect to the flat
    weight vector, computed by the library's training kernels (see
    phx_mlp_loss_grad)."""
    p = np.ascontiguousarray(params, np.float32)
    xx = np.ascontiguousarray(x, np.float32)
    yy = np.ascontiguousarray(y, np.float32)
    g = np.empty_like(p)
    loss = C.c_double()
    rc = lib().phx_mlp_loss_grad(p.ctypes.data, p.size, xx.ctypes.data, yy.ctypes.data, yy.size, g.ctypes.data,
                                 C.byref(loss))
    if rc != 0:
        raise PhxError(f"phx_mlp_loss_grad: {ERRORS.get(rc, rc)}")
    return loss.value, g
