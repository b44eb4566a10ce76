"""ctypes front end of the oracle (oracle/phx_oracle.c).

TEST INFRASTRUCTURE ONLY: the CPU restatement of the reference path used as
the parity checker by tests/, __graft_entry__.smoke() and as bench.py's
`cpu_baseline`.  The product (phenlei_b200) never imports this module.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libphx_oracle.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class _Grid(C.Structure):
    _fields_ = [("n_node", C.c_int), ("n_face", C.c_int), ("n_cell", C.c_int), ("n_bface", C.c_int),
                ("x", _dp), ("y", _dp), ("z", _dp), ("face_off", _ip), ("face2node", _ip),
                ("left", _ip), ("right", _ip), ("cell_off", _ip), ("cell2node", _ip),
                ("n_region", C.c_int), ("region_type", _ip), ("bface_region", _ip)]


class _Metrics(C.Structure):
    _fields_ = [("xfn", _dp), ("yfn", _dp), ("zfn", _dp), ("area", _dp), ("xfc", _dp), ("yfc", _dp),
                ("zfc", _dp), ("xcc", _dp), ("ycc", _dp), ("zcc", _dp), ("vol", _dp), ("skew", _dp),
                ("walldist", _dp), ("avg_vol", C.c_double), ("c2f_off", _ip), ("c2f", _ip),
                ("iwt", _dp), ("ixx", _dp), ("iyy", _dp), ("izz", _dp), ("ixy", _dp), ("ixz", _dp), ("iyz", _dp)]


class _Params(C.Structure):
    _fields_ = [("gama", C.c_double), ("mach", C.c_double), ("attack", C.c_double), ("sideslip", C.c_double),
                ("prim_inf", C.c_double * 5), ("coef_state", C.c_double), ("p_total", C.c_double),
                ("viscous", C.c_int), ("reynolds", C.c_double), ("prandtl", C.c_double),
                ("prandtl_turb", C.c_double), ("tsuth_nd", C.c_double), ("wall_temperature", C.c_double),
                ("gradient", C.c_int), ("limiter", C.c_int), ("venkat_coeff", C.c_double),
                ("recon_method", C.c_int), ("scheme", C.c_int), ("entropy_fix", C.c_int),
                ("entropy_acoustic", C.c_double), ("entropy_convective", C.c_double),
                ("cfl_start", C.c_double), ("cfl_end", C.c_double), ("cfl_vary_step", C.c_int),
                ("ktmax", C.c_double), ("n_sweeps", C.c_int), ("lusgs_tol", C.c_double),
                ("skewness_angle", C.c_double), ("nut_inf", C.c_double), ("vist_inf", C.c_double),
                ("turb_cfl_scale", C.c_double), ("turb_skew_angle", C.c_double), ("ausmpw_limiter", C.c_double),
                ("flow_init_step", C.c_int), ("first_order", C.c_int)]

# uns_limiter_name (GetLimiterID, API/Physics/src/Limiter.cpp:1279-1300)
LIMITERS = {"nolim": 0, "vencat": 1, "1st": 2, "barth": 3}
# uns_scheme_name (GetSchemeID, API/Physics/src/Flux_Inviscid.cpp:16-86)
SCHEMES = {"roe": 0, "ausmpw+": 1, "steger": 2, "vanleer": 3, "hlle": 4, "ausmdv": 5, "ausmpw": 6,
           "vanleer_Rotate": 7}


class _Work(C.Structure):
    _fields_ = [("gama", _dp), ("t", _dp), ("dqdx", _dp), ("dqdy", _dp), ("dqdz", _dp), ("limit", _dp),
                ("res", _dp), ("inv_spec", _dp), ("vis_spec", _dp), ("dt", _dp), ("dq", _dp),
                ("visl", _dp), ("vist", _dp), ("dtdx", _dp), ("dtdy", _dp), ("dtdz", _dp),
                ("res_norm", C.c_double), ("n_negative", C.c_int),
                ("qt", _dp), ("res_t", _dp), ("spec_t", _dp), ("dqt", _dp), ("matl", _dp), ("matr", _dp),
                ("dntx", _dp), ("dnty", _dp), ("dntz", _dp), ("qnode", _dp), ("tnode_prev", _dp),
                ("have_tnode_prev", C.c_int), ("qtnode", _dp), ("have_qtnode", C.c_int)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"oracle library missing: {LIB_PATH} (make -C oracle)")
        _lib = C.CDLL(LIB_PATH)
        _lib.ox_cfl.restype = C.c_double
        _lib.ox_residual_norm.restype = C.c_double
        _lib.ox_update.restype = C.c_int
        _lib.ox_timestep_raw.restype = C.c_double
    return _lib


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


def entropy_fix_coefficient(mach: float, scale: float = 1.0) -> float:
    """Param_NSSolver::SetEntropyFixCoefficients (CFD/NSSolver/src/Param_NSSolver.cpp:224-268)."""
    if mach <= 0.6:
        e = 0.0001
    elif mach <= 2.0:
        x0, x1, y0, y1 = 0.6, 2.0, 0.0001, 0.01
        e = y0 * (mach - x1) / (x0 - x1) + y1 * (mach - x0) / (x1 - x0)
    elif mach <= 5.0:
        x0, x1, y0, y1 = 2.0, 5.0, 0.01, 0.5
        e = y0 * (mach - x1) / (x0 - x1) + y1 * (mach - x0) / (x1 - x0)
    else:
        e = 1.0
    return e * scale


def total_pressure(gama: float, mach: float) -> float:
    """PerfectGas::ComputePTotal (API/Physics/src/PerfectGas.cpp:1609-1640)."""
    p = 1.0 / (gama * mach * mach)
    m12 = mach * mach
    gp1, gm1 = gama + 1.0, gama - 1.0
    c1 = 2.0 / gm1 + m12
    c2 = 2.0 * gama / gm1 * m12 - 1.0
    cc = gama / (gama - 1.0)
    t0t = 1.0 + 0.5 * gm1 * c1 / c2
    if mach > 1.0:
        p *= (2.0 * gama / gp1 * m12 - gm1 / gp1)
    # pow of a negative base is NaN in C, as in the reference (subsonic Mach
    # numbers make t0t negative); NaN disables the pressure-based CFL limit.
    return p * (math.pow(t0t, cc) if t0t >= 0.0 else float("nan"))


def make_params(**kw) -> _Params:
    """Oracle parameters from hypara-style keys (same defaults as the product's
    phenlei_b200.params.SolverParams)."""
    gama = kw.get("refGama", 1.4)
    mach = kw.get("refMachNumber", 0.5)
    att = math.radians(kw.get("attackd", 0.0))
    sid = math.radians(kw.get("angleSlide", 0.0))
    p = _Params()
    p.gama, p.mach, p.attack, p.sideslip = gama, mach, att, sid
    coef = 1.0 / (gama * mach * mach)
    pinf = [1.0, math.cos(att) * math.cos(sid), math.sin(att) * math.cos(sid), math.sin(sid), coef]
    for i in range(5):
        p.prim_inf[i] = pinf[i]
    p.coef_state = coef
    p.p_total = total_pressure(gama, mach)
    p.viscous = kw.get("viscousType", 0)
    p.reynolds = kw.get("refReNumber", 1.0)
    p.prandtl = kw.get("prl", 0.72)
    p.prandtl_turb = kw.get("prt", 0.90)
    p.tsuth_nd = kw.get("tsuth_nd", 110.4 / kw.get("refDimensionalTemperature", 288.15))
    p.wall_temperature = kw.get("wallTemperature", -1.0)
    p.gradient = {"ggcell": 0, "lsq": 1, "ggnode": 2}[kw.get("gradientName", "ggcell")]
    p.limiter = LIMITERS[kw.get("uns_limiter_name", "vencat")]
    p.venkat_coeff = kw.get("venkatCoeff", 5.0)
    p.recon_method = kw.get("reconmeth", 1)
    p.scheme = SCHEMES[kw.get("uns_scheme_name", "roe")]
    p.ausmpw_limiter = kw.get("AusmpwPlusLimiter", 1.0)
    p.flow_init_step = kw.get("flowInitStep", 100)   # cfd_para.hypara:1290
    if kw.get("flowInitMethod", 0) not in (0, 2):
        raise ValueError("flowInitMethod 1 (boundary-layer start) and 3 (GMRES) are not on the path")
    p.entropy_fix = kw.get("roeEntropyFixMethod", 3)
    e = entropy_fix_coefficient(mach, kw.get("roeEntropyScale", 1.0))
    p.entropy_acoustic = p.entropy_convective = e
    p.cfl_start = kw.get("CFLStart", 0.01)
    p.cfl_end = kw.get("CFLEnd", 10.0)
    p.cfl_vary_step = kw.get("CFLVaryStep", 500)
    p.ktmax = kw.get("ktmax", 1.0e10)
    p.n_sweeps = kw.get("nLUSGSSweeps", 1)
    p.lusgs_tol = kw.get("LUSGSTolerance", 0.01)
    p.skewness_angle = kw.get("skewnessAngle", 60.0)
    # Param_TurbSolver::Init: freeStreamTurbVar[ISA] = muoo / (rho_inf * 1 + SMALL)
    p.nut_inf = kw.get("muoo", 3.0) / (1.0 * 1.0 + 1e-40)
    p.vist_inf = kw.get("freeStreamViscosity", 1.0e-3)
    p.turb_cfl_scale = kw.get("turbCFLScale", 1.0)
    p.turb_skew_angle = kw.get("turbSkewnessAngle", 0.0)
    return p


class Oracle:
    """Oracle state for one mesh: grid, metrics and the primitive field."""

    def __init__(self, mesh, params: dict, wall_dist=None):
        if mesh.n_face and int(np.min(mesh.face_nnode)) < 3:
            # the restated path is the three-dimensional one (phx_ctx_create refuses the same grids)
            raise ValueError("faces of fewer than three nodes: a two-dimensional grid")
        self.mesh = mesh
        self.keep = []
        nf, nc, nb = mesh.n_face, mesh.n_cell, mesh.n_bface
        self.nt = nt = nc + nb
        fo = mesh.face_offsets().astype(np.int32)
        co = mesh.cell_offsets().astype(np.int32)
        right = mesh.right.astype(np.int32).copy()
        right[:nb] = nc + np.arange(nb, dtype=np.int32)
        rtype, breg = mesh.solver_regions()
        arrs = dict(x=np.ascontiguousarray(mesh.x, np.float64), y=np.ascontiguousarray(mesh.y, np.float64),
                    z=np.ascontiguousarray(mesh.z, np.float64), fo=fo, f2n=mesh.face2node.astype(np.int32),
                    left=mesh.left.astype(np.int32), right=right, co=co, c2n=mesh.cell2node.astype(np.int32),
                    rtype=rtype, breg=breg)
        self.keep.append(arrs)
        g = _Grid()
        g.n_node, g.n_face, g.n_cell, g.n_bface = mesh.n_node, nf, nc, nb
        g.x, g.y, g.z = _p(arrs["x"]), _p(arrs["y"]), _p(arrs["z"])
        g.face_off, g.face2node = _p(fo, _ip), _p(arrs["f2n"], _ip)
        g.left, g.right = _p(arrs["left"], _ip), _p(right, _ip)
        g.cell_off, g.cell2node = _p(co, _ip), _p(arrs["c2n"], _ip)
        g.n_region, g.region_type, g.bface_region = len(rtype), _p(rtype, _ip), _p(arrs["breg"], _ip)
        self.g = g
        self.geo = {k: np.zeros(nf) for k in ("xfn", "yfn", "zfn", "area", "xfc", "yfc", "zfc")}
        self.geo.update({k: np.zeros(nt) for k in ("xcc", "ycc", "zcc", "vol")})
        self.geo["skew"] = np.zeros(nc)
        self.c2f_off = np.zeros(nc + 1, np.int32)
        self.c2f = np.zeros(2 * nf - nb, np.int32)
        m = _Metrics()
        for k, v in self.geo.items():
            setattr(m, k, _p(v))
        self.walldist = None
        if wall_dist is not None:
            self.walldist = np.ascontiguousarray(wall_dist, np.float64)
            m.walldist = _p(self.walldist)
        else:
            m.walldist = _dp()
        m.c2f_off, m.c2f = _p(self.c2f_off, _ip), _p(self.c2f, _ip)
        self.lsq = {"iwt": np.zeros(nf)}
        self.lsq.update({k: np.zeros(nc) for k in ("ixx", "iyy", "izz", "ixy", "ixz", "iyz")})
        for k, v in self.lsq.items():
            setattr(m, k, _p(v))
        lib().ox_compute_metrics(C.byref(g), C.byref(m))
        self.m = m
        self.params = dict(params)
        self.p = make_params(**params)
        self.q = np.zeros((5, nt))
        self.q[:, :nc] = np.array(self.p.prim_inf[:])[:, None]
        self.w_arrays = {}
        w = _Work()
        for name, shape in [("gama", (nt,)), ("t", (nt,)), ("dqdx", (5, nt)), ("dqdy", (5, nt)),
                            ("dqdz", (5, nt)), ("limit", (nt,)), ("res", (5, nt)), ("inv_spec", (nc,)),
                            ("vis_spec", (nc,)), ("dt", (nt,)), ("dq", (5, nt)), ("visl", (nt,)),
                            ("vist", (nt,)), ("dtdx", (nt,)), ("dtdy", (nt,)), ("dtdz", (nt,)),
                            ("qt", (nt,)), ("res_t", (nt,)), ("spec_t", (nt,)), ("dqt", (nt,)),
                            ("matl", (nf,)), ("matr", (nf,)), ("dntx", (nt,)), ("dnty", (nt,)), ("dntz", (nt,)),
                            ("qnode", (5, mesh.n_node)), ("tnode_prev", (mesh.n_node,)),
                            ("qtnode", (mesh.n_node,))]:
            a = np.zeros(shape)
            self.w_arrays[name] = a
            setattr(w, name, _p(a))
        self.w = w
        self.step = 0
        if self.p.viscous == 3:
            if self.walldist is None:
                raise ValueError("the SA model needs the wall distance of every cell")
            self.w_arrays["qt"][:] = self.p.nut_inf

    @property
    def avg_vol(self):
        return self.m.avg_vol

    def set_state(self, q_cells: np.ndarray, qt_cells=None):
        self.q[:, : self.mesh.n_cell] = q_cells
        self.w.have_tnode_prev = 0
        self.w.have_qtnode = 0
        if qt_cells is not None:
            self.w_arrays["qt"][: self.mesh.n_cell] = qt_cells

    def iterate(self, nsteps: int = 1):
        hist = []
        for _ in range(nsteps):
            self.step += 1
            lib().ox_ns_iteration(C.byref(self.g), C.byref(self.m), C.byref(self.p), self.step,
                                  _p(self.q), C.byref(self.w))
            hist.append(self.w.res_norm)
        return np.array(hist)

    def work(self, name):
        return self.w_arrays[name]

    def node_values(self):
        """GG-node node values [5][n_node] and temperature node values [n_node] of
        the current state, with its boundary values and temperature formed first
        (what PostSolve hands the next iteration's gradient)."""
        nn, nt = self.mesh.n_node, self.nt
        q = self.q.copy()
        gama, t = np.zeros(nt), np.zeros(nt)
        L = lib()
        L.ox_gamma_temperature(C.byref(self.g), C.byref(self.p), _p(q), _p(gama), _p(t))
        L.ox_ns_boundary(C.byref(self.g), C.byref(self.m), C.byref(self.p), _p(q), _p(gama))
        L.ox_gamma_temperature(C.byref(self.g), C.byref(self.p), _p(q), _p(gama), _p(t))
        qn, tn = np.zeros((5, nn)), np.zeros(nn)
        L.ox_node_values(C.byref(self.g), C.byref(self.m), _p(q), 5, _p(t), _p(qn), _p(tn))
        return qn, tn

    def forces(self):
        """Wall force sums of AirForceCoefParts (16 values) from the current state."""
        out = np.zeros(16)
        lib().ox_forces(C.byref(self.g), C.byref(self.m), C.byref(self.p), _p(self.q), C.byref(self.w), _p(out))
        return out
