"""The oracle (C restatement) against golden vectors produced by the
reference solver itself (tests/golden/make_golden.py).  CPU only."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from tests.conftest import rel_err

GEOM = ("xfn", "yfn", "zfn", "area", "xfc", "yfc", "zfc", "xcc", "ycc", "zcc", "vol")


SCHEME_TAGS = ("steger", "vanleer", "hlle", "ausmdv", "ausmpwp", "ausmpw", "vanleerrot")
SCHEME_CASES = [f"euler_bump_16x8x2_{t}_step3" for t in SCHEME_TAGS] + \
    [f"euler_tetcube_4_{t}_m16_step2" for t in SCHEME_TAGS]


INIT_CASES = ["euler_bump_16x8x2_init5_step2", "euler_bump_16x8x2_nolim_init2_step3"]
LIMITER_CASES = ["euler_bump_16x8x2_barth_step3", "euler_tetcube_4_barth_step2", "euler_bump_16x8x2_1st_step3"]


@pytest.mark.parametrize("name", ["euler_bump_16x8x2_step1", "euler_bump_16x8x2_step40", "euler_tetcube_4_step3"]
                         + SCHEME_CASES + INIT_CASES + LIMITER_CASES)
def test_oracle_matches_reference(golden, name):
    d = golden(name)
    m = d["mesh_obj"]
    nc = m.n_cell
    o = Oracle(m, d["params_dict"])
    for k in GEOM:
        assert rel_err(o.geo[k], d[k]) <= 1e-14, k
    if "state_in" in d:
        o.set_state(d["state_in"][:, :nc])
    hist = o.iterate(int(d["nsteps"]))
    assert rel_err(hist, d["res_hist"]) <= 1e-12
    assert rel_err(o.q[:, :nc], d["q"][:, :nc]) <= 1e-12
    assert rel_err(o.work("res")[:, :nc], d["res"][:, :nc]) <= 1e-12
    assert rel_err(o.work("dt")[:nc], d["dt"][:nc]) <= 1e-12
    assert rel_err(o.work("limit"), d["limit"]) <= 1e-12
    assert rel_err(o.work("dqdx")[:, :nc], d["gradPrimtiveVarX"][:, :nc]) <= 1e-12
    assert rel_err(o.work("dqdz")[:, :nc], d["gradPrimtiveVarZ"][:, :nc]) <= 1e-12
    assert rel_err(o.work("inv_spec"), d["invSpectralRadius"]) <= 1e-12
    assert rel_err(o.forces(), d["forces"]) <= 1e-12


@pytest.mark.parametrize("name", ["laminar_bump_16x8x2_lsq_step1", "laminar_bump_16x8x2_step20",
                                  "laminar_tetcube_4_lsq_step3", "laminar_bump_16x8x2_init3_step5",
                                  "laminar_bump_16x8x2_barth_lsq_step2"])
def test_oracle_matches_reference_laminar(golden, name):
    """Laminar NS: Sutherland viscosity, temperature gradient, viscous flux and
    spectral radius, no-slip adiabatic walls, GG-cell and LSQ gradients."""
    d = golden(name)
    m = d["mesh_obj"]
    nc = m.n_cell
    o = Oracle(m, d["params_dict"])
    if "state_in" in d:
        o.set_state(d["state_in"][:, :nc])
    hist = o.iterate(int(d["nsteps"]))
    assert rel_err(hist, d["res_hist"]) <= 1e-12
    assert rel_err(o.q[:, :nc], d["q"][:, :nc]) <= 1e-12
    assert rel_err(o.work("res")[:, :nc], d["res"][:, :nc]) <= 1e-12
    assert rel_err(o.work("dt")[:nc], d["dt"][:nc]) <= 1e-12
    assert rel_err(o.work("visl")[:nc], d["visl"][:nc]) <= 1e-12
    assert rel_err(o.work("vis_spec"), d["visSpectralRadius"]) <= 1e-12
    assert rel_err(o.work("dqdy")[:, :nc], d["gradPrimtiveVarY"][:, :nc]) <= 1e-12
    assert rel_err(o.work("dtdx")[:nc], d["gradTemperatureX"][:nc]) <= 1e-12
    assert rel_err(o.work("dtdz")[:nc], d["gradTemperatureZ"][:nc]) <= 1e-12
    assert rel_err(o.forces(), d["forces"]) <= 1e-12


@pytest.mark.parametrize("name", ["sa_bump_16x8x2_step1", "sa_bump_16x8x2_lsq_step3", "sa_bump_16x8x2_step30",
                                  "sa_bump_prism_16x8x2_step2", "sa_bump_16x8x2_init2_step3",
                                  "sa_plate_16x8x2_ausmpwp_step2", "sa_plate_16x8x2_ausmpwp_step20"])
def test_oracle_matches_reference_sa(golden, name):
    """Spalart-Allmaras (NSMB formation) coupled to the NS step: boundary
    values, eddy viscosity, source (negative-nu~ branch included), upwind
    convection, diffusion, spectral radius, scalar LU-SGS."""
    d = golden(name)
    m = d["mesh_obj"]
    nc = m.n_cell
    o = Oracle(m, d["params_dict"], wall_dist=d["walldist"])
    if "state_in" in d:
        o.set_state(d["state_in"][:5, :nc], d["state_in"][5, :nc])
    hist = o.iterate(int(d["nsteps"]))
    assert rel_err(hist, d["res_hist"]) <= 1e-12
    assert rel_err(o.q[:, :nc], d["q"][:, :nc]) <= 1e-12
    assert rel_err(o.work("res")[:, :nc], d["res"][:, :nc]) <= 1e-12
    assert rel_err(o.work("qt")[:nc], d["q_turb"][:nc]) <= 1e-12
    assert rel_err(o.work("vist"), d["vist"]) <= 1e-12
    assert rel_err(o.work("res_t")[:nc], d["res_turb"][:nc]) <= 1e-12
    assert rel_err(o.work("spec_t")[:nc], d["spec_turb"][:nc]) <= 1e-12
    assert rel_err(o.work("dntx")[:nc], d["gradTurbulenceX"][:nc]) <= 1e-12
    assert rel_err(o.forces(), d["forces"]) <= 1e-12


def test_oracle_detects_planted_error(golden):
    """A mistake planted in the oracle's input shows up in the comparison."""
    d = golden("euler_bump_16x8x2_step1")
    m = d["mesh_obj"]
    o = Oracle(m, d["params_dict"])
    s = d["state_in"][:, : m.n_cell].copy()
    s[4, 5] *= 1.0 + 1e-6
    o.set_state(s)
    o.iterate(1)
    assert rel_err(o.work("res")[:, : m.n_cell], d["res"][:, : m.n_cell]) > 1e-10


@pytest.mark.parametrize("name", ["euler_bump_16x8x2_ggnode_step1", "laminar_bump_16x8x2_ggnode_step1",
                                  "laminar_bump_16x8x2_ggnode_step20", "euler_tetcube_4_ggnode_step3"])
def test_oracle_matches_reference_ggnode(golden, name):
    """GG-node gradient (the reference's default): node values with the
    boundary-type priorities and 1/distance weights, face values from the face's
    nodes (0.5 (L + ghost) on non-symmetry boundary faces), ghost gradients
    copied from the owner; the node values the reference's PostSolve formed
    after the last iteration against the oracle's node values of its final state."""
    d = golden(name)
    m = d["mesh_obj"]
    nc = m.n_cell
    o = Oracle(m, d["params_dict"])
    if "state_in" in d:
        o.set_state(d["state_in"][:, :nc])
    hist = o.iterate(int(d["nsteps"]))
    assert rel_err(hist, d["res_hist"]) <= 1e-12
    assert rel_err(o.q[:, :nc], d["q"][:, :nc]) <= 1e-12
    assert rel_err(o.work("res")[:, :nc], d["res"][:, :nc]) <= 1e-12
    assert rel_err(o.work("dqdx")[:, :nc], d["gradPrimtiveVarX"][:, :nc]) <= 1e-12
    assert rel_err(o.work("dqdy")[:, :nc], d["gradPrimtiveVarY"][:, :nc]) <= 1e-12
    assert rel_err(o.work("dqdz")[:, :nc], d["gradPrimtiveVarZ"][:, :nc]) <= 1e-12
    assert rel_err(o.work("limit"), d["limit"]) <= 1e-12
    if "gradTemperatureX" in d:
        assert rel_err(o.work("dtdx")[:nc], d["gradTemperatureX"][:nc]) <= 1e-12
    qn, _ = o.node_values()
    assert rel_err(qn, d["qnode"]) <= 1e-14
    assert rel_err(o.forces(), d["forces"]) <= 1e-12


@pytest.mark.parametrize("name", ["sa_bump_16x8x2_ggnode_step1", "sa_bump_16x8x2_ggnode_step20"])
def test_oracle_matches_reference_sa_ggnode(golden, name):
    """GG-node with Spalart-Allmaras: the nu~ gradient from the node values the
    turbulence PostSolve formed (face-based sums, symmetry / far-field / wall
    nodes rebuilt from those faces only), checked with the node values the
    reference formed after the last iteration."""
    d = golden(name)
    m = d["mesh_obj"]
    nc = m.n_cell
    o = Oracle(m, d["params_dict"], wall_dist=d["walldist"])
    if "state_in" in d:
        o.set_state(d["state_in"][:5, :nc], d["state_in"][5, :nc])
    hist = o.iterate(int(d["nsteps"]))
    assert rel_err(hist, d["res_hist"]) <= 1e-12
    assert rel_err(o.q[:, :nc], d["q"][:, :nc]) <= 1e-12
    assert rel_err(o.work("qt")[:nc], d["q_turb"][:nc]) <= 1e-12
    assert rel_err(o.work("vist"), d["vist"]) <= 1e-12
    assert rel_err(o.work("res_t")[:nc], d["res_turb"][:nc]) <= 1e-12
    assert rel_err(o.work("dntx")[:nc], d["gradTurbulenceX"][:nc]) <= 1e-12
    assert rel_err(o.work("qtnode"), d["qTurbNode"]) <= 1e-14
    assert rel_err(o.forces(), d["forces"]) <= 1e-12


ZONE_CASES = ["zones2_euler_bump_16x8x2_step10", "zones3_laminar_bump_16x8x2_lsq_step10",
              "zones2_euler_bump_16x8x2_barth_ktmax_step10", "zones2_sa_bump_16x8x2_step10",
              "zones3_sa_bump_16x8x2_prism_step5"]


@pytest.mark.parametrize("name", ZONE_CASES)
def test_partitioned_oracle_matches_reference_zones(golden, name):
    """The oracle on a partitioned grid (oracle/partitioned.py) against the
    reference's own run on the same zones, all on one rank: interface ghosts,
    SwapGeometry, the minimum time step over the zones, the NS dq exchanged
    between the sweeps and no SA dq, over 5-10 iterations."""
    from oracle.partitioned import PartitionedOracle

    d = golden(name)
    m = d["mesh_obj"]
    nc = m.n_cell
    params = d["params_dict"]
    sa = params.get("viscousType", 0) == 3
    po = PartitionedOracle(m, params, int(d["nparts"]), owner=d["owner"],
                           wall_dist=d["walldist"] if sa else None)
    st = d["state_in"]
    po.set_state(st[:5], st[5] if sa else None)
    hist = po.iterate(int(d["nsteps"]))
    assert rel_err(hist, d["res_hist"]) <= 1e-12
    assert rel_err(po.gather("q"), d["q"]) <= 1e-12
    assert rel_err(po.gather("res"), d["res"]) <= 1e-12
    assert rel_err(po.gather("dt"), d["dt"]) <= 1e-12
    assert rel_err(po.gather("limit"), d["limit"]) <= 1e-12
    assert rel_err(po.gather("dqdx"), d["gradPrimtiveVarX"]) <= 1e-12
    if sa:
        assert rel_err(po.gather("qt"), d["q_turb"]) <= 1e-12
        assert rel_err(po.gather("vist"), d["vist"]) <= 1e-12
