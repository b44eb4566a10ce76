"""Generates the golden fixtures in tests/golden/ by running the REFERENCE
solver itself (oracle/_ref/ref_harness, built from the reference's own
sources by oracle/refbuild/Makefile) on small seeded cases.

    make -C oracle/refbuild REF=<reference root> -j8 all harness
    python tests/golden/make_golden.py

Each fixture is an .npz holding the case parameters (as JSON), the input state,
and the reference's arrays after the requested number of outer iterations.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.refrun import run_reference  # noqa: E402
from phenlei_b200 import mesh as M  # noqa: E402
from phenlei_b200.cases import perturbed_state  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

EULER_BUMP = {"viscousType": 0, "uns_scheme_name": "roe", "uns_limiter_name": "vencat", "ivencat": 7,
              "venkatCoeff": 5.0, "gradientName": "ggcell", "reconmeth": 1, "roeEntropyFixMethod": 3, "tscheme": 4,
              "nLUSGSSweeps": 1, "CFLStart": 0.01, "CFLEnd": 10.0, "CFLVaryStep": 500, "refMachNumber": 0.5,
              "attackd": 0.0, "refGama": 1.4}

# Laminar NS: viscous adiabatic walls on the bump, Sutherland viscosity, Re 1e4.
LAMINAR = dict(EULER_BUMP, viscousType=1, refMachNumber=0.3, refReNumber=1.0e4, refDimensionalTemperature=288.15,
               prl=0.72, wallTemperature=-1.0)

# Spalart-Allmaras (NSMB formation), adiabatic no-slip walls, Re 1e5.
SA = dict(LAMINAR, viscousType=3, viscousName="1eq-sa", refReNumber=1.0e5, muoo=3.0)

# SA flat plate, M 0.2, Re 5e6 per unit length, T 300 K, AUSMPW+, CFL 50.
SA_PLATE = dict(SA, refMachNumber=0.2, refReNumber=5.0e6, refDimensionalTemperature=300.0, prt=0.9,
                uns_scheme_name="ausmpw+", CFLEnd=50.0)


def turb_state(m, params, seed):
    """Seeded nu~ field around the free-stream value, about 10% of the cells negative."""
    rng = np.random.default_rng(seed)
    nu = params.get("muoo", 3.0) * (0.2 + 1.5 * rng.random(m.n_cell))
    neg = rng.random(m.n_cell) < 0.1
    nu[neg] = -0.5 * rng.random(int(neg.sum()))
    return nu


def mesh_spec(m, kind, args):
    return {"kind": kind, "args": args}


def fixture(name, kind, args, params, nsteps, perturb_seed=None, amplitude=0.02, turb_seed=None):
    m = getattr(M, kind)(**args)
    nc, nt = m.n_cell, m.n_cell + m.n_bface
    state = None
    if perturb_seed is not None:
        state = perturbed_state(m, params, seed=perturb_seed, amplitude=amplitude)
    sa = params.get("viscousType", 0) == 3
    if sa and turb_seed is not None:
        if state is None:
            from phenlei_b200.cases import freestream
            state = np.repeat(freestream(params)[:, None], nc, axis=1)
        state = np.vstack([state, turb_state(m, params, turb_seed)[None, :]])
    dumps = [("q", 5, nt), ("res", 5, nt), ("dt", 0, nt), ("limit2D", 5, nt), ("gradPrimtiveVarX", 5, nt),
             ("gradPrimtiveVarY", 5, nt), ("gradPrimtiveVarZ", 5, nt), ("invSpectralRadius", 0, nc)]
    viscous = params.get("viscousType", 0) > 0
    if viscous:
        dumps += [("visl", 0, nt), ("visSpectralRadius", 0, nc), ("gradTemperatureX", 1, nt),
                  ("gradTemperatureY", 1, nt), ("gradTemperatureZ", 1, nt)]
    if sa:
        dumps += [("vist", 0, nt), ("q_turb", 1, nt), ("res_turb", 1, nt), ("spec_turb", 1, nt),
                  ("gradTurbulenceX", 1, nt)]
    ggnode = params.get("gradientName") == "ggnode"
    if ggnode:
        dumps += [("qnode", 5, m.n_node)]
        if sa:
            dumps += [("qTurbNode", 1, m.n_node)]
    r = run_reference(m, params, nsteps, dumps=dumps, state=state)
    out = {"params": json.dumps(params), "mesh": json.dumps({"kind": kind, "args": args}),
           "nsteps": nsteps, "res_hist": r["res_hist"]}
    if state is not None:
        out["state_in"] = state
    for k in ("q", "res", "dt", "gradPrimtiveVarX", "gradPrimtiveVarY", "gradPrimtiveVarZ", "invSpectralRadius",
              "xfn", "yfn", "zfn", "area", "xfc", "yfc", "zfc", "xcc", "ycc", "zcc", "vol"):
        out[k] = r[k]
    if viscous:
        for k in ("visl", "visSpectralRadius"):
            out[k] = r[k]
        for k in ("gradTemperatureX", "gradTemperatureY", "gradTemperatureZ"):
            out[k] = r[k].reshape(-1)[:nt]
    if sa:
        out["vist"] = r["vist"]
        out["walldist"] = r["walldist"]
        for k in ("q_turb", "res_turb", "spec_turb", "gradTurbulenceX"):
            out[k] = r[k].reshape(-1)[:nt]
    if ggnode:
        out["qnode"] = r["qnode"]
        if sa:
            out["qTurbNode"] = r["qTurbNode"].reshape(-1)[: m.n_node]
    out["limit"] = r["limit2D"][0]
    out["forces"] = r["forces"]
    path = os.path.join(OUT, name + ".npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path))


def zone_fixture(name, kind, args, params, nsteps, nparts, perturb_seed, turb_seed=None):
    """The reference run on `nparts` zones of the mesh (phenlei_b200.partition:
    slab_owner, then split), all on one rank as the reference runs several
    zones per process, with the reference's interface exchanges.  Stores the
    partition (owner), the input state, the global residual monitor and the
    zones' arrays gathered into global cell order."""
    from oracle.refrun import run_reference_zones
    from phenlei_b200 import partition as P

    m = getattr(M, kind)(**args)
    nc = m.n_cell
    owner = P.slab_owner(m, nparts)
    parts = P.split(m, owner)
    q0 = perturbed_state(m, params, seed=perturb_seed)
    sa = params.get("viscousType", 0) == 3
    state = q0
    if sa:
        state = np.vstack([q0, turb_state(m, params, turb_seed)[None, :]])
    nt = lambda p: p.mesh.n_cell + p.mesh.n_bface  # noqa: E731
    ncz = lambda p: p.mesh.n_cell  # noqa: E731
    dumps = [("q", 5, nt), ("res", 5, nt), ("dt", 0, nt), ("limit2D", 5, nt), ("gradPrimtiveVarX", 5, nt)]
    if sa:
        dumps += [("q_turb", 1, nt), ("vist", 0, nt), ("walldist", 0, ncz)]
    r = run_reference_zones(parts, params, nsteps, dumps=dumps, states=[state[:, p.cells] for p in parts])
    out = {"params": json.dumps(params), "mesh": json.dumps({"kind": kind, "args": args}), "nsteps": nsteps,
           "nparts": nparts, "owner": owner.astype(np.int32), "state_in": state, "res_hist": r["res_hist"]}
    gathered = {"q": np.zeros((5, nc)), "res": np.zeros((5, nc)), "dt": np.zeros(nc), "limit": np.zeros(nc),
                "gradPrimtiveVarX": np.zeros((5, nc))}
    if sa:
        gathered.update(q_turb=np.zeros(nc), vist=np.zeros(nc), walldist=np.zeros(nc))
    forces = np.zeros(16)
    for part, z in zip(parts, r["zones"]):
        c, n = part.cells, part.mesh.n_cell
        gathered["q"][:, c] = z["q"][:, :n]
        gathered["res"][:, c] = z["res"][:, :n]
        gathered["dt"][c] = z["dt"][:n]
        gathered["limit"][c] = z["limit2D"][0, :n]
        gathered["gradPrimtiveVarX"][:, c] = z["gradPrimtiveVarX"][:, :n]
        if sa:
            gathered["q_turb"][c] = z["q_turb"].reshape(-1)[:n]
            gathered["vist"][c] = z["vist"][:n]
            gathered["walldist"][c] = z["walldist"][:n]
        forces += z["forces"]
    out.update(gathered)
    out["forces"] = forces
    path = os.path.join(OUT, name + ".npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path))


if __name__ == "__main__":
    only = sys.argv[1:]
    if only:
        _fixture = fixture

        def fixture(name, *a, **k):  # noqa: F811 - regenerate the named fixtures only
            if name in only:
                _fixture(name, *a, **k)

        _zone_fixture = zone_fixture

        def zone_fixture(name, *a, **k):  # noqa: F811
            if name in only:
                _zone_fixture(name, *a, **k)
    # Euler bump, seeded perturbation, one iteration: every intermediate array.
    fixture("euler_bump_16x8x2_step1", "channel_bump", {"nx": 16, "ny": 8, "nz": 2}, EULER_BUMP, 1, perturb_seed=7)
    # Euler bump from the free stream, 40 iterations through the CFL ramp.
    fixture("euler_bump_16x8x2_step40", "channel_bump", {"nx": 16, "ny": 8, "nz": 2}, EULER_BUMP, 40)
    # Euler on a jittered tetrahedral cube (all far field), perturbed, 3 iterations.
    fixture("euler_tetcube_4_step3", "tet_cube", {"n": 4, "jitter": 0.15, "seed": 3},
            dict(EULER_BUMP, refMachNumber=0.3), 3, perturb_seed=11)
    # Laminar bump (no-slip adiabatic walls), LSQ gradient, perturbed, one iteration.
    fixture("laminar_bump_16x8x2_lsq_step1", "channel_bump", {"nx": 16, "ny": 8, "nz": 2},
            dict(LAMINAR, gradientName="lsq"), 1, perturb_seed=7)
    # Laminar bump, GG-cell gradient, 20 iterations from the free stream.
    fixture("laminar_bump_16x8x2_step20", "channel_bump", {"nx": 16, "ny": 8, "nz": 2}, LAMINAR, 20)
    # Laminar jittered tetrahedra (the laminar cube's element type), LSQ, perturbed, 3 iterations.
    fixture("laminar_tetcube_4_lsq_step3", "tet_cube", {"n": 4, "jitter": 0.15, "seed": 3},
            dict(LAMINAR, gradientName="lsq"), 3, perturb_seed=11)
    # SA bump, perturbed flow and nu~ (negative cells included), one iteration.
    fixture("sa_bump_16x8x2_step1", "channel_bump", {"nx": 16, "ny": 8, "nz": 2}, SA, 1, perturb_seed=7,
            turb_seed=5)
    # SA bump, LSQ, perturbed, 3 iterations.
    fixture("sa_bump_16x8x2_lsq_step3", "channel_bump", {"nx": 16, "ny": 8, "nz": 2},
            dict(SA, gradientName="lsq"), 3, perturb_seed=9, turb_seed=6)
    # SA bump on the mixed hex / prism mesh (3 prism layers at the walls), perturbed, 2 iterations.
    fixture("sa_bump_prism_16x8x2_step2", "channel_bump", {"nx": 16, "ny": 8, "nz": 2, "prism_layers": 3}, SA, 2,
            perturb_seed=8, turb_seed=4)
    # GG-node gradient (the reference's default gradientName): Euler bump, perturbed, one iteration.
    fixture("euler_bump_16x8x2_ggnode_step1", "channel_bump", {"nx": 16, "ny": 8, "nz": 2},
            dict(EULER_BUMP, gradientName="ggnode"), 1, perturb_seed=7)
    # GG-node, laminar bump (wall, far-field and symmetry nodes), perturbed, one iteration.
    fixture("laminar_bump_16x8x2_ggnode_step1", "channel_bump", {"nx": 16, "ny": 8, "nz": 2},
            dict(LAMINAR, gradientName="ggnode"), 1, perturb_seed=7)
    # GG-node, laminar bump from the free stream, 20 iterations.
    fixture("laminar_bump_16x8x2_ggnode_step20", "channel_bump", {"nx": 16, "ny": 8, "nz": 2},
            dict(LAMINAR, gradientName="ggnode"), 20)
    # GG-node on jittered tetrahedra (all far field), perturbed, 3 iterations.
    fixture("euler_tetcube_4_ggnode_step3", "tet_cube", {"n": 4, "jitter": 0.15, "seed": 3},
            dict(EULER_BUMP, refMachNumber=0.3, gradientName="ggnode"), 3, perturb_seed=11)
    # GG-node with SA: perturbed flow and nu~, one iteration; and 20 iterations from the free stream.
    fixture("sa_bump_16x8x2_ggnode_step1", "channel_bump", {"nx": 16, "ny": 8, "nz": 2},
            dict(SA, gradientName="ggnode"), 1, perturb_seed=7, turb_seed=5)
    fixture("sa_bump_16x8x2_ggnode_step20", "channel_bump", {"nx": 16, "ny": 8, "nz": 2},
            dict(SA, gradientName="ggnode"), 20)
    # SA bump from the free stream, 30 iterations.
    fixture("sa_bump_16x8x2_step30", "channel_bump", {"nx": 16, "ny": 8, "nz": 2}, SA, 30)
    # The other inviscid schemes of the dispatcher (Flux_Inviscid.cpp:88-134): Euler bump, perturbed,
    # 3 iterations; and a supersonic free stream (M = 1.6) through jittered tetrahedra, perturbed,
    # 2 iterations, so the supersonic branches of each splitting run.
    for scheme, tag in (("steger", "steger"), ("vanleer", "vanleer"), ("hlle", "hlle"), ("ausmdv", "ausmdv"),
                        ("ausmpw+", "ausmpwp"), ("ausmpw", "ausmpw"), ("vanleer_Rotate", "vanleerrot")):
        fixture(f"euler_bump_16x8x2_{tag}_step3", "channel_bump", {"nx": 16, "ny": 8, "nz": 2},
                dict(EULER_BUMP, uns_scheme_name=scheme), 3, perturb_seed=7)
        fixture(f"euler_tetcube_4_{tag}_m16_step2", "tet_cube", {"n": 4, "jitter": 0.15, "seed": 3},
                dict(EULER_BUMP, uns_scheme_name=scheme, refMachNumber=1.6), 2, perturb_seed=11, amplitude=0.1)
    # Flow initialisation (flowInitStep > 0: first order, zero limiter, Van Leer flux): inside the phase
    # only; across its end (laminar); with no limiter (nolim keeps limit2D = 1 but still skips the
    # reconstruction); and with SA.
    fixture("euler_bump_16x8x2_init5_step2", "channel_bump", {"nx": 16, "ny": 8, "nz": 2},
            dict(EULER_BUMP, flowInitStep=5), 2, perturb_seed=7)
    fixture("laminar_bump_16x8x2_init3_step5", "channel_bump", {"nx": 16, "ny": 8, "nz": 2},
            dict(LAMINAR, flowInitStep=3), 5, perturb_seed=7)
    fixture("euler_bump_16x8x2_nolim_init2_step3", "channel_bump", {"nx": 16, "ny": 8, "nz": 2},
            dict(EULER_BUMP, uns_limiter_name="nolim", flowInitStep=2), 3, perturb_seed=7)
    fixture("sa_bump_16x8x2_init2_step3", "channel_bump", {"nx": 16, "ny": 8, "nz": 2},
            dict(SA, flowInitStep=2), 3, perturb_seed=7, turb_seed=5)
    # The other unstructured limiters (GetLimiterID, Limiter.cpp:1279-1300): Barth-Jespersen from rho and p
    # (bump, laminar LSQ bump, jittered tetrahedra), and "1st" (first order at every step, Roe flux).
    fixture("euler_bump_16x8x2_barth_step3", "channel_bump", {"nx": 16, "ny": 8, "nz": 2},
            dict(EULER_BUMP, uns_limiter_name="barth"), 3, perturb_seed=7)
    fixture("laminar_bump_16x8x2_barth_lsq_step2", "channel_bump", {"nx": 16, "ny": 8, "nz": 2},
            dict(LAMINAR, uns_limiter_name="barth", gradientName="lsq"), 2, perturb_seed=7)
    fixture("euler_tetcube_4_barth_step2", "tet_cube", {"n": 4, "jitter": 0.15, "seed": 3},
            dict(EULER_BUMP, uns_limiter_name="barth", refMachNumber=0.3), 2, perturb_seed=11)
    fixture("euler_bump_16x8x2_1st_step3", "channel_bump", {"nx": 16, "ny": 8, "nz": 2},
            dict(EULER_BUMP, uns_limiter_name="1st"), 3, perturb_seed=7)
    # The SA flat plate flow on a small plate (no-slip plate after a symmetry lead-in): SA, M 0.2, Re 5e6,
    # T 300 K, AUSMPW+ (the unstructured dispatcher has no AUSM+), CFL 50; perturbed flow and nu~,
    # 2 iterations; and 20 iterations from the free stream.
    fixture("sa_plate_16x8x2_ausmpwp_step2", "flat_plate", {"nx": 16, "ny": 8, "nz": 2, "first_spacing": 1e-4},
            SA_PLATE, 2, perturb_seed=7, turb_seed=5)
    fixture("sa_plate_16x8x2_ausmpwp_step20", "flat_plate", {"nx": 16, "ny": 8, "nz": 2, "first_spacing": 1e-4},
            SA_PLATE, 20)
    # Partitioned grids: the reference's own run on 2 and 3 zones of the bump (slab
    # partition), interface exchanges between the zones, 10 iterations.
    zone_fixture("zones2_euler_bump_16x8x2_step10", "channel_bump", {"nx": 16, "ny": 8, "nz": 2}, EULER_BUMP, 10,
                 2, perturb_seed=3)
    zone_fixture("zones3_laminar_bump_16x8x2_lsq_step10", "channel_bump", {"nx": 16, "ny": 8, "nz": 2},
                 dict(LAMINAR, gradientName="lsq"), 10, 3, perturb_seed=5)
    zone_fixture("zones2_euler_bump_16x8x2_barth_ktmax_step10", "channel_bump", {"nx": 16, "ny": 8, "nz": 2},
                 dict(EULER_BUMP, uns_limiter_name="barth", ktmax=1.5), 10, 2, perturb_seed=7)
    zone_fixture("zones2_sa_bump_16x8x2_step10", "channel_bump", {"nx": 16, "ny": 8, "nz": 2}, SA, 10, 2,
                 perturb_seed=7, turb_seed=9)
    zone_fixture("zones3_sa_bump_16x8x2_prism_step5", "channel_bump", {"nx": 16, "ny": 8, "nz": 2, "prism_layers": 3},
                 SA, 5, 3, perturb_seed=11, turb_seed=13)
