"""The benchmark cases: hypara keys and initial states.

Synthetic, seeded stand-ins with the shapes, sizes and flow parameters of the
benchmark cases (no external grids or data are used; the meshes come from
phenlei_b200.mesh):

* ``EULER_BUMP``  inviscid 3-D channel, 10% circular-arc bump, 64x32x4 hexes
* ``LAMINAR``     laminar NS (with gradientName "lsq" on the 100^3 x 6 jittered
                  tetrahedral cube), free stream plus seeded sinusoids
* ``SA_PLATE``    Spalart-Allmaras flat plate, 512x192x32 hexes, M 0.2, Re 5e6;
                  with sa_source "mlp_fallback" it runs the learned source, and
                  ``SA_PLATE_UNSEEN`` (M 0.3, Re 3e6) tests its generalisation
* ``SA_BUMP``     transonic channel bump, 16M hex / prism cells, M 0.8, Re 1e7
"""
from __future__ import annotations

import math

import numpy as np

from . import mesh as M

EULER_BUMP = {"viscousType": 0, "uns_scheme_name": "roe", "uns_limiter_name": "vencat", "ivencat": 7,
              "venkatCoeff": 5.0, "gradientName": "ggcell", "reconmeth": 1, "roeEntropyFixMethod": 3,
              "tscheme": 4, "nLUSGSSweeps": 1, "CFLStart": 0.01, "CFLEnd": 10.0, "CFLVaryStep": 500,
              "refMachNumber": 0.5, "attackd": 0.0, "refGama": 1.4, "flowInitStep": 0}

# Laminar NS (the laminar cube's keys): Sutherland viscosity, Re 1e4 per unit length,
# adiabatic no-slip walls.
LAMINAR = dict(EULER_BUMP, viscousType=1, refMachNumber=0.3, refReNumber=1.0e4, refDimensionalTemperature=288.15,
               prl=0.72, wallTemperature=-1.0)

# Transonic bump flow, Spalart-Allmaras, Re 1e7 per unit length.
SA_BUMP = dict(EULER_BUMP, viscousType=3, refMachNumber=0.8, refReNumber=1.0e7, refDimensionalTemperature=288.15,
               prl=0.72, prt=0.9, wallTemperature=-1.0, muoo=3.0, CFLEnd=20.0)


# SA flat plate, M 0.2, Re 5e6 per unit length, T_inf 300 K, adiabatic
# no-slip plate, nu~_inf = 3 nu, CFL 50.  AUSM+ is not in the reference's
# unstructured flux dispatcher (Flux_Inviscid.cpp:88-134); AUSMPW+ stands in.
SA_PLATE = dict(EULER_BUMP, viscousType=3, refMachNumber=0.2, refReNumber=5.0e6, refDimensionalTemperature=300.0,
                prl=0.72, prt=0.9, wallTemperature=-1.0, muoo=3.0, uns_scheme_name="ausmpw+", CFLEnd=50.0)

# The learned source's unseen flow: the same plate at M 0.3, Re 3e6.
SA_PLATE_UNSEEN = dict(SA_PLATE, refMachNumber=0.3, refReNumber=3.0e6)


def freestream(params: dict) -> np.ndarray:
    """Non-dimensional free-stream primitive state (PerfectGas::ComputeReferencePrimitive,
    API/Physics/src/PerfectGas.cpp:1276-1302)."""
    g = params.get("refGama", 1.4)
    mach = params.get("refMachNumber", 0.73)
    a = math.radians(params.get("attackd", 0.0))
    b = math.radians(params.get("angleSlide", 0.0))
    return np.array([1.0, math.cos(a) * math.cos(b), math.sin(a) * math.cos(b), math.sin(b), 1.0 / (g * mach * mach)])


def cell_centres(m) -> np.ndarray:
    """Node-average cell centres (for seeding fields only)."""
    off = m.cell_offsets()
    cnt = np.diff(off)
    idx = np.repeat(np.arange(m.n_cell), cnt)
    c = np.zeros((m.n_cell, 3))
    for k, a in enumerate((m.x, m.y, m.z)):
        c[:, k] = np.bincount(idx, weights=a[m.cell2node], minlength=m.n_cell) / cnt
    return c


def perturbed_state(m, params: dict, seed: int = 0, amplitude: float = 0.02, modes: int = 3) -> np.ndarray:
    """Free stream plus seeded random-phase sinusoids: `modes` wavenumbers per
    axis, relative amplitude `amplitude` on each of rho, u, v, w, p (u, v, w
    scaled by the free-stream speed)."""
    rng = np.random.default_rng(seed)
    q0 = freestream(params)
    c = cell_centres(m)
    lo, hi = c.min(axis=0), c.max(axis=0)
    span = np.maximum(hi - lo, 1e-12)
    x = (c - lo) / span
    q = np.empty((5, m.n_cell))
    for v in range(5):
        f = np.zeros(m.n_cell)
        for ax in range(3):
            for k in range(1, modes + 1):
                f += np.sin(2.0 * math.pi * k * x[:, ax] + rng.uniform(0.0, 2.0 * math.pi)) / (3.0 * modes)
        scale = q0[v] if v in (0, 4) else 1.0
        q[v] = q0[v] + amplitude * scale * f * 3.0
    return q
