"""Runs the reference solver (oracle/_ref/ref_harness, built by
oracle/refbuild/Makefile from the reference's own sources) on an in-memory
grid and returns the arrays it dumps.  Test infrastructure: used only to
generate and check golden fixtures in the container that holds the
reference sources; nothing on the product path imports it.

Parameters are given as hypara key/value pairs on top of the reference's
default parameter file (PHengLEI/examples/bin/cfd_para.hypara in the reference
project, staged as oracle/_ref/cfd_para.hypara by oracle/refbuild/Makefile).
"""
from __future__ import annotations

import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
HARNESS = os.path.join(HERE, "_ref", "ref_harness")
# the reference's default parameter file, staged beside the harness by the build
DEFAULT_PARA = os.path.join(HERE, "_ref", "cfd_para.hypara")


def available() -> bool:
    """True when the reference build (harness and its default parameter file) is present."""
    return os.path.exists(HARNESS) and os.path.exists(DEFAULT_PARA)


def _fmt(key, val):
    if isinstance(val, str):
        return f'string {key} = "{val}";'
    if isinstance(val, (bool, int, np.integer)):
        return f"int {key} = {int(val)};"
    return f"double {key} = {float(val)!r};"


# Settings every oracle run shares: a single grid level, no file output, the
# flow initialisation phase off (the product and the oracle both start second
# order from the first step), residual/force monitors every step.
BASE_PARAMS = {
    "ndim": 3, "nsimutask": 0, "maxSimuStep": 1000000, "intervalStepFlow": 100000000,
    "intervalStepPlot": 100000000, "intervalStepSample": 100000000,
    "intervalStepForce": 100000000, "intervalStepRes": 100000000,
    "flowInitStep": 0, "nMGLevel": 1, "gridfile": "./grid/inmemory.fts",
    "isPlotVolumeField": 0, "numberOfGridProcessor": 0,
}


def run_reference(mesh, params: dict, nsteps: int, dumps=(), state=None, workdir=None, wall_dist=None):
    """Run `nsteps` outer iterations of the reference solver.

    dumps: iterable of (name, rows, cols) grid arrays to return.
    state: optional primitive field [nEq, nCell] (plus turbulence rows) that
    replaces the reference's own initial field.
    wall_dist: optional wall distance [nCell] that replaces the reference's
    own wall-distance search (used by the timing runs, whose set-up it shortens).
    Returns a dict of numpy arrays (dumped arrays, geometry, residual history).
    """
    from phenlei_b200.mesh import write_mesh

    if not available():
        raise RuntimeError("oracle/_ref/ref_harness is not built (make -C oracle/refbuild REF=<root> all harness)")
    tmp = os.path.abspath(workdir or tempfile.mkdtemp(prefix="phx_ref_"))
    os.makedirs(os.path.join(tmp, "bin"), exist_ok=True)
    os.makedirs(os.path.join(tmp, "grid"), exist_ok=True)
    os.makedirs(os.path.join(tmp, "results"), exist_ok=True)
    os.makedirs(os.path.join(tmp, "out"), exist_ok=True)
    p = dict(BASE_PARAMS)
    p.update(params)
    with open(os.path.join(tmp, "bin", "key.hypara"), "w") as f:
        f.write('string title = "oracle";\n')
        f.write(f'string defaultParaFile = "{DEFAULT_PARA}";\n')
        f.write("int ndim = 3;\nint nparafile = 1;\nint nsimutask = 0;\n")
        f.write('string parafilename = "./bin/case.hypara";\nint numberOfGridProcessor = 0;\n')
    with open(os.path.join(tmp, "bin", "case.hypara"), "w") as f:
        for k, v in p.items():
            f.write(_fmt(k, v) + "\n")
    with open(os.path.join(tmp, "bin", "boundary_condition.hypara"), "w") as f:
        f.write("int nBoundaryConditions = 0;\n")
    mpath = os.path.join(tmp, "grid", "mesh.bin")
    write_mesh(mpath, mesh)
    spath = "-"
    if state is not None:
        spath = os.path.join(tmp, "grid", "state.bin")
        np.ascontiguousarray(state, dtype="<f8").tofile(spath)
    args = [HARNESS, mpath, tmp, os.path.join(tmp, "out"), str(nsteps), spath]
    args += [f"{n}:{r}:{c}" for (n, r, c) in dumps]
    env = dict(os.environ)
    env.pop("PHX_REF_WALLDIST", None)
    if wall_dist is not None:
        wpath = os.path.join(tmp, "grid", "walldist.bin")
        np.ascontiguousarray(wall_dist, dtype="<f8").tofile(wpath)
        env["PHX_REF_WALLDIST"] = wpath
    proc = subprocess.run(args, capture_output=True, text=True, env=env)
    if proc.returncode != 0:
        raise RuntimeError(f"reference harness failed ({proc.returncode}):\n{proc.stdout[-4000:]}\n{proc.stderr[-4000:]}")
    out = {}
    odir = os.path.join(tmp, "out")
    for fn in os.listdir(odir):
        if fn.endswith(".bin"):
            out[fn[:-4]] = np.fromfile(os.path.join(odir, fn), dtype="<f8")
    for (n, r, c) in dumps:
        if n in out and r > 0:
            out[n] = out[n].reshape(r, c)
    out["_log"] = proc.stdout
    return out
