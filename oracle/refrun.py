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
# the same harness over the reference built with its OpenMP loops over zones
# (make -C oracle/refbuild OMP=1 ...): one zone per thread
HARNESS_OMP = os.path.join(HERE, "_ref", "ref_harness_omp")
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
    # NSSolver::ComputeCFL (CFD/NSSolver/src/NSSolver.cpp:619-626) inserts CFLMethod = 0
    # into the global parameter map when the key is absent.  In the OpenMP build that
    # insert runs from every zone thread at once (Controller::TimeStep's parallel zone
    # loop) and races on the map; it crashed a few percent of 8-thread runs.  The key
    # set here has the same value and leaves the threads read-only lookups.
    "CFLMethod": 0,
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


def interface_arrays(parts):
    """Per part, the interface data a partitioned grid file of the reference
    holds for a zone (IO_HDF5Read::ReadInterfaceInfo,
    API/PreProcess/src/Pre_HDF5File.cpp:1366-1401): for each interface face k
    (the part's boundary faces iface_first + k), the neighbouring zone, the
    index of the same face in that zone's interface list, and the boundary
    face number."""
    index = []
    for part in parts:
        g = part.faces[part.iface_first:part.iface_first + part.n_iface]
        index.append({int(f): k for k, f in enumerate(g)})
    out = []
    for part in parts:
        n = part.n_iface
        g = part.faces[part.iface_first:part.iface_first + n]
        zone = np.empty(n, np.int32)
        for q, other in enumerate(parts):
            if q != part.rank:
                hit = np.array([int(f) in index[q] for f in g], bool)
                zone[hit] = q
        inter = np.array([index[zone[k]][int(g[k])] for k in range(n)], np.int32)
        out.append((zone, inter, np.arange(part.iface_first, part.iface_first + n, dtype=np.int32)))
    return out


def run_reference_zones(parts, params: dict, nsteps: int, dumps=(), states=None, workdir=None, threads=0,
                        wall_dists=None):
    """`nsteps` outer iterations of the reference solver on the zones `parts`
    (phenlei_b200.partition.split), all in one process as the reference runs
    several zones on one rank.  dumps: (name, rows, cols) per zone, where
    cols may be a callable of the part.  states: per zone the input field as
    for run_reference.  threads > 0 runs the OpenMP build of the reference with
    that many threads (its loops over zones run in parallel).  wall_dists: per
    zone wall distances that replace the reference's search.  Returns
    {"res_hist": global monitor, "zones": [dict per zone], "loop_s": the
    iteration loop's wall time}."""
    from phenlei_b200.mesh import write_mesh

    if not available():
        raise RuntimeError("oracle/_ref/ref_harness is not built (make -C oracle/refbuild REF=<root> all harness)")
    tmp = os.path.abspath(workdir or tempfile.mkdtemp(prefix="phx_ref_zones_"))
    for d in ("bin", "grid", "results", "out"):
        os.makedirs(os.path.join(tmp, d), exist_ok=True)
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
    mpaths, spaths = [], []
    for part, (zone, inter, bface) in zip(parts, interface_arrays(parts)):
        mp = os.path.join(tmp, "grid", f"zone{part.rank}.bin")
        write_mesh(mp, part.mesh)
        with open(mp + ".itf", "wb") as f:
            np.array([len(zone)], "<i8").tofile(f)
            for a in (zone, inter, bface):
                np.ascontiguousarray(a, "<i4").tofile(f)
        mpaths.append(mp)
        if states is not None:
            sp = os.path.join(tmp, "grid", f"state{part.rank}.bin")
            np.ascontiguousarray(states[part.rank], dtype="<f8").tofile(sp)
            spaths.append(sp)
    spec = []
    for (n, r, c) in dumps:
        spec.append((n, r, c))
    # the dump sizes differ per zone: dump the largest and cut per zone
    harness = HARNESS
    if threads > 0:
        if not os.path.exists(HARNESS_OMP):
            raise RuntimeError("oracle/_ref/ref_harness_omp is not built (make -C oracle/refbuild OMP=1 ...)")
        harness = HARNESS_OMP
    args = [harness, ",".join(mpaths), tmp, os.path.join(tmp, "out"), str(nsteps), ",".join(spaths) or "-"]
    sizes = {}
    for (n, r, c) in spec:
        cmax = max(c(part) for part in parts) if callable(c) else c
        sizes[n] = (r, c)
        args.append(f"{n}:{r}:{cmax}")
    env = dict(os.environ)
    env.pop("PHX_REF_WALLDIST", None)
    if threads > 0:
        env["OMP_NUM_THREADS"] = str(threads)
    if wall_dists is not None:
        wpaths = []
        for part in parts:
            wp = os.path.join(tmp, "grid", f"walldist{part.rank}.bin")
            np.ascontiguousarray(wall_dists[part.rank], dtype="<f8").tofile(wp)
            wpaths.append(wp)
        env["PHX_REF_WALLDIST"] = ",".join(wpaths)
    proc = subprocess.run(args, capture_output=True, text=True, env=env)
    if proc.returncode != 0:
        raise RuntimeError(f"reference harness failed ({proc.returncode}):\n{proc.stdout[-4000:]}\n{proc.stderr[-4000:]}")
    res = {"res_hist": np.fromfile(os.path.join(tmp, "out", "res_hist.bin"), dtype="<f8"), "zones": [],
           "loop_s": float(np.fromfile(os.path.join(tmp, "out", "iter_seconds.bin"), dtype="<f8")[0]),
           "_log": proc.stdout}
    for part in parts:
        zdir = os.path.join(tmp, "out", f"zone{part.rank}")
        z = {}
        for fn in os.listdir(zdir):
            if fn.endswith(".bin"):
                z[fn[:-4]] = np.fromfile(os.path.join(zdir, fn), dtype="<f8")
        for n, (r, c) in sizes.items():
            if n in z:
                cz = c(part) if callable(c) else c
                cmax = z[n].size // max(r, 1)
                z[n] = z[n].reshape(r, cmax)[:, :cz] if r > 0 else z[n][:cz]
        res["zones"].append(z)
    return res
