"""Throughput benchmark of the phx per-iteration path on one or more B200s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl phx|reference]
                    [--workload NAME] [--precision fp64|mixed]

One "step" is one outer iteration of the solver (Controller::Relaxation with
LU-SGS) over the whole mesh.  `value` is Mcell-iterations/s with the state
resident in HBM (CUDA events on the library's stream, max over ranks);
`e2e` is the same metric through the public C ABI with the state in pinned
host memory: every step uploads the primitive state, runs the iteration and
downloads the updated state and the residual monitor.

Multi-GPU (N ranks, one per GPU): domain decomposition with weak scaling.
Rank r builds zone r of a channel N times the workload's length (the
workload's own mesh per rank, its x extent and cell count times N for the
whole job), with interface faces at the cuts, and steps it phase by phase with
the reference's halo exchanges (phenlei_b200.zones): NCCL point-to-point halos
and all-reduces.  `value` is all ranks' cells x steps over the slowest rank's
device time.  With fewer GPUs than ranks (the halo path on one GPU) the ranks
share it and the rows go through gloo on the host.  Workloads that are not a
channel split their one mesh into N zones by recursive coordinate bisection
instead (strong scaling).

`--impl reference` times the reference's own solver, built from its sources
with its OpenMP loops over zones (oracle/_ref/ref_harness_omp), on a bounded
sample of the same workload split into one zone per host thread; without that
build, one zone on one core (oracle/_ref/ref_harness), and without any build
of the reference, the oracle's single-threaded C restatement of the path.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-iters/s on 1 B200: mixed+MLP-SA vs plain FP64, at |ΔCL|,|ΔCD|≤1e-4"

# Bytes each cell moves per iteration under the compulsory-byte rule (each
# array element counted once per pass that reads or writes it; gathered
# neighbour values counted once per cell; face arrays once per face per pass),
# computed for the kernels below from the arrays each pass reads and writes
# (kernel_bytes lists them per phase).  Element sizes: FP64 metrics 8 B,
# working state 8 B (FP64) or 4 B (mixed), indices 4 B.


def workloads():
    from phenlei_b200 import cases
    from phenlei_b200 import mesh as M

    return {
        # The 16M-cell transonic bump's mesh size and Mach number with inviscid physics.
        "transonic_bump_euler_16M": dict(
            mesh=lambda: M.channel_bump(1024, 92, 128, thickness=0.08, length=3.0, wall_spacing=0.001),
            channel=dict(nx=1024, ny=92, nz=128, thickness=0.08, length=3.0, wall_spacing=0.001),
            params=dict(cases.EULER_BUMP, refMachNumber=0.8, CFLEnd=20.0),
            desc="3-D transonic channel bump 8% thick, 1024x92x128 hex (12.06M cells), M=0.8, Roe+Venkat, "
                 "GG-cell, LU-SGS CFL 20, inviscid"),
        # Mixed hex / prism bump, 1024x92x128 with the 30 wall-adjacent
        # layers as prisms (15,990,784 cells), M=0.8, Re=1e7, SA, Roe + Venkat, CFL 20.
        "transonic_bump_sa_16M": dict(
            mesh=lambda: M.channel_bump(1024, 92, 128, thickness=0.08, length=3.0, wall_spacing=0.001,
                                        prism_layers=30),
            channel=dict(nx=1024, ny=92, nz=128, thickness=0.08, length=3.0, wall_spacing=0.001, prism_layers=30),
            params=dict(cases.SA_BUMP),
            wall_dist=True,
            desc="3-D transonic channel bump 8% thick, 1024x92x128 with 30 prism layers at the walls "
                 "(15.99M hex+prism cells), M=0.8, Re=1e7, Spalart-Allmaras, Roe+Venkat, GG-cell, LU-SGS CFL 20"),
        "sa_bump_1M": dict(
            mesh=lambda: M.channel_bump(256, 92, 32, thickness=0.08, wall_spacing=0.001, prism_layers=30),
            channel=dict(nx=256, ny=92, nz=32, thickness=0.08, length=3.0, wall_spacing=0.001, prism_layers=30),
            params=dict(cases.SA_BUMP),
            wall_dist=True,
            desc="SA channel bump 256x92x32 with 30 prism layers (1.0M hex+prism cells), M=0.8, Re=1e7"),
        "euler_bump_8k": dict(
            mesh=lambda: M.channel_bump(64, 32, 4),
            params=dict(cases.EULER_BUMP),
            desc="Euler channel bump 64x32x4 hex (8,192 cells), M=0.5"),
        "euler_bump_1M": dict(
            mesh=lambda: M.channel_bump(256, 128, 32),
            channel=dict(nx=256, ny=128, nz=32),
            params=dict(cases.EULER_BUMP),
            desc="Euler channel bump 256x128x32 hex (1.05M cells), M=0.5"),
        # 100^3 hexes x 6 jittered tetrahedra, laminar, least squares.
        "laminar_cube_6M": dict(
            mesh=lambda: M.tet_cube(100, jitter=0.15, seed=1),
            params=dict(cases.LAMINAR, gradientName="lsq"),
            desc="laminar cube, 100^3 hexes x 6 jittered tets (6.0M cells), M=0.3, Re=1e4, LSQ, "
                 "Roe+Venkat, LU-SGS"),
        # SA flat plate 512x192x32 (3.1M hexes), first cell y+ about 1, M 0.2, Re 5e6, AUSMPW+, CFL 50,
        # 5,000 iterations.  Its converged run trains the learned source on its states (2M samples, 20 epochs)
        # and then also runs the unseen flow M 0.3, Re 3e6.
        "sa_plate_3M": dict(
            mesh=lambda: M.flat_plate(512, 192, 32),
            params=dict(cases.SA_PLATE),
            wall_dist=True, iterations=5000, train_epochs=20, unseen=dict(cases.SA_PLATE_UNSEEN),
            desc="SA flat plate 512x192x32 hex (3.15M cells), lead-in 0.33, plate 2, M=0.2, Re=5e6, "
                 "T=300 K, AUSMPW+, Venkat, GG-cell, LU-SGS CFL 50; unseen flow M=0.3, Re=3e6"),
        "sa_plate_200k": dict(
            mesh=lambda: M.flat_plate(128, 96, 16, first_spacing=1e-5),
            params=dict(cases.SA_PLATE),
            wall_dist=True, iterations=5000, train_epochs=20, unseen=dict(cases.SA_PLATE_UNSEEN),
            desc="SA flat plate 128x96x16 hex (197k cells), M=0.2, Re=5e6, AUSMPW+, CFL 50"),
        "laminar_bump_1M": dict(
            mesh=lambda: M.channel_bump(256, 128, 32),
            params=dict(cases.LAMINAR),
            desc="laminar channel bump 256x128x32 hex (1.05M cells), no-slip walls, M=0.3, Re=1e4, GG-cell"),
    }


DEFAULT_WORKLOAD = "transonic_bump_sa_16M"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


# DRAM bytes per cell of one launch of a sweep kernel, mixed precision:
# dram__bytes_read.sum + dram__bytes_write.sum of one ncu --set full capture
# of lusgs_kernel<float> on the 0.999M-cell SA bump (940.16 MB + 95.03 MB).
# Both sweeps read every cell's records once, so a launch's traffic at
# another mesh size is this figure times the cells.
MEASURED_TRAFFIC_PER_CELL = {("lusgs", "mixed"): (940.16e6 + 95.03e6) / 999424}


def kernel_bytes(m, precision: str, viscous: int = 0, gradient: str = "ggcell") -> dict:
    """Algorithmic bytes per launch of each phase under the compulsory-byte rule
    (each array element counted once per pass that reads or writes it; cell
    values gathered through faces counted once per cell; face arrays once per
    face per pass; indices 4 B, FP64 metrics and master state 8 B, working
    state E = 8 B (FP64) or 4 B (mixed)).  The comment above each term names
    the arrays it counts."""
    nc, nb, nf = m.n_cell, m.n_bface, m.n_face
    nt = nc + nb
    L = 2 * (nf - nb) + nb          # cell -> face entries
    E = 8 if precision == "fp64" else 4
    vis = viscous > 0
    sa = viscous == 3
    lsq = gradient == "lsq"
    out = {}
    # NS boundary: owner master state + normal -> ghost master state + working record (5 + c2, hm)
    bnd = nb * (5 * 8 + 3 * 8 + 4 + 5 * 8 + 7 * E) + (nb * E if sa else 0)
    out["boundary"] = bnd
    # gradient + limiter: working state of cells and ghosts, per face normal*area (GG) or weight + centres (LSQ),
    # face centre (limiter), lr, c2f; cell centre, volume, volpow (+ LSQ matrix); writes gradients + limiter
    nvar = 6 if vis else 5
    g = nt * (5 * E) + nf * (4 * 8 + 3 * 8 + 8) + (L + nc + 1) * 4 + nc * (4 * 8 + 8) + nc * (3 * nvar * E + E)
    if lsq:
        g += nt * 3 * 8 + nc * 6 * 8 + nf * 8
    if sa:
        g += nc * E
    out["gradient_limiter"] = g
    # face pass: state + limiter of both sides (once per cell), gradients, cell centres, face geometry and lr;
    # writes face flux (5 + spectral parts) and the MXDQ factors of each face use (3 + viscous term)
    fp = nt * 6 * E + nc * 15 * E + nt * 3 * 8 + nf * (7 * 8 + 8) + nf * 6 * E + L * (3 + (1 if vis else 0)) * E
    if vis:
        fp += nc * 3 * E + nf * (4 + 1) * E + nf * 1
    if sa:
        fp += nt * E
    # cell pass: face fluxes through c2f + lr, skew, volume, pressure; writes residual, spectral radii, dt
    cp = nf * 6 * E + (L + nc + 1) * 4 + nf * 4 + nc * (8 + 8 + E) + nc * (8 * E)
    if vis:
        cp += nf * 5 * E
    out["residual"] = fp + cp
    # LU-SGS, two sweeps: per entry neighbour / face / factor indices and the factors, face normal + area,
    # neighbour state (u v w c2 hm) and dq once per cell per sweep, own res + spectral radii + dt + volume,
    # dq / delta-flux writes and reads, and the sentinel fill of the three 8-slot write-once records
    lu = (L * 3 * 4 + L * 4 * E + 2 * nf * 4 * 8 + 2 * nc * 5 * E + 2 * nc * 5 * E
          + 2 * nc * (7 * E + E + 8) + 2 * nc * 5 * E + 2 * nc * 5 * E + 3 * nc * 8 * E)
    out["lusgs"] = lu
    # update: FP64 master state in and out (ghosts copied), dq, residual (monitor); working record out
    out["update"] = nc * (5 * 8 + 5 * E + 5 * E + 5 * 8 + 7 * E) + nb * 2 * 5 * 8 + bnd
    if sa:
        sb = nb * (8 + 2 * E + 5 * 8 + 3 * 8 + 4 + 8 + 2 * E)
        vg = nt * E + nc * (2 * E + E) + nf * (4 * 8 + 8) + (L + nc + 1) * 4 + nc * 4 * 8 + nc * (E + 3 * E)
        sf = nt * (4 * E + 3 * E + 4 * 8) + nf * (7 * 8 + 8) + nf * 6 * E + L * E
        sc = nc * (6 * E + 3 * E + 3 * E + E + 8 + E + 8) + nf * 6 * E + (L + nc + 1) * 4 + nf * 4 + nc * 2 * E
        out["sa_residual"] = 2 * sb + vg + sf + sc
        out["sa_lusgs"] = L * 2 * 4 + L * E + 2 * nc * 2 * E + 2 * nc * E + 2 * nc * E + 2 * nc * E + 3 * nc * E
        out["sa_update"] = nc * (8 + E + 8 + E) + sb
    out["iteration"] = sum(out.values())
    return out


def minimal_bytes(m, precision: str, viscous: int = 0, gradient: str = "ggcell") -> int:
    """Compulsory bytes of one iteration of the minimal pass structure: P1
    gradient, P2 limiter, P3 face residual (reconstruction, inviscid and
    viscous fluxes, spectral radii, time step), P4 SA source and diagonal,
    P5/P6 the LU-SGS sweeps, P7 the update, and the SA passes alike.  Only
    the algorithm's arrays count, no record of this implementation (face-flux
    records, LU-SGS factors, sentinels): each array element once per pass that
    reads or writes it, cell values gathered through faces once per cell,
    face metrics (unit normal, area, left/right cell, centre where used) once
    per face per pass, cell-to-face indices once per sweep.  Element sizes:
    FP64 metrics and the conservative master state 8 B; state, gradient,
    limiter, dq, residual 8 B (FP64) or 4 B (mixed); indices 4 B."""
    nc, nb, nf = m.n_cell, m.n_bface, m.n_face
    nt = nc + nb
    L = 2 * (nf - nb) + nb
    E = 8 if precision == "fp64" else 4
    vis = viscous > 0
    sa = viscous == 3
    lsq = gradient == "lsq"
    face = nf * (4 * 8 + 2 * 4)               # unit normal, area, left/right
    cen = nf * 3 * 8                          # face centre
    nv = 6 if vis else 5                      # primitives (+ temperature)
    p1 = nt * 5 * E + face + nc * 8 + nc * 3 * nv * E
    if lsq:
        p1 += nf * 8 + nc * 6 * 8 + nt * 3 * 8
    p2 = nt * 2 * E + nc * 6 * E + cen + nf * 2 * 4 + nc * 3 * 8 + nc * E
    p3 = nt * 5 * E + nc * 3 * nv * E + nt * E + face + cen + nt * 3 * 8 + nc * (5 + 2 + 1) * E
    if vis:
        p3 += nt * 2 * E
    sweep = nc * 5 * E + nc * 2 * E + nt * 5 * E + face + L * 4 + nc * 4 + 2 * nc * 5 * E
    p56 = 2 * sweep
    p7 = nc * (5 * 8 + 5 * E + 5 * 8)
    tot = p1 + p2 + p3 + p56 + p7
    if sa:
        # nu~ gradient, source (vorticity from the NS gradient, wall distance) and
        # diagonal, SA face terms, two scalar sweeps, update
        tot += nt * E + face + nc * 8 + nc * 3 * E
        tot += nc * (E + 9 * E + 3 * E + 8 + 8 + E) + nc * 2 * E
        tot += nt * (E + 4 * E + 2 * E) + face + cen + nt * 3 * 8 + nc * E
        tot += 2 * (nc * 2 * E + nt * E + face + L * 4 + nc * 4 + 2 * nc * E)
        tot += nc * (8 + E + 8)
    return tot


def balanced_subsample(f, t, n, seed=0, grid=64):
    """At most n samples, an equal share per occupied bin of a grid over the
    first two features (ln chi, ln s), chosen at random within each bin."""
    rng = np.random.default_rng(seed)
    lo, hi = f[:, :2].min(0), f[:, :2].max(0)
    b = np.clip(((f[:, :2] - lo) / np.maximum(hi - lo, 1e-30) * grid).astype(np.int64), 0, grid - 1)
    order = rng.permutation(len(t))
    key = (b[:, 0] * grid + b[:, 1])[order]
    srt = np.argsort(key, kind="stable")
    ks = key[srt]
    cap = max(1, n // np.unique(ks).size)
    rank = np.arange(len(ks)) - np.searchsorted(ks, ks, side="left")
    sel = order[srt[rank < cap]]
    return f[sel], t[sel]


def run_phx(args, rank, world, precision, m, wd, e2e=True, mlp_blob=None, train=False):
    import torch

    from phenlei_b200 import solver as S

    dev = rank % max(torch.cuda.device_count(), 1)
    torch.cuda.set_device(dev)
    wl = workloads()[args.workload]
    t0 = time.time()
    params = dict(wl["params"])
    if mlp_blob is not None:
        params["sa_source"] = "mlp_fallback"
    s = S.NSSolverUnstruct(m, precision=precision, wall_dist=wd, **params)
    if mlp_blob is not None:
        s.set_mlp_blob(mlp_blob)
    stream = torch.cuda.current_stream()
    s.set_stream(stream.cuda_stream)
    setup_s = time.time() - t0
    nc = m.n_cell
    # warm-up
    s.Relaxation(args.warmup)
    torch.cuda.synchronize()
    # the learned source's training set also holds the early, near-uniform
    # flow: samples after the warm-up (untimed) join those of the final state
    early = s.capture_sa_samples()[:2] if train else None
    # timed region (device): K iterations
    sampler = ClockSampler(dev)
    sampler.start()
    launches0 = s.launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    hist = s.Relaxation(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = s.launches - launches0
    clocks = sampler.stop()
    # per-kernel timing pass (phase entry points, same stream)
    phase_ms = {}
    names = [("boundary", s.Boundary), ("gradient_limiter", s.ComputeGradientAndLimiter),
             ("residual", s.UpdateResiduals), ("lusgs", s.LUSGS), ("update", s.UpdateFlowField)]
    if wl["params"].get("viscousType", 0) == 3:
        names += [("sa_residual", s.TurbUpdateResiduals), ("sa_lusgs", s.TurbLUSGS),
                  ("sa_update", s.TurbUpdateFlowField)]
    reps = max(1, min(args.steps, 10))
    acc = {n: 0.0 for n, _ in names}
    for _ in range(reps):
        s.step = s.step + 1
        for n, fn in names:
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            acc[n] += a.elapsed_time(b)
    phase_ms = {n: v / reps for n, v in acc.items()}
    iters = s.step
    forces = s.AirForceCoef() if params.get("viscousType", 0) > 0 else None
    vist = None
    if params.get("viscousType", 0) == 3:
        # a number measured on a diverged turbulence field is no number
        vist = s.get(S.PHX_VIST)[:nc]
        if not (np.all(np.isfinite(s.get(S.PHX_Q_TURB)[:nc])) and np.all(np.isfinite(vist))):
            raise RuntimeError(f"{precision} run: the SA field is not finite after {s.step} iterations")
    mlp_info = None
    if mlp_blob is not None:
        mlp_info = {"cells_learned": s.mlp_cells()}
    if train:
        # training set of the learned SA source: features and exact targets of
        # this run's state after the warm-up and its current state, subsampled
        # evenly over the (ln chi, ln s) plane (at most 2M samples, an equal
        # share per occupied bin of a 64 x 64 grid, seeded), 60 epochs, batch
        # 8192, Adam lr 1e-3 (the trainer runs on this GPU)
        f, t, _, _ = s.capture_sa_samples()
        f, t = np.concatenate([early[0], f]), np.concatenate([early[1], t])
        early = None
        f, t = balanced_subsample(f, t, 2_000_000, seed=0)
        t1 = time.perf_counter()
        loss = s.train_sa_mlp(f, t, epochs=60, batch=8192, lr=1e-3, seed=0)
        mlp_info = {"samples": int(len(t)), "epochs": 60, "batch": 8192, "final_loss": loss,
                    "train_s": round(time.perf_counter() - t1, 2), "blob": s.mlp_blob()}
    if not e2e:
        res = dict(ms=ms, launches=launches, clocks=clocks, phase_ms=phase_ms, e2e_s=None, nc=nc, mesh=m,
                   hist=hist, setup_s=setup_s, nt=s.nt, forces=forces, mlp=mlp_info, vist=vist, iters=iters)
        s.close()
        return res
    # end-to-end through the C ABI with pinned host buffers
    qh = torch.empty((5, s.nt), dtype=torch.float64).pin_memory()
    qh.copy_(torch.from_numpy(s.get(S.PHX_Q)))
    qptr = qh.data_ptr()
    lib = S.lib()
    hist1 = np.zeros(1)
    e2e_steps = max(1, min(args.steps, 20))
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    for _ in range(e2e_steps):
        s._check(lib.phx_set_state(s.h, S.PHX_Q, qptr, 5 * s.nt), "set_state")
        s._check(lib.phx_ns_relaxation(s.h, 1, hist1.ctypes.data), "relaxation")
        s._check(lib.phx_get_state(s.h, S.PHX_Q, qptr, 5 * s.nt), "get_state")
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t1) / e2e_steps
    res = dict(ms=ms, launches=launches, clocks=clocks, phase_ms=phase_ms, e2e_s=e2e_s, nc=nc, mesh=m,
               hist=hist, setup_s=setup_s, nt=s.nt, forces=forces, mlp=mlp_info, vist=vist, iters=iters)
    s.close()
    return res


def run_zones(args, rank, world, precision, wl, zone, wd, mlp_blob=None, train=False, e2e=True):
    """One arm of the multi-GPU run: this rank's zone stepped with the halo
    exchanges (phenlei_b200.zones.DistributedZone); warm-up, then K timed
    iterations between a barrier and a synchronize on both sides."""
    import torch
    import torch.distributed as dist

    from phenlei_b200 import partition as P
    from phenlei_b200 import solver as S
    from phenlei_b200.zones import DistributedZone

    params = dict(wl["params"])
    if mlp_blob is not None:
        params["sa_source"] = "mlp_fallback"
    t0 = time.time()
    if zone is not None:
        dz = DistributedZone(None, params, wall_dist=wd, precision=precision, part=zone)
    else:
        mesh = wl["mesh"]()
        # strong scaling of one mesh: recursive bisection keeps the cut faces fewer than slabs
        dz = DistributedZone(mesh, params, owner=P.rcb_owner(mesh, world), wall_dist=wd, precision=precision)
    z = dz.zones[0]
    if mlp_blob is not None:
        z.set_mlp_blob(mlp_blob)
    setup_s = time.time() - t0
    dz.iterate(args.warmup)
    torch.cuda.synchronize()
    early = z.capture_sa_samples()[:2] if train else None
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    launches0 = z.launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dist.barrier()
    torch.cuda.synchronize()
    e0.record()
    hist = dz.iterate(args.steps)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = z.launches - launches0
    clocks = sampler.stop()
    timer = {}
    reps = max(1, min(args.steps, 10))
    dz.iterate(reps, timer=timer)
    torch.cuda.synchronize()
    phase_ms = {k: sum(a.elapsed_time(b) for a, b in v) / reps for k, v in timer.items()}
    forces = dz.AirForceCoef() if params.get("viscousType", 0) > 0 else None
    nc = z.mesh.n_cell
    mlp_info = {"cells_learned": z.mlp_cells()} if mlp_blob is not None else None
    if train:
        # the learned source's training set, as on one GPU: every zone's
        # samples after the warm-up and at the end, subsampled evenly over the
        # (ln chi, ln s) plane to a share of the 2M samples, gathered on rank 0,
        # which trains; the model goes to every rank
        f, t, _, _ = z.capture_sa_samples()
        f, t = np.concatenate([early[0], f]), np.concatenate([early[1], t])
        f, t = balanced_subsample(f, t, 2_000_000 // world, seed=rank)
        got = [None] * world
        dist.all_gather_object(got, (f, t))
        blob = [None]
        info = [None]
        if rank == 0:
            f = np.concatenate([g[0] for g in got])
            t = np.concatenate([g[1] for g in got])
            t1 = time.perf_counter()
            loss = z.train_sa_mlp(f, t, epochs=60, batch=8192, lr=1e-3, seed=0)
            blob = [z.mlp_blob()]
            info = [{"samples": int(len(t)), "epochs": 60, "batch": 8192, "final_loss": loss,
                     "train_s": round(time.perf_counter() - t1, 2)}]
        dist.broadcast_object_list(blob, src=0)
        dist.broadcast_object_list(info, src=0)
        mlp_info = dict(info[0], blob=blob[0])
    e2e_s = None
    if e2e:
        # end to end through the public API: every step uploads this zone's
        # primitive state from pinned host memory (and its interface ghosts
        # from the neighbours), runs the iteration and reads the state back
        qh = torch.empty((5, z.nt), dtype=torch.float64).pin_memory()
        qh.copy_(torch.from_numpy(z.get(S.PHX_Q)))
        lib = S.lib()
        steps = max(1, min(args.steps, 20))
        dist.barrier()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        for _ in range(steps):
            z._check(lib.phx_set_state(z.h, S.PHX_Q, qh.data_ptr(), 5 * z.nt), "set_state")
            dz._exchange_state()
            dz.iterate(1)
            z._check(lib.phx_get_state(z.h, S.PHX_Q, qh.data_ptr(), 5 * z.nt), "get_state")
        torch.cuda.synchronize()
        e2e_s = (time.perf_counter() - t1) / steps
    out = dict(ms=ms, launches=launches, clocks=clocks, phase_ms=phase_ms, e2e_s=e2e_s, nc=nc, mesh=z.mesh,
               hist=hist, setup_s=setup_s, nt=z.nt, forces=forces, mlp=mlp_info, iters=z.step,
               cells_total=dz.n_cell_total)
    dz.close()
    return out


def main_zones(args, rank, world, wl):
    """bench.py --gpus N (N > 1): the workload decomposed into N zones."""
    import datetime

    import torch
    import torch.distributed as dist

    from phenlei_b200 import mesh as M
    from phenlei_b200.zones import channel_zone

    ndev = torch.cuda.device_count()
    torch.cuda.set_device(rank % max(ndev, 1))
    backend = "nccl" if ndev >= world else "gloo"
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    # one collective of all ranks first: the halo exchanges that follow are
    # point-to-point batches between neighbours only
    dist.barrier()
    sa = wl["params"].get("viscousType", 0) == 3
    if "channel" in wl:
        # weak scaling: this rank's slab of a channel `world` times as long
        ch = dict(wl["channel"])
        nx, length = ch.pop("nx"), ch.pop("length", 3.0)
        zone = channel_zone(rank, world, nx=nx * world, length=length * world, dz=length / nx, **ch)
        # the zone's own walls: the wall distance of a cell near a cut can
        # differ from the whole channel's (an input field, not a result)
        wd = M.wall_distance(zone.mesh) if sa else None
        scaling, layout = "weak", "channel %d x the workload's length, one %d-cell slab per rank" % (
            world, zone.mesh.n_cell)
    else:
        zone, scaling = None, "strong"
        wd = M.wall_distance(wl["mesh"]()) if sa else None
        layout = "the workload's mesh split into %d parts by recursive coordinate bisection" % world
    r64 = blob = None
    if args.mlp_blob:
        blob = np.load(args.mlp_blob).astype(np.float32)
    if args.precision == "mixed" and not args.no_fp64_arm:
        r64 = run_zones(args, rank, world, "fp64", wl, zone, wd, e2e=False,
                        train=sa and not args.exact_source and blob is None)
        if r64["mlp"]:
            blob = r64["mlp"].pop("blob")
    r = run_zones(args, rank, world, args.precision, wl, zone, wd, mlp_blob=blob)

    def slowest(v):
        t = torch.tensor([v], dtype=torch.float64, device="cuda" if backend == "nccl" else "cpu")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    ms = slowest(r["ms"])
    e2e_s = slowest(r["e2e_s"])
    ms64 = slowest(r64["ms"]) if r64 is not None else None
    tot = r["cells_total"]
    value = tot * args.steps / (ms / 1e3) / 1e6
    peak, peak_kind = measured_peaks()
    kb = kernel_bytes(r["mesh"], args.precision, wl["params"].get("viscousType", 0),
                      wl["params"].get("gradientName", "ggcell"))
    phase = r["phase_ms"]
    dom = max(phase, key=phase.get)
    achieved = kb[dom] / (phase[dom] / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "Mcell-iters/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
        "higher_is_better": True, "scaling": scaling, "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32+f64",
        "data": "synthetic (seeded generated mesh, free-stream start)",
        "config": {"workload": args.workload, "desc": wl["desc"], "cells": tot, "cells_per_rank": r["nc"],
                   "precision": args.precision, "layout": layout,
                   "parallelism": "dp%d domain decomposition (interface halos over %s)" % (
                       world, "NCCL" if backend == "nccl" else "gloo, host-staged: ranks share a GPU"),
                   "l2": "inputs larger than L2 (state %.0f MB per rank)" % (5 * 8 * r["nt"] / 1e6)},
        "gpu_launches": int(r["launches"]),
        "phase_ms": {k: round(v, 4) for k, v in phase.items()},
        "roofline": {"kernel": dom, "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_kind": peak_kind, "algorithmic_bytes": kb[dom],
                     "traffic": None, "rank": 0},
        "clocks": r["clocks"],
        "e2e": {"value": round(tot / e2e_s / 1e6, 3), "unit": "Mcell-iters/s",
                "h2d_bytes_per_step": 5 * 8 * r["nt"] * world, "d2h_bytes_per_step": 5 * 8 * r["nt"] * world},
        "residual_last": float(r["hist"][-1]) if len(r["hist"]) else None,
    }
    if r64 is not None:
        v64 = tot * args.steps / (ms64 / 1e3) / 1e6
        line["fp64_arm"] = {"value": round(v64, 3), "ms_per_step": round(ms64 / args.steps, 4)}
        line["speedup_vs_fp64"] = round(value / v64, 3)
        if r["forces"] and r64["forces"]:
            line["accuracy_vs_fp64"] = {"dCL": abs(r["forces"]["CL"] - r64["forces"]["CL"]),
                                        "dCD": abs(r["forces"]["CD"] - r64["forces"]["CD"]),
                                        "after_iterations": r["iters"]}
    line["config"]["sa_source"] = (("learned (MLP, exact outside its hull)" if blob is not None else "exact")
                                   if sa else None)
    if rank == 0:
        print(json.dumps(line))
    dist.barrier()
    dist.destroy_process_group()


def converge(args, m, wd):
    """The workload's full iteration count for the three arms on one GPU
    (FP64 exact source, mixed exact source, mixed learned source), from the
    free stream.  The learned source is trained on FP64 states captured along
    the FP64 run (early, middle and final), so it sees the flow it meets.
    Reports CL, CD and the residual monitor of every arm at the end, the
    differences of the mixed arms against FP64, and each arm's whole-run
    throughput (CUDA events around the whole run)."""
    import torch

    from phenlei_b200 import solver as S

    torch.cuda.set_device(0)
    wl = workloads()[args.workload]
    params = dict(wl["params"])
    sa = params.get("viscousType", 0) == 3
    n = args.iterations or wl.get("iterations", 3000)
    nc = m.n_cell
    out = {"workload": args.workload, "cells": nc, "iterations": n}

    def run(precision, blob=None, capture_at=()):
        p = dict(params)
        if blob is not None:
            p["sa_source"] = "mlp_fallback"
        s = S.NSSolverUnstruct(m, precision=precision, wall_dist=wd, **p)
        if blob is not None:
            s.set_mlp_blob(blob)
        stream = torch.cuda.current_stream()
        s.set_stream(stream.cuda_stream)
        caps, hist, done, ms = [], [], 0, 0.0
        for stop in sorted(set([c for c in capture_at if 0 < c < n] + [n])):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            hist.append(s.Relaxation(stop - done))
            e1.record(stream)
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
            done = stop
            if stop in capture_at or (capture_at and stop == n):
                caps.append(s.capture_sa_samples()[:2])
        h = np.concatenate(hist)
        f = s.AirForceCoef()
        # skin-friction drag: the viscous parts of the wall force sums, rotated as CD is
        cdf = S.force_coefficients(np.where(np.arange(16) % 2 == 0, f["sums"], 0.0), s.params.attackd,
                                   s.params.angleSlide)["CD"]
        r = {"CL": f["CL"], "CD": f["CD"], "CD_friction": cdf, "res_max": float(np.max(h)), "res_last": float(h[-1]),
             "res_drop_orders": round(float(np.log10(np.max(h) / h[-1])), 3), "ms_per_iter": round(ms / n, 4),
             "mcell_iters_per_s": round(nc * n / (ms / 1e3) / 1e6, 3)}
        if sa:
            r["vist"] = s.get(S.PHX_VIST)[:nc]
        if blob is not None:
            r["cells_learned_per_iteration"] = round(s.mlp_cells() / n, 1)
        blob_out = None
        if caps:
            f_, t_ = np.concatenate([c[0] for c in caps]), np.concatenate([c[1] for c in caps])
            f_, t_ = balanced_subsample(f_, t_, 2_000_000, seed=0)
            epochs = wl.get("train_epochs", 60)
            t1 = time.perf_counter()
            loss = s.train_sa_mlp(f_, t_, epochs=epochs, batch=8192, lr=1e-3, seed=0)
            r["mlp"] = {"samples": int(len(t_)), "epochs": epochs, "final_loss": loss,
                        "train_s": round(time.perf_counter() - t1, 2)}
            blob_out = s.mlp_blob()
        s.close()
        return r, blob_out

    r64, blob = run("fp64", capture_at=(30, n // 10, n) if sa else ())
    arms = {"fp64": r64}
    arms["mixed_exact"], _ = run("mixed")
    if sa:
        arms["mixed_learned"], _ = run("mixed", blob=blob)

    def compare(arms, ref):
        for name, r in arms.items():
            if r is ref:
                continue
            r["dCL_vs_fp64"] = abs(r["CL"] - ref["CL"])
            r["dCD_vs_fp64"] = abs(r["CD"] - ref["CD"])
            r["dCDf_vs_fp64"] = abs(r["CD_friction"] - ref["CD_friction"])
            if sa:
                r["dVIST_rel_vs_fp64"] = float(np.max(np.abs(r["vist"] - ref["vist"])) / np.max(np.abs(ref["vist"])))
            r["speedup_vs_fp64"] = round(r["mcell_iters_per_s"] / ref["mcell_iters_per_s"], 3)
        for r in arms.values():
            r.pop("vist", None)

    compare(arms, r64)
    out["arms"] = arms
    if sa and wl.get("unseen"):
        # the learned source on a flow it was not trained on
        params.clear()
        params.update(wl["unseen"])
        u64, _ = run("fp64")
        unseen = {"fp64": u64}
        unseen["mixed_learned"], _ = run("mixed", blob=blob)
        compare(unseen, u64)
        out["unseen"] = {"flow": {k: wl["unseen"][k] for k in ("refMachNumber", "refReNumber")}, "arms": unseen}
    return out


def cpu_sample(wl_name):
    """The mesh the CPU arms run on: the workload itself when it has about a
    million cells or fewer, else a mesh of the same case kind with about one
    million cells (the reference solves it at about a third of a million
    cell-iterations per second on one core, so the full 16M-cell mesh would
    take minutes per iteration), and a description of it."""
    from phenlei_b200 import mesh as M

    if wl_name == "transonic_bump_sa_16M":
        return (M.channel_bump(256, 92, 32, thickness=0.08, length=3.0, wall_spacing=0.001, prism_layers=30),
                "256x92x32 channel bump with 30 prism layers (999,424 cells): the 16M bump's case kind and layer count")
    if wl_name == "transonic_bump_euler_16M":
        return (M.channel_bump(256, 92, 32, thickness=0.08, length=3.0, wall_spacing=0.001),
                "256x92x32 hex channel bump (753,664 cells), the same case kind")
    if wl_name == "sa_plate_3M":
        return M.flat_plate(256, 96, 16), "256x96x16 flat plate (393,216 cells), the same case kind"
    m = workloads()[wl_name]["mesh"]()
    return m, "the workload's own mesh"


def host_threads() -> int:
    """Host threads this process may run on."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_baseline(args, wl_name, budget_s=25.0):
    """The reference's own CPU solver on a bounded sample of the workload, with
    every host thread it can use: the reference parallelises across zones
    (its OpenMP loops over zones, e.g. Controller::TimeStep,
    CFD/Solver/src/Controller.cpp:684-704), so the sample is split into one
    slab zone per thread and run by oracle/_ref/ref_harness_omp (the reference
    built from its sources with USE_OMP).  Without that build, one zone on one
    core (oracle/_ref/ref_harness); without either, the oracle port
    (single-threaded C restatement, bit-exact with the reference).  The
    throughput is taken over the iteration loop alone."""
    from oracle import refrun
    from phenlei_b200 import mesh as M
    from phenlei_b200 import partition as P

    wl = workloads()[wl_name]
    m, what = cpu_sample(wl_name)
    wd = M.wall_distance(m) if wl.get("wall_dist") else None
    params = dict(wl["params"])
    threads = host_threads()
    if refrun.available() and os.path.exists(refrun.HARNESS_OMP) and threads > 1:
        parts = P.split(m, P.slab_owner(m, threads))
        # about 0.35 Mcell-iterations/s on one thread, each further thread adding about 0.15 of that
        # (the reference threads only some of its loops over zones): as many iterations as fit the
        # budget, at least 2
        n = int(max(2, min(args.steps, budget_s * 0.35e6 * (1 + 0.15 * (threads - 1)) / m.n_cell)))
        failed = []
        for _ in range(2):   # the reference's threaded code has raced before: one more try, then one core
            try:
                r = refrun.run_reference_zones(parts, params, n, threads=threads,
                                               wall_dists=None if wd is None else [wd[p.cells] for p in parts])
            except (RuntimeError, OSError) as e:
                failed.append(str(e).splitlines()[0])
                continue
            sec = r["loop_s"]
            return {"value": round(m.n_cell * n / sec / 1e6, 4), "unit": "Mcell-iters/s", "cores": threads,
                    "kind": "reference", "ms_per_step": round(sec / n * 1e3, 2), "iterations": n,
                    "cells": m.n_cell,
                    "sample": f"{what}, split into {threads} slab zones; {n} iterations in {sec:.1f} s by the "
                              f"reference solver built from its own sources with its OpenMP zone loops "
                              f"(oracle/_ref/ref_harness_omp), one zone per thread on {threads} host threads"
                              + (f" (after a failed try: {failed[0]})" if failed else "")}
        print("the threaded reference failed twice; timing one zone on one core: " + "; ".join(failed),
              file=sys.stderr)
    if refrun.available():
        # about 0.35 Mcell-iterations/s: as many iterations as fit the budget, at least 2
        n = int(max(2, min(args.steps, budget_s * 0.35e6 / m.n_cell)))
        r = refrun.run_reference(m, params, n, wall_dist=wd)
        sec = float(r["iter_seconds"][0])
        kind, how = "reference", "the reference solver built from its own sources (oracle/_ref/ref_harness)"
    else:
        from oracle.oracle import Oracle

        o = Oracle(m, params, wall_dist=wd)
        o.iterate(1)
        n = int(max(2, min(args.steps, budget_s * 0.78e6 / m.n_cell)))
        t0 = time.perf_counter()
        o.iterate(n)
        sec = time.perf_counter() - t0
        kind, how = "port", "the oracle (single-threaded C restatement of the reference path)"
    return {"value": round(m.n_cell * n / sec / 1e6, 4), "unit": "Mcell-iters/s", "cores": 1, "kind": kind,
            "ms_per_step": round(sec / n * 1e3, 2), "iterations": n, "cells": m.n_cell,
            "sample": f"{what}; {n} iterations in {sec:.1f} s by {how}; one zone on one core (the reference "
                      "parallelises only across zones and MPI ranks)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="phx", choices=["phx", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD)
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--no-fp64-arm", action="store_true", help="skip the FP64 comparison run of a mixed run")
    ap.add_argument("--exact-source", action="store_true", help="mixed SA runs keep the exact SA source")
    ap.add_argument("--save-mlp", default=None, help="write the trained learned-source model (.npy)")
    ap.add_argument("--mlp-blob", default=None, help="use this learned-source model (.npy) instead of training one")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--converge", action="store_true",
                    help="run the workload's full iteration count for every arm and report converged CL/CD")
    ap.add_argument("--iterations", type=int, default=0,
                    help="iterations of a --converge run (default: the workload's own count)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    wl = workloads()[args.workload]

    if args.impl == "reference":
        if rank != 0:
            return
        cb = cpu_baseline(args, args.workload)
        line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "Mcell-iters/s",
                "n_gpus": args.gpus, "steps": cb["iterations"], "warmup": 0, "ms_per_step": cb["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded generated mesh, free-stream start)",
                "config": {"workload": args.workload, "desc": wl["desc"],
                           "parallelism": f"{cb['cores']} CPU thread(s), one zone each",
                           "same_config": cb["sample"].startswith("the workload's own mesh"),
                           "sample": cb["sample"]},
                "cpu_baseline": cb, "e2e": {"value": cb["value"], "unit": "Mcell-iters/s",
                                             "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    if args.converge:
        from phenlei_b200 import mesh as M

        m = wl["mesh"]()
        wd = M.wall_distance(m) if wl.get("wall_dist") else None
        print(json.dumps({"converge": converge(args, m, wd)}))
        return

    if world > 1:
        return main_zones(args, rank, world, wl)
    from phenlei_b200 import mesh as M
    import torch

    torch.cuda.set_device(0)
    m = wl["mesh"]()
    wd = M.wall_distance(m) if wl.get("wall_dist") else None
    sa = wl["params"].get("viscousType", 0) == 3
    r64 = None
    blob = None
    if args.mlp_blob:
        blob = np.load(args.mlp_blob).astype(np.float32)
    if args.precision == "mixed" and not args.no_fp64_arm:
        # the headline ratio: mixed path (with the learned SA source on SA
        # workloads) against the plain FP64 path on the same mesh; the FP64
        # arm runs first and its final state trains the learned source
        r64 = run_phx(args, rank, world, "fp64", m, wd, e2e=False,
                      train=sa and not args.exact_source and blob is None)
        if r64["mlp"]:
            blob = r64["mlp"].pop("blob")
            if args.save_mlp and rank == 0:
                np.save(args.save_mlp, blob)
    # the mixed path with the exact SA source: the third arm the
    # headline is read against (what the learned source adds or costs)
    rx = None
    if r64 is not None and blob is not None:
        rx = run_phx(args, rank, world, args.precision, m, wd, e2e=False)
    r = run_phx(args, rank, world, args.precision, m, wd, mlp_blob=blob)
    ms = r["ms"]
    nc = r["nc"]
    per_gpu = nc * args.steps / (ms / 1e3) / 1e6
    value = per_gpu * world
    peak, peak_kind = measured_peaks()
    kb = kernel_bytes(r["mesh"], args.precision, wl["params"].get("viscousType", 0),
                      wl["params"].get("gradientName", "ggcell"))
    mb = minimal_bytes(r["mesh"], args.precision, wl["params"].get("viscousType", 0),
                       wl["params"].get("gradientName", "ggcell"))
    phase = r["phase_ms"]
    dom = max(phase, key=phase.get)
    achieved = kb[dom] / (phase[dom] / 1e3) / 1e9
    tpc = MEASURED_TRAFFIC_PER_CELL.get((dom, args.precision))
    traffic = round(tpc * nc) if tpc else None
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "Mcell-iters/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32+f64",
        "data": "synthetic (seeded generated mesh, free-stream start)",
        "config": {"workload": args.workload, "desc": wl["desc"], "cells": nc, "precision": args.precision,
                   "parallelism": "1 GPU",
                   "l2": "inputs larger than L2 (state %.0f MB)" % (5 * 8 * r["nt"] / 1e6)},
        "gpu_launches": int(r["launches"]),
        "phase_ms": {k: round(v, 4) for k, v in phase.items()},
        "roofline": {"kernel": dom, "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                     "algorithmic_bytes": kb[dom], "traffic": traffic},
        "iteration_bytes": kb["iteration"],
        "iteration_roofline_frac": round(kb["iteration"] / (ms / args.steps / 1e3) / 1e9 / peak, 4),
        # the same over the minimal pass structure's compulsory bytes (no records of this implementation)
        "iteration_compulsory_bytes": mb,
        "iteration_compulsory_roofline_frac": round(mb / (ms / args.steps / 1e3) / 1e9 / peak, 4),
        "clocks": r["clocks"],
        "e2e": {"value": round(nc / r["e2e_s"] / 1e6 * world, 3), "unit": "Mcell-iters/s",
                "h2d_bytes_per_step": 5 * 8 * r["nt"], "d2h_bytes_per_step": 5 * 8 * r["nt"] + 8},
        "residual_last": float(r["hist"][-1]) if len(r["hist"]) else None,
    }
    if r64 is not None:
        v64 = nc * args.steps / (r64["ms"] / 1e3) / 1e6 * world
        line["fp64_arm"] = {"value": round(v64, 3), "ms_per_step": round(r64["ms"] / args.steps, 4),
                            "phase_ms": {k: round(v, 4) for k, v in r64["phase_ms"].items()},
                            "residual_last": float(r64["hist"][-1]) if len(r64["hist"]) else None}
        line["speedup_vs_fp64"] = round(value / v64, 3)
        if rx is not None:
            vx = nc * args.steps / (rx["ms"] / 1e3) / 1e6 * world
            line["mixed_exact_arm"] = {"value": round(vx, 3), "ms_per_step": round(rx["ms"] / args.steps, 4),
                                       "phase_ms": {k: round(v, 4) for k, v in rx["phase_ms"].items()},
                                       "speedup_vs_fp64": round(vx / v64, 3)}
            if rx["forces"] and r64["forces"]:
                line["mixed_exact_arm"]["dCL"] = abs(rx["forces"]["CL"] - r64["forces"]["CL"])
                line["mixed_exact_arm"]["dCD"] = abs(rx["forces"]["CD"] - r64["forces"]["CD"])
            if rx["vist"] is not None and r64["vist"] is not None:
                line["mixed_exact_arm"]["dVIST_rel"] = float(np.max(np.abs(rx["vist"] - r64["vist"]))
                                                             / np.max(np.abs(r64["vist"])))
        if r["forces"] and r64["forces"]:
            line["accuracy_vs_fp64"] = {"dCL": abs(r["forces"]["CL"] - r64["forces"]["CL"]),
                                        "dCD": abs(r["forces"]["CD"] - r64["forces"]["CD"]),
                                        "CL_fp64": r64["forces"]["CL"], "CD_fp64": r64["forces"]["CD"],
                                        "after_iterations": r["iters"]}
            if r["vist"] is not None and r64["vist"] is not None:
                # eddy viscosity, max-norm relative difference over all cells
                line["accuracy_vs_fp64"]["dVIST_rel"] = float(np.max(np.abs(r["vist"] - r64["vist"]))
                                                             / np.max(np.abs(r64["vist"])))
                line["accuracy_vs_fp64"]["dVIST_rms_rel"] = float(np.sqrt(np.mean((r["vist"] - r64["vist"]) ** 2))
                                                                 / np.sqrt(np.mean(r64["vist"] ** 2)))
                line["accuracy_vs_fp64"]["VIST_max_fp64"] = float(np.max(r64["vist"]))
    if rx is not None and blob is not None:
        # what the learned source buys against the exact source it replaces, on the same mixed path and steps
        g = {"iteration_ms": {"learned": round(ms / args.steps, 4), "exact": round(rx["ms"] / args.steps, 4)},
             "sa_residual_ms": {"learned": round(r["phase_ms"]["sa_residual"], 4),
                                "exact": round(rx["phase_ms"]["sa_residual"], 4)},
             "throughput_ratio_learned_over_exact": round(rx["ms"] / ms, 4)}
        if r["forces"] and rx["forces"]:
            g["dCL_vs_exact"] = abs(r["forces"]["CL"] - rx["forces"]["CL"])
            g["dCD_vs_exact"] = abs(r["forces"]["CD"] - rx["forces"]["CD"])
        if r["vist"] is not None and rx["vist"] is not None:
            g["dVIST_rel_vs_exact"] = float(np.max(np.abs(r["vist"] - rx["vist"])) / np.max(np.abs(rx["vist"])))
        line["mlp_gain"] = g
    line["config"]["sa_source"] = (("learned (MLP, exact outside its hull)" if blob is not None else "exact")
                                   if sa else None)
    if blob is not None:
        line["mlp"] = dict((r64 or {}).get("mlp") or {"loaded": args.mlp_blob}, cells_learned_per_iteration=round(
            r["mlp"]["cells_learned"] / r["iters"], 1), cells=nc)
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args, args.workload)
    print(json.dumps(line))


if __name__ == "__main__":
    main()
