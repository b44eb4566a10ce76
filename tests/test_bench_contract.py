"""bench.py's reference arm and its byte models, on the CPU.

* ``bench.py --impl reference`` prints one JSON line with the keys the bench
  contract names (metric, value, unit, steps, warmup, ms_per_step,
  higher_is_better, config, cpu_baseline, e2e with zero copy bytes), its
  throughput agreeing with its own step time.
* Under a launcher (RANK > 0) the reference arm exits without work or output.
* When the threaded reference run fails twice, the arm times one zone on one
  core instead of failing.
* The compulsory-byte count of the minimal pass structure never exceeds this
  build's own per-pass count, and both grow with the cell count.
"""
import json
import os
import subprocess
import sys

import pytest

from oracle import refrun
from tests.conftest import ROOT


def _bench(*args, env=None):
    e = dict(os.environ, **(env or {}))
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT, env=e,
                          capture_output=True, text=True, timeout=600)


@pytest.mark.skipif(not refrun.available(), reason="the reference build (oracle/_ref) is absent")
def test_reference_arm_prints_one_contract_line():
    r = _bench("--impl", "reference", "--workload", "euler_bump_8k", "--steps", "3", "--warmup", "3")
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "dtype", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference"
    assert d["higher_is_better"] is True
    assert d["config"]["workload"] == "euler_bump_8k"
    assert d["config"]["same_config"] is True   # the 8,192-cell bump is its own sample
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    # value (Mcell-iterations/s) and the step time describe the same run
    assert abs(cb["cells"] / (d["ms_per_step"] / 1e3) / 1e6 - d["value"]) <= 0.02 * d["value"]


def test_reference_arm_is_rank_zero_only():
    r = _bench("--impl", "reference", "--workload", "euler_bump_8k", "--steps", "3", "--warmup", "3",
               env={"RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("viscous,gradient", [(0, "ggcell"), (1, "lsq"), (3, "ggcell")])
def test_compulsory_bytes_below_this_build_per_pass_bytes(precision, viscous, gradient):
    sys.path.insert(0, ROOT)
    import bench
    from phenlei_b200 import mesh as M

    small, large = M.channel_bump(16, 8, 2), M.channel_bump(32, 16, 4)
    for m in (small, large):
        kb = bench.kernel_bytes(m, precision, viscous, gradient)
        mb = bench.minimal_bytes(m, precision, viscous, gradient)
        assert 0 < mb <= kb["iteration"]
    assert bench.minimal_bytes(large, precision, viscous, gradient) > bench.minimal_bytes(small, precision, viscous,
                                                                                           gradient)


@pytest.mark.skipif(not refrun.available(), reason="the reference build (oracle/_ref) is absent")
def test_reference_arm_falls_back_to_one_core_when_the_threaded_run_fails(monkeypatch):
    import argparse

    sys.path.insert(0, ROOT)
    import bench

    calls = []

    def broken(*a, **k):
        calls.append(1)
        raise RuntimeError("reference harness failed (-11)")

    monkeypatch.setattr(refrun, "run_reference_zones", broken)
    monkeypatch.setattr(bench, "host_threads", lambda: 4)
    cb = bench.cpu_baseline(argparse.Namespace(steps=2), "euler_bump_8k")
    assert len(calls) == 2
    assert cb["cores"] == 1 and cb["kind"] == "reference" and cb["value"] > 0
