import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built phx library")


def reference_file(rel):
    """A file of the reference project (path relative to its root), or None
    where this machine does not hold the project.  The root comes from
    PHX_REFERENCE_ROOT or from the one the build of oracle/_ref recorded."""
    root = os.environ.get("PHX_REFERENCE_ROOT")
    rec = os.path.join(ROOT, "oracle", "_ref", "reference_root.txt")
    if not root and os.path.exists(rec):
        root = open(rec).read().strip()
    if not root:
        return None
    p = os.path.join(root, rel)
    return p if os.path.exists(p) else None


def load_golden(name):
    """A fixture written by tests/golden/make_golden.py from the reference solver."""
    from phenlei_b200 import mesh as M

    d = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    spec = json.loads(str(d["mesh"]))
    d["mesh_obj"] = getattr(M, spec["kind"])(**spec["args"])
    d["params_dict"] = json.loads(str(d["params"]))
    # the reference runs behind the fixtures pin flowInitStep to 0 unless the fixture sets it
    d["params_dict"].setdefault("flowInitStep", 0)
    return d


def rel_err(a, b):
    """Norm-wise relative error max|a-b| / max|b| (pointwise relative error is
    meaningless where the reference value is near zero)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = max(float(np.max(np.abs(b))), 1e-300)
    return float(np.max(np.abs(a - b))) / den


@pytest.fixture(scope="session")
def golden():
    return load_golden
