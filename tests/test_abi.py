"""The C-ABI library loads and exports every entry point include/phx.h declares
(no device calls)."""
import ctypes
import os
import re

import pytest

from phenlei_b200 import solver

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    out = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            out |= set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(phx_\w+)\s*\(", txt, re.M))
    return out


def test_library_exports_all_declared_symbols():
    if not os.path.exists(solver.LIB_PATH):
        pytest.skip("libphx.so not built")
    lib = ctypes.CDLL(solver.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in sorted(syms) if not hasattr(lib, s)]
    assert not missing, missing


def test_default_params_match_reference_defaults():
    if not os.path.exists(solver.LIB_PATH):
        pytest.skip("libphx.so not built")
    p = solver.make_params()
    assert p.refGama == 1.4 and p.venkatCoeff == 5.0 and p.CFLVaryStep == 500
    assert p.nLUSGSSweeps == 1 and p.roeEntropyFixMethod == 3
    assert p.uns_scheme_name == 0 and p.AusmpwPlusLimiter == 1.0
    assert p.flowInitStep == 100 and p.flowInitMethod == 0


def test_scheme_names_map_to_the_abi_ids():
    """uns_scheme_name strings (GetSchemeID, API/Physics/src/Flux_Inviscid.cpp:16-86)
    map to the same ids in the solver mirror, the oracle and include/phx.h."""
    from oracle.oracle import SCHEMES

    assert solver._STRING_KEYS["uns_scheme_name"] == SCHEMES
    hdr = open(os.path.join(os.path.dirname(__file__), "..", "include", "phx.h")).read()
    for name, sid in SCHEMES.items():
        assert f'#define PHX_SCHEME_{name.upper().replace("+", "_PLUS")} {sid}' in hdr, name


def _create_error(**kw):
    """The PHX_ERR_* name phx_ctx_create returns for these keys on this
    machine (parameter checks run before any CUDA call)."""
    from phenlei_b200 import cases
    from phenlei_b200 import mesh as M

    try:
        solver.NSSolverUnstruct(M.channel_bump(8, 4, 2), **dict(cases.EULER_BUMP, **kw))
    except solver.PhxError as e:
        return str(e).rsplit(" ", 1)[-1]
    return "PHX_OK"


@pytest.mark.parametrize("kw", [dict(flowInitMethod=1), dict(flowInitMethod=3), dict(flowInitStep=-1),
                                dict(roeEntropyFixMethod=2), dict(nLUSGSSweeps=2), dict(ivencat=6),
                                dict(gradientName=3), dict(uns_scheme_name=8), dict(uns_limiter_name=4),
                                dict(viscousType=2), dict(precision=7)])
def test_unsupported_settings_are_rejected(kw):
    """Settings outside the path (other entropy fixes, several LU-SGS sweeps,
    other Venkatakrishnan variants, boundary-layer / GMRES starts, unknown
    ids) fail with PHX_ERR_ARG rather than running something else."""
    if not os.path.exists(solver.LIB_PATH):
        pytest.skip("libphx.so not built")
    assert _create_error(**kw) == "PHX_ERR_ARG"


@pytest.mark.parametrize("kw", [dict(uns_scheme_name=s) for s in ("steger", "vanleer", "hlle", "ausmdv", "ausmpw+", "ausmpw", "vanleer_Rotate")]
                         + [dict(uns_limiter_name=n) for n in ("nolim", "1st", "barth")]
                         + [dict(flowInitStep=100), dict(flowInitMethod=2), dict(gradientName="ggnode")])
def test_supported_settings_pass_the_checks(kw):
    """Every supported setting gets past the parameter checks (on a machine
    without a GPU the first CUDA call then fails)."""
    if not os.path.exists(solver.LIB_PATH):
        pytest.skip("libphx.so not built")
    assert _create_error(**kw) != "PHX_ERR_ARG"
