"""phx_residual_norm_noalloc: the allocation-free residual monitor, called
through the C ABI on a device residual, against the context's own monitor
(phx_residual_norm) on two calls in a row.  Collected last (file name) so it
also runs after every other GPU test in the same process.

Tolerance: 1e-13 relative; the two reductions sum the same FP64 squares in
different orders."""
import ctypes as C

import numpy as np
import pytest

from phenlei_b200 import cases
from phenlei_b200 import mesh as M
from phenlei_b200 import solver as S

pytestmark = pytest.mark.gpu

TOL = 1e-13


def _noalloc():
    f = S.lib().phx_residual_norm_noalloc
    f.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_int, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def test_noalloc_residual_norm_matches_context_monitor():
    import torch

    m = M.channel_bump(64, 32, 4)
    s = S.NSSolverUnstruct(m, **cases.EULER_BUMP)
    s.set_q_cells(cases.perturbed_state(m, cases.EULER_BUMP, seed=12))
    f = _noalloc()
    for _ in range(2):   # two solver steps, each checked with two monitor calls in a row
        s.Relaxation(1)
        ref = s.GetResidual()
        res = torch.empty((5, s.nt), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        s._check(S.lib().phx_get_state_device(s.h, S.PHX_RES, res.data_ptr(), res.numel()), "get_state_device")
        for _ in range(2):
            out = np.zeros(5)
            rc = f(res.data_ptr(), m.n_cell, s.nt, 5, out.ctypes.data, None)
            assert rc == 0
            assert np.max(np.abs(out - ref)) <= TOL * np.max(np.abs(ref))


@pytest.mark.parametrize("n_cell,pad,nvar", [(300_000, 777, 8), (1, 0, 3), (1, 5, 8)])
def test_noalloc_matches_numpy_on_a_random_array(n_cell, pad, nvar):
    """Sizes past the partial-sum pass's 1024-block cap (its grid-stride loop),
    the maximum number of variables, a row stride larger than the cell count,
    and a single cell; two calls in a row."""
    import torch

    rng = np.random.default_rng(n_cell + pad + nvar)
    n_total = n_cell + pad
    x = rng.standard_normal((nvar, n_total))
    res = torch.from_numpy(x).cuda()
    torch.cuda.synchronize()
    ref = np.sqrt(np.mean(x[:, :n_cell] ** 2, axis=1))
    f = _noalloc()
    for _ in range(2):
        out = np.zeros(nvar)
        rc = f(res.data_ptr(), n_cell, n_total, nvar, out.ctypes.data, None)
        assert rc == 0
        assert np.max(np.abs(out - ref) / ref) <= TOL


def test_noalloc_rejects_more_variables_than_its_scratch_holds():
    import torch

    res = torch.zeros((9, 16), dtype=torch.float64, device="cuda")
    out = np.zeros(9)
    rc = _noalloc()(res.data_ptr(), 16, 16, 9, out.ctypes.data, None)
    assert rc == -1   # PHX_ERR_ARG, nothing launched
