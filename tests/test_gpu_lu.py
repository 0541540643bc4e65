"""Blocked LU of the binned coupling matrix (panels + GEMM trailing updates) against the
single-kernel factorisation and numpy; singular matrices are reported."""

import numpy as np
import pytest
import torch

from gmaster_b200 import _lib
from gmaster_b200.workspaces import LUFactor

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [300, 700, 1541])
def test_blocked_lu_solves_like_numpy(cuda, n):
    rng = np.random.default_rng(n)
    a = rng.normal(size=(n, n)) + n ** 0.5 * np.eye(n)
    b = rng.normal(size=(n, 5))
    lu = LUFactor(torch.from_numpy(a).cuda())
    lu.check()
    x = lu.solve(torch.from_numpy(b).cuda()).cpu().numpy()
    want = np.linalg.solve(a, b)
    assert np.max(np.abs(x - want)) / np.max(np.abs(want)) < 1e-11
    inv = lu.inverse().cpu().numpy()
    assert np.max(np.abs(inv @ a - np.eye(n))) < 1e-10
    # the single-kernel factorisation gives the same solution
    one = torch.from_numpy(a).cuda().clone()
    piv = torch.empty(n, dtype=torch.int32, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.call("gm_lu_factor", n, _lib.ptr(one), _lib.ptr(piv), _lib.ptr(st), _lib.stream_handle())
    y = torch.from_numpy(b).cuda().contiguous().clone()
    _lib.call("gm_lu_solve", n, _lib.ptr(one), _lib.ptr(piv), 5, _lib.ptr(y), _lib.stream_handle())
    assert np.max(np.abs(y.cpu().numpy() - x)) / np.max(np.abs(want)) < 1e-11


def test_blocked_lu_reports_singular(cuda):
    n = 400
    rng = np.random.default_rng(1)
    a = rng.normal(size=(n, n))
    a[:, 123] = 0.0
    lu = LUFactor(torch.from_numpy(a).cuda())
    with pytest.raises(np.linalg.LinAlgError):
        lu.check()
