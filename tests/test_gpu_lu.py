"""Blocked LU of the binned coupling matrix (panels + the FP64 tile kernel for the trailing
updates) against the single-kernel factorisation and numpy; singular matrices are reported;
many right-hand sides in one solve equal one-at-a-time solves bit for bit."""

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
    # the trailing-update kernel: one panel step against numpy
    k0, k1 = 64, 128
    m = rng.normal(size=(n, n))
    d = torch.from_numpy(m).cuda().contiguous().clone()
    _lib.call("gm_lu_update", n, _lib.ptr(d), k0, k1, _lib.stream_handle())
    want_m = m.copy()
    want_m[k1:, k1:] -= m[k1:, k0:k1] @ m[k0:k1, k1:]
    np.testing.assert_allclose(d.cpu().numpy(), want_m, rtol=0, atol=1e-12 * np.abs(want_m).max())
    # many right-hand sides at once (the batched decouple) equal separate solves exactly
    many = lu.solve(torch.from_numpy(b).cuda()).cpu().numpy()
    for j in range(b.shape[1]):
        one_col = lu.solve(torch.from_numpy(b[:, j].copy()).cuda()).cpu().numpy()
        np.testing.assert_array_equal(many[:, j], one_col)
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
