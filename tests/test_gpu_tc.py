"""The tcgen05 machinery (bulk copy, mbarrier, TMEM, UMMA descriptors, tcgen05.ld)
against a float32 matmul of the same bf16 operands."""

import pytest

from gmaster_b200 import tc

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,K", [(16, 64), (64, 128), (128, 128), (256, 192)])
def test_tc_selftest_matches_matmul(cuda, N, K):
    err, scale, flag = tc.selftest(N, K)
    assert flag == 0
    assert err <= 1e-5 * scale
