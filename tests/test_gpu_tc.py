"""The tcgen05 machinery (bulk copy, mbarrier, TMEM, UMMA descriptors, tcgen05.ld)
against a float32 matmul of the same bf16 operands."""

import pytest

from gmaster_b200 import tc

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,K", [(16, 64), (64, 128), (128, 128), (256, 192)])
@pytest.mark.parametrize("a_mn,b_mn", [(False, False), (True, False), (False, True), (True, True)])
def test_tc_selftest_matches_matmul(cuda, N, K, a_mn, b_mn):
    if b_mn and N % 64:
        pytest.skip("MN-major B needs N % 64 == 0")
    err, scale, flag = tc.selftest(N, K, a_mn=a_mn, b_mn=b_mn)
    assert flag == 0
    assert err <= 1e-5 * scale
