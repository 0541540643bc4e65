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


def test_tc_bounded_wait_times_out_and_releases(cuda):
    """A barrier that no copy completes: every wait gives up after 1 ms, the kernel reports
    the timeout, writes nothing and returns its tensor memory (the following normal self-test
    allocates it again and is exact); the context stays usable.  The host maps the flag to
    the timeout error of the tensor-core transforms."""
    import time

    import torch

    from gmaster_b200 import sht_tc

    t0 = time.time()
    flag, untouched = tc.selftest_timeout(wait_ns=1_000_000)
    elapsed = time.time() - t0
    assert flag == 1 and untouched
    assert elapsed < 5.0
    err, scale, flag = tc.selftest(128, 128)
    assert flag == 0 and err <= 1e-5 * scale
    # the host side of the same flag: a set error word raises and is cleared
    tp = sht_tc.get_tc_plan(8, 23)
    tp.err.fill_(1)
    with pytest.raises(RuntimeError, match="timed out"):
        sht_tc._check(tp)
    assert int(tp.err.item()) == 0
    torch.cuda.synchronize()
