"""The allocation-free tensor-core analysis entry point (gm_tc_analysis_noalloc).

Some callers cannot allocate device memory: a custom call inside a framework that owns
every allocation, or a service that reserves its memory once and must not call cudaMalloc
afterwards.  gm_tc_analysis_noalloc serves them by keeping its recurrence-state scratch in
a static device array inside the library.  This test calls it through the C ABI twice in a
row and then a third time with half as many CTAs (so the static array holds a different
slot layout than the call before it), and requires each result to equal, bit for bit,
gm_tc_analysis with a caller-provided scratch buffer: both launch the same deterministic
kernel on the same inputs, and every order m is reduced by one CTA in a fixed order, so
any leftover state or slot mix-up in the static array would show as a difference.
Nside 256 (lmax 767) needs three l-superblocks, so the state really goes through the
scratch.  The file is named to be collected last; it passes alone in a fresh process too.
"""

import numpy as np
import pytest
import torch

from gmaster_b200 import _lib, sht, sht_tc

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("spin,ncomp", [(0, 4), (2, 4)])
def test_noalloc_analysis_matches_scratch_entry_point(cuda, spin, ncomp):
    nside, lmax = 256, 767
    tp = sht_tc.get_tc_plan(nside, lmax)
    p = tp.plan
    rng = np.random.default_rng(31 + spin)
    maps = torch.from_numpy(rng.normal(size=(ncomp, 12 * nside ** 2))).cuda()
    spec = sht.ring_analysis(p, maps, _lib.MIXED)
    b = sht_tc._Batch(tp, spin, ncomp)
    b.zero_alm()
    rhs_map = torch.empty((p.L, p.nlanes, ncomp, 4), dtype=torch.float32, device=p.device)
    img_scale = sht_tc.pow2_scale(spec.view(torch.float32)) / 2.0
    _lib.call("gm_tc_pack", p.nside, p.lmax, spin, ncomp, _lib.ptr(spec), _lib.ptr(rhs_map),
              _lib.ptr(b.img[0]), _lib.ptr(b.img[1]) if spin else None, img_scale,
              _lib.stream_handle(p.device))
    stream = _lib.stream_handle(p.device)
    variants = (0,) if spin == 0 else (-2, 2)

    def run(noalloc, nctas):
        alm = torch.zeros_like(b.alm_i)
        err = torch.zeros(1, dtype=torch.int32, device=p.device)
        for sp, img in zip(variants, b.img):
            common = (p.nside, p.lmax, spin, sp, ncomp, _lib.ptr(p.geom), _lib.ptr(p.seeds),
                      _lib.ptr(tp.coef[spin]), _lib.ptr(img), _lib.ptr(alm), 1.0 / img_scale)
            if noalloc:
                _lib.call("gm_tc_analysis_noalloc", *common, nctas, _lib.ptr(err), stream)
            else:
                scratch = torch.empty(_lib.load().gm_tc_ana_scratch_bytes(p.nside, nctas) // 8,
                                      dtype=torch.float64, device=p.device)
                _lib.call("gm_tc_analysis", *common, _lib.ptr(scratch), nctas, _lib.ptr(err), stream)
        torch.cuda.synchronize()
        assert int(err.item()) == 0
        return alm.cpu().numpy()

    ref = run(False, tp.nctas)
    assert np.abs(ref).max() > 0
    for nctas in (tp.nctas, tp.nctas, max(1, tp.nctas // 2)):
        got = run(True, nctas)
        np.testing.assert_array_equal(got, ref)


def test_noalloc_rejects_oversized_requests(cuda):
    with pytest.raises(_lib.GMError) as err:
        _lib.call("gm_tc_analysis_noalloc", 4096, 12287, 0, 0, 1, None, None, None, None, None, 1.0,
                  148, None, None)
    assert err.value.status == 1
    assert "lane slots" in str(err.value)
