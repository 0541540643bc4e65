"""Every compiled tile shape of the SIMT Legendre kernels gives the result of the built-in
choice (only the summation order differs), and the autotuner picks one of them."""

import pytest
import torch

from gmaster_b200 import _lib, autotune, sht

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec,tol", [(_lib.FP64, 1e-13), (_lib.MIXED, 2e-6)])
@pytest.mark.parametrize("spin,ncomp", [(0, 3), (2, 2)])
def test_every_tile_matches_default(cuda, prec, tol, spin, ncomp):
    plan = sht.get_plan(32, 95)
    real = torch.float64 if prec == _lib.FP64 else torch.float32
    gen = torch.Generator(device="cuda")
    gen.manual_seed(5 + spin)
    rhs = torch.randn((plan.L, plan.nlanes, ncomp, 4), generator=gen, dtype=real, device="cuda")
    alm_in = torch.zeros((ncomp, plan.nelem), dtype=torch.complex128, device="cuda")
    alm_in.real.normal_(generator=gen)
    alm_in.imag.normal_(generator=gen)
    st = _lib.stream_handle(plan.device)

    def ana(tile):
        out = torch.zeros((ncomp, plan.nelem), dtype=torch.complex128, device="cuda")
        _lib.call("gm_legendre_analysis_tile", prec, spin, plan.nside, plan.lmax, ncomp,
                  _lib.ptr(plan.geom), _lib.ptr(plan.seeds), _lib.ptr(rhs), _lib.ptr(out), 1.0, tile, st)
        return out

    def syn(tile):
        out = torch.empty_like(rhs)
        _lib.call("gm_legendre_synthesis_tile", prec, spin, plan.nside, plan.lmax, ncomp,
                  _lib.ptr(plan.geom), _lib.ptr(plan.seeds), _lib.ptr(alm_in), _lib.ptr(out), tile, st)
        return out

    a0, s0 = ana(-1), syn(-1)
    for t in range(len(autotune.tiles(spin))):
        a, s = ana(t), syn(t)
        assert float((a - a0).abs().max() / a0.abs().max()) < tol, t
        assert float((s - s0).abs().max() / s0.abs().max()) < tol, t
    with pytest.raises(_lib.GMError):
        ana(len(autotune.tiles(spin)))


def test_autotuner_choice_is_cached_and_used(cuda):
    plan = sht.get_plan(16, 47)
    was = autotune.autotune_enabled()
    autotune.set_autotune(True)
    try:
        maps = torch.randn((2, plan.npix), dtype=torch.float64, device="cuda")
        got = sht.map2alm_device(maps, 2, 16, 47, 1, "mixed")
        key = [k for k in autotune.choices() if ":s2:n16:l47:c2" in k]
        assert key and all(autotune.choices()[k][0] in autotune.tiles(2) for k in key)
        assert all(len(autotune.choices()[k][1]) == len(autotune.tiles(2)) for k in key)
    finally:
        autotune.set_autotune(False)
    want = sht.map2alm_device(maps, 2, 16, 47, 1, "mixed")
    autotune.set_autotune(was)
    assert float((got - want).abs().max() / want.abs().max()) < 2e-6
