"""Host helpers for the tensor-core (tcgen05) operand images."""

import numpy as np
import torch

from . import _lib


def sw128_offsets(R, K):
    """Byte offsets of element (r, k) in a K-major 128-byte-swizzled image of R rows."""
    r = np.arange(R)[:, None]
    k = np.arange(K)[None, :]
    kk = k % 64
    chunk = (kk // 8) ^ (r % 8)
    return (k // 64) * R * 128 + (r // 8) * 1024 + (r % 8) * 128 + chunk * 16 + (kk % 8) * 2


def sw128_mn_offsets(R, K):
    """Byte offsets of element (r, k) in an MN-major 128-byte-swizzled image (R % 64 == 0)."""
    r = np.arange(R)[:, None]
    k = np.arange(K)[None, :]
    chunk = ((r % 64) // 8) ^ (k % 8)
    return (k // 8) * (R // 64) * 1024 + (r // 64) * 1024 + (k % 8) * 128 + chunk * 16 + (r % 8) * 2


def sw128_image(mat16, mn=False):
    """uint16 (R, K) matrix -> uint8 image of R*K*2 bytes in the swizzled layout."""
    R, K = mat16.shape
    img = np.zeros(R * K, dtype=np.uint16)
    off = sw128_mn_offsets(R, K) if mn else sw128_offsets(R, K)
    img[off // 2] = mat16
    return img.view(np.uint8)


def selftest(N=128, K=128, seed=0, device="cuda", a_mn=False, b_mn=False):
    """Run the one-CTA tcgen05 GEMM check; returns (max abs error, scale, err flag)."""
    g = torch.Generator().manual_seed(seed)
    a = torch.randn(128, K, generator=g).to(torch.bfloat16)
    b = torch.randn(N, K, generator=g).to(torch.bfloat16)
    want = a.float() @ b.float().T
    ai = torch.from_numpy(sw128_image(a.view(torch.int16).numpy().view(np.uint16), a_mn)).to(device)
    bi = torch.from_numpy(sw128_image(b.view(torch.int16).numpy().view(np.uint16), b_mn)).to(device)
    d = torch.full((128, N), float("nan"), dtype=torch.float32, device=device)
    err = torch.zeros(1, dtype=torch.int32, device=device)
    _lib.call("gm_tc_selftest", N, K, int(a_mn), int(b_mn), _lib.ptr(ai), _lib.ptr(bi), _lib.ptr(d),
              _lib.ptr(err),
              _lib.stream_handle(torch.device(device)))
    torch.cuda.synchronize()
    got = d.cpu()
    return float((got - want).abs().max()), float(want.abs().max()), int(err.item())


def selftest_timeout(wait_ns=1_000_000, N=64, K=64, device="cuda"):
    """Run the self-test with its operand copies withheld: returns (err flag, output
    untouched), the flag 1 once every bounded wait has run out after `wait_ns`."""
    dev = torch.device(device)
    ai = torch.zeros(128 * K * 2, dtype=torch.uint8, device=dev)
    bi = torch.zeros(N * K * 2, dtype=torch.uint8, device=dev)
    d = torch.full((128, N), 7.0, dtype=torch.float32, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.call("gm_tc_selftest_timeout", N, K, _lib.ptr(ai), _lib.ptr(bi), _lib.ptr(d), _lib.ptr(err),
              int(wait_ns), _lib.stream_handle(dev))
    torch.cuda.synchronize()
    return int(err.item()), bool(torch.all(d == 7.0).item())
