"""The tcgen05 BF16 GEMM (ngpu_gemm_bf16_tn) against numpy FP64 products of
the same bf16 values; FP32 accumulation bound: |err| <= 1e-5 * sum_k |a b|
(fp32 rounding of a K-term sum), plus the fused epilogues (bias + GELU with
row-major and transposed bf16 copies; gradient times GELU')."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _gelu(z):
    return 0.5 * z * (1.0 + np.tanh(0.7978845608028654 * (z + 0.044715 * z ** 3)))


def _gelu_grad(z):
    u = 0.7978845608028654 * (z + 0.044715 * z ** 3)
    t = np.tanh(u)
    return 0.5 * (1 + t) + 0.5 * z * (1 - t * t) * 0.7978845608028654 * (1 + 3 * 0.044715 * z * z)


@pytest.fixture(params=["tma", "cp.async"])
def gemm_path(request, monkeypatch):
    """Both forms of the kernel: the TMA-fed warp-specialised one (the
    default) and the cp.async one (NGPU_GEMM_TMA=0)."""
    monkeypatch.setenv("NGPU_GEMM_TMA", "1" if request.param == "tma" else "0")
    return request.param


def _bf16(x):
    import torch
    return torch.as_tensor(x, dtype=torch.float32).to(torch.bfloat16)


def _gemm(A, B, epi=0, bn=128, bias=None, zin=None):
    import torch
    from neurogpu_b200 import _ffi
    M, K = A.shape
    N = B.shape[0]
    dev = torch.device("cuda")
    a, b = A.to(dev).contiguous(), B.to(dev).contiguous()
    out = torch.full((M, N), float("nan"), device=dev)
    ob = torch.zeros((M, N), dtype=torch.bfloat16, device=dev)
    obt = torch.zeros((N, M), dtype=torch.bfloat16, device=dev)
    bi = None if bias is None else torch.as_tensor(bias, dtype=torch.float32, device=dev)
    zi = None if zin is None else torch.as_tensor(zin, dtype=torch.float32, device=dev).contiguous()
    p = lambda t: None if t is None else C.c_void_p(t.data_ptr())
    _ffi.check("ngpu_gemm_bf16_tn", _ffi.lib().ngpu_gemm_bf16_tn(
        p(a), p(b), M, N, K, K, K, epi, bn, p(out), p(ob), p(obt), N, M, p(bi), p(zi),
        C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    flag = C.c_int32()
    _ffi.check("ngpu_gemm_error", _ffi.lib().ngpu_gemm_error(C.byref(flag)))
    assert flag.value == 0
    return out.cpu().numpy(), ob.float().cpu().numpy(), obt.float().cpu().numpy()


@pytest.mark.parametrize("M,N,K,bn", [(128, 128, 64, 128), (256, 512, 512, 128), (200, 20, 64, 32),
                                      (1000, 96, 128, 64), (384, 512, 256, 256), (8192, 512, 512, 128)])
def test_gemm_matches_fp64(ngpu_built, gemm_path, M, N, K, bn):
    rng = np.random.default_rng(M + N + K)
    A = _bf16(rng.normal(size=(M, K)))
    B = _bf16(rng.normal(size=(N, K)))
    a64, b64 = A.float().numpy().astype(np.float64), B.float().numpy().astype(np.float64)
    want = a64 @ b64.T
    got, _, _ = _gemm(A, B, 0, bn)
    bound = 1e-5 * (np.abs(a64) @ np.abs(b64).T) + 1e-30
    assert np.all(np.abs(got - want) <= bound)


@pytest.mark.parametrize("M,N,K,bn", [(512, 512, 4096, 128), (512, 64, 8192, 64), (200, 20, 1024, 32),
                                      (128, 128, 64, 128)])
def test_gemm_split_k_matches_fp64(ngpu_built, gemm_path, M, N, K, bn):
    """Epilogue 4: K spread over CTAs whose partial sums add into the zeroed
    output; the same fp32 bound as one CTA per tile (sums of K terms in
    another order)."""
    rng = np.random.default_rng(M + 3 * N + K)
    A = _bf16(rng.normal(size=(M, K)))
    B = _bf16(rng.normal(size=(N, K)))
    a64, b64 = A.float().numpy().astype(np.float64), B.float().numpy().astype(np.float64)
    want = a64 @ b64.T
    got, _, _ = _gemm(A, B, 4, bn)
    bound = 1e-5 * (np.abs(a64) @ np.abs(b64).T) + 1e-30
    assert np.all(np.abs(got - want) <= bound)


def test_gemm_bias_gelu_epilogue(ngpu_built, gemm_path):
    rng = np.random.default_rng(7)
    M, N, K = 300, 128, 192
    A, B = _bf16(rng.normal(size=(M, K))), _bf16(rng.normal(size=(N, K)) * 0.2)
    bias = rng.normal(size=N).astype(np.float32)
    z64 = A.float().numpy().astype(np.float64) @ B.float().numpy().astype(np.float64).T + bias
    z, h, ht = _gemm(A, B, 1, 128, bias=bias)
    np.testing.assert_allclose(z, z64, rtol=1e-4, atol=1e-4)
    h_want = _gelu(z.astype(np.float64))
    np.testing.assert_allclose(h, h_want, rtol=1e-2, atol=1e-2)          # bf16 output
    np.testing.assert_array_equal(ht, h.T)


def test_gemm_gelu_grad_epilogue(ngpu_built, gemm_path):
    rng = np.random.default_rng(8)
    M, N, K = 256, 64, 128
    A, B = _bf16(rng.normal(size=(M, K))), _bf16(rng.normal(size=(N, K)) * 0.3)
    zin = rng.normal(size=(M, N)).astype(np.float32)
    d64 = A.float().numpy().astype(np.float64) @ B.float().numpy().astype(np.float64).T
    _, dz, dzt = _gemm(A, B, 3, 64, zin=zin)
    want = d64 * _gelu_grad(zin.astype(np.float64))
    np.testing.assert_allclose(dz, want, rtol=1e-2, atol=1e-2)
    np.testing.assert_array_equal(dzt, dz.T)


def _units(M, N, bn):
    return -(-M // 128) * -(-N // bn)


@pytest.mark.parametrize("M,N,K,bn", [(4200, 300, 192, 32), (2560, 1024, 256, 64), (4800, 1000, 128, 128),
                                      (4400, 2304, 320, 256)])
def test_persistent_gemm_matches_fp64_and_per_tile_kernel(ngpu_built, monkeypatch, M, N, K, bn):
    """More than two tiles per SM (ragged edges included): the persistent kernel,
    whose accumulator is double-buffered in tensor memory, against FP64 and,
    bit for bit, against the one-CTA-per-tile kernel (same MMAs in the same
    order per tile)."""
    assert _units(M, N, bn) > 2 * 148
    monkeypatch.setenv("NGPU_GEMM_TMA", "1")
    rng = np.random.default_rng(M + N + K + bn)
    A = _bf16(rng.normal(size=(M, K)))
    B = _bf16(rng.normal(size=(N, K)))
    a64, b64 = A.float().numpy().astype(np.float64), B.float().numpy().astype(np.float64)
    got, _, _ = _gemm(A, B, 0, bn)
    bound = 1e-5 * (np.abs(a64) @ np.abs(b64).T) + 1e-30
    assert np.all(np.abs(got - a64 @ b64.T) <= bound)
    monkeypatch.setenv("NGPU_GEMM_PERSISTENT", "0")
    per_tile, _, _ = _gemm(A, B, 0, bn)
    np.testing.assert_array_equal(got, per_tile)


@pytest.mark.parametrize("epi,M,N,K,bn", [(1, 7700, 640, 128, 128), (3, 9500, 256, 64, 64), (2, 19000, 512, 64, 256)])
def test_persistent_gemm_epilogues_match_per_tile_kernel(ngpu_built, monkeypatch, epi, M, N, K, bn):
    """The fused epilogues (bias + GELU with its transposed copy, GELU'
    gradient, bias) out of the persistent kernel's two accumulators: equal,
    bit for bit, to the one-CTA-per-tile kernel's."""
    assert _units(M, N, bn) > 2 * 148
    monkeypatch.setenv("NGPU_GEMM_TMA", "1")
    rng = np.random.default_rng(epi * 1000 + M)
    A, B = _bf16(rng.normal(size=(M, K))), _bf16(rng.normal(size=(N, K)) * 0.2)
    bias = rng.normal(size=N).astype(np.float32) if epi in (1, 2) else None
    zin = rng.normal(size=(M, N)).astype(np.float32) if epi == 3 else None
    got = _gemm(A, B, epi, bn, bias=bias, zin=zin)
    monkeypatch.setenv("NGPU_GEMM_PERSISTENT", "0")
    ref = _gemm(A, B, epi, bn, bias=bias, zin=zin)
    for g_, r_ in zip(got, ref):
        np.testing.assert_array_equal(g_, r_)
    if epi == 2:
        z64 = A.float().numpy().astype(np.float64) @ B.float().numpy().astype(np.float64).T + bias
        np.testing.assert_allclose(got[0], z64, rtol=1e-4, atol=1e-4)
