"""GPU: the tensor-core GEMM (cjx_gemm: TMA + tcgen05.mma + TMEM) against float64 torch.

Inputs are exact BF16 / FP16 values, so products are exact in FP32 and the
only error is the FP32 summation order: |C - C_ref| <= 1e-5 * (|A| |B|^T)
elementwise (plus the BF16 rounding of the output when it is stored as
BF16: relative 2^-8).
"""

import pytest

pytestmark = pytest.mark.gpu

SHAPES = [  # M, N, K  (ragged M, N and K edges exercise the TMA zero fill and the store masks)
    (128, 128, 64),
    (300, 96, 200),
    (1000, 256, 1024),
    (256, 768, 1024),
    (64, 32, 16),
    (4096, 64, 288),
    (130, 40, 9),
    (2048, 512, 4096),
]


def _operands(m, n, k, dtype, seed, ld_pad=0):
    import torch

    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    kk = ((k + 7) // 8) * 8 + ld_pad
    a = torch.zeros((m, kk), device="cuda", dtype=dtype)
    b = torch.zeros((n, kk), device="cuda", dtype=dtype)
    a[:, :k] = torch.randn((m, k), generator=g, device="cuda").to(dtype)
    b[:, :k] = torch.randn((n, k), generator=g, device="cuda").to(dtype)
    if kk > k:  # garbage beyond K must not leak into the product
        a[:, k:] = 1000.0
        b[:, k:] = -1000.0
    return a, b


def _ref(a, b, k):
    ad, bd = a[:, :k].double(), b[:, :k].double()
    return ad @ bd.T, ad.abs() @ bd.abs().T


@pytest.mark.parametrize("m,n,k", SHAPES)
def test_gemm_fp32_out(cuda_device, m, n, k):
    import torch

    from cryojax_b200 import _native as nat

    a, b = _operands(m, n, k, torch.bfloat16, m + n + k)
    c = torch.full((m, n), float("nan"), device="cuda", dtype=torch.float32)
    nat.gemm(a, b, c, k=k)
    assert nat.device_status() == 0
    ref, bound = _ref(a, b, k)
    assert torch.all((c.double() - ref).abs() <= 1e-5 * bound + 1e-30), (c.double() - ref).abs().max()


def test_gemm_bias_relu_bf16_out(cuda_device):
    import torch

    from cryojax_b200 import _native as nat

    m, n, k = 777, 200, 320
    a, b = _operands(m, n, k, torch.bfloat16, 5)
    bias = torch.randn(n, device="cuda", dtype=torch.float32)
    c = torch.empty((m, 208), device="cuda", dtype=torch.bfloat16)  # ldc > n
    nat.gemm(a, b, c, n=n, k=k, bias=bias, flags=nat.CJX_GEMM_RELU | nat.CJX_GEMM_OUT_BF16)
    assert nat.device_status() == 0
    ref, bound = _ref(a, b, k)
    ref = torch.clamp(ref + bias.double(), min=0)
    got = c[:, :n].double()
    assert torch.all((got - ref).abs() <= 1e-5 * bound + 2.0**-8 * ref.abs() + 1e-30)


@pytest.mark.parametrize("split", [1, 3, 16])
def test_gemm_split_k_accumulate(cuda_device, split):
    import torch

    from cryojax_b200 import _native as nat

    m, n, k = 64, 288, 8192  # a weight-gradient shape: small output, long K
    a, b = _operands(m, n, k, torch.bfloat16, 11)
    c0 = torch.randn((m, n), device="cuda", dtype=torch.float32)
    c = c0.clone()
    nat.gemm(a, b, c, k=k, flags=nat.CJX_GEMM_ACCUMULATE, split_k=split)
    assert nat.device_status() == 0
    ref, bound = _ref(a, b, k)
    assert torch.all((c.double() - c0.double() - ref).abs() <= 1e-5 * bound + 1e-6)


def test_gemm_fp16_inputs(cuda_device):
    import torch

    from cryojax_b200 import _native as nat

    m, n, k = 512, 384, 1664
    a, b = _operands(m, n, k, torch.float16, 21)
    c = torch.empty((m, n), device="cuda", dtype=torch.float32)
    nat.gemm(a, b, c, k=k, flags=nat.CJX_GEMM_F16)
    assert nat.device_status() == 0
    ref, bound = _ref(a, b, k)
    assert torch.all((c.double() - ref).abs() <= 1e-5 * bound + 1e-30)


def test_gemm_argument_errors(cuda_device):
    import torch

    from cryojax_b200 import _native as nat

    a = torch.zeros((128, 20), device="cuda", dtype=torch.bfloat16)  # ld 20: not a multiple of 8
    b = torch.zeros((128, 20), device="cuda", dtype=torch.bfloat16)
    c = torch.zeros((128, 128), device="cuda", dtype=torch.float32)
    with pytest.raises(nat.CryojaxB200Error):
        nat.gemm(a, b, c)
    a = torch.zeros((128, 64), device="cuda", dtype=torch.bfloat16)
    with pytest.raises(nat.CryojaxB200Error):  # split-K without accumulate
        nat.gemm(a, a, c, split_k=2)


def test_bounded_wait_gives_up_and_reports(cuda_device):
    """A wait on a barrier nothing arrives on ends after its limit with status 105; the GPU stays usable."""
    import time

    import torch

    from cryojax_b200 import _native as nat

    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    nat.selftest_bounded_wait(50_000_000, status)  # 50 ms
    torch.cuda.synchronize()
    assert time.perf_counter() - t0 >= 0.05
    assert int(status.item()) == 105
    # the context is still good: a GEMM right after runs and records no error
    a = torch.randn((128, 64), device="cuda").to(torch.bfloat16)
    c = torch.empty((128, 128), device="cuda")
    nat.gemm(a, a, c)
    assert nat.device_status() == 0
    torch.testing.assert_close(c, (a.float() @ a.float().T), rtol=1e-3, atol=1e-3)
    with pytest.raises(nat.CryojaxB200Error):
        nat.selftest_bounded_wait(10_000_000_000, status)  # beyond the 2 s cap
