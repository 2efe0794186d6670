"""The tcgen05 GEMM of the surrogate network against a plain PyTorch fp32
reference of the same operation (same bf16 inputs): linear, 5-tap
convolution over levels with the SiLU/residual epilogue, and the backward
epilogue.  Tolerances: f32 outputs 1e-4 relative to the output scale
(accumulation order only); bf16 outputs 1e-2 (one bf16 rounding)."""
import pytest

from openifs_b200 import tcgemm

pytestmark = pytest.mark.gpu
LP, KLEV = 144, 137


@pytest.fixture(params=[0, 1], ids=["warp_specialised", "single_thread"], autouse=True)
def impl(request, cuda):
    tcgemm.set_impl(request.param)
    yield request.param
    tcgemm.set_impl(0)


def _torch():
    import torch
    return torch


def _valid(rows, lp, klev, dev):
    torch = _torch()
    pos = torch.arange(rows, device=dev) % lp
    return ((pos >= 2) & (pos < 2 + klev)).float()[:, None]


def _conv_ref(a, w, taps):
    torch = _torch()
    af = a.float()
    rows = af.shape[0]
    acc = torch.zeros(rows, w.shape[-2], device=a.device)
    for t in range(taps):
        sh = t - taps // 2
        src = torch.zeros_like(af)
        if sh >= 0:
            src[: rows - sh] = af[sh:]
        else:
            src[-sh:] = af[: rows + sh]
        acc += src @ w[t].float().T
    return acc


@pytest.mark.parametrize("n", [64, 128])
def test_linear_f32(cuda, n):
    torch = _torch()
    g = torch.Generator(device="cuda").manual_seed(1)
    rows, k = 1000, 128
    a = torch.randn(rows, k, device="cuda", generator=g).bfloat16()
    w = (torch.randn(1, n, k, device="cuda", generator=g) / k ** 0.5).bfloat16()
    b = torch.randn(n, device="cuda", generator=g)
    out = torch.empty(rows, n, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    tcgemm.conv_gemm(a, w, tcgemm.EPI_LINEAR_F32, n, bias=b, outf=out, err=err)
    torch.cuda.synchronize()
    ref = _conv_ref(a, w, 1) + b
    assert int(err.item()) == 0
    rel = float((out - ref).abs().max() / ref.abs().max())
    assert rel < 1e-4, rel


@pytest.mark.parametrize("k", [128, 256])
def test_conv5_silu_residual(cuda, k):
    torch = _torch()
    g = torch.Generator(device="cuda").manual_seed(2)
    ncol, n = 9, 128
    rows = ncol * LP
    valid = _valid(rows, LP, KLEV, "cuda")
    a = (torch.randn(rows, k, device="cuda", generator=g) * valid).bfloat16()
    w = (torch.randn(5, n, k, device="cuda", generator=g) / (5 * k) ** 0.5).bfloat16()
    b = torch.randn(n, device="cuda", generator=g) * 0.1
    res = (torch.randn(rows, n, device="cuda", generator=g) * valid).bfloat16()
    out = torch.empty(rows, n, device="cuda", dtype=torch.bfloat16)
    pre = torch.empty_like(out)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    tcgemm.conv_gemm(a, w, tcgemm.EPI_SILU, n, taps=5, lp=LP, klev=KLEV, bias=b, out=out, out_pre=pre,
                     resid=res, err=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    z = (_conv_ref(a, w, 5) + b) * valid
    h = (torch.nn.functional.silu(z) + res.float()) * valid
    assert float((pre.float() - z).abs().max()) < 1e-2 * float(z.abs().max())
    assert float((out.float() - h).abs().max()) < 1e-2 * float(h.abs().max())
    # padding rows are exactly zero
    assert float((out.float() * (1 - valid)).abs().max()) == 0.0


def test_backward_epilogue(cuda):
    torch = _torch()
    g = torch.Generator(device="cuda").manual_seed(3)
    ncol, n, k = 8, 128, 128
    rows = ncol * LP
    valid = _valid(rows, LP, KLEV, "cuda")
    a = (torch.randn(rows, k, device="cuda", generator=g) * valid).bfloat16()
    w = (torch.randn(5, n, k, device="cuda", generator=g) / (5 * k) ** 0.5).bfloat16()
    zprev = torch.randn(rows, n, device="cuda", generator=g).bfloat16()
    gres = (torch.randn(rows, n, device="cuda", generator=g) * valid).bfloat16()
    dz = torch.empty(rows, n, device="cuda", dtype=torch.bfloat16)
    gout = torch.empty_like(dz)
    tcgemm.conv_gemm(a, w, tcgemm.EPI_BWD, n, taps=5, lp=LP, klev=KLEV, out=dz, resid=gres,
                     zprev=zprev, gout=gout)
    torch.cuda.synchronize()
    gg = (_conv_ref(a, w, 5) + gres.float()) * valid
    zf = zprev.float()
    s = torch.sigmoid(zf)
    dref = gg * s * (1 + zf * (1 - s)) * valid
    assert float((gout.float() - gg).abs().max()) < 1e-2 * float(gg.abs().max())
    assert float((dz.float() - dref).abs().max()) < 1e-2 * float(dref.abs().max())


def test_many_tiles_persistent(cuda):
    """More tiles than SMs: the persistent tile loop and the stage/phase
    bookkeeping across tiles."""
    torch = _torch()
    g = torch.Generator(device="cuda").manual_seed(4)
    ncol, n, k = 512, 128, 128
    rows = ncol * LP  # 576 tiles of 128 rows
    valid = _valid(rows, LP, KLEV, "cuda")
    a = (torch.randn(rows, k, device="cuda", generator=g) * valid).bfloat16()
    w = (torch.randn(5, n, k, device="cuda", generator=g) / (5 * k) ** 0.5).bfloat16()
    out = torch.empty(rows, n, device="cuda", dtype=torch.bfloat16)
    pre = torch.empty_like(out)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    tcgemm.conv_gemm(a, w, tcgemm.EPI_SILU, n, taps=5, lp=LP, klev=KLEV, out=out, out_pre=pre, err=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    z = _conv_ref(a, w, 5) * valid
    assert float((pre.float() - z).abs().max()) < 1e-2 * float(z.abs().max())
