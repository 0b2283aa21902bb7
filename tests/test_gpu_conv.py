"""Tensor-core 3x3x3 convolution against an FP64 CPU convolution (B200).

The learned preconditioner's convolutions run on tcgen05 in BF16 with FP32
accumulation.  Each case feeds the kernel BF16 inputs and weights and
compares with torch's CPU conv3d in FP64 on the same BF16-rounded values:
the only differences left are FP32 accumulation order and the BF16 rounding
of the output (2^-8 relative).  Halo rows must come back exactly zero.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["v1", "persistent"])
def variant(request, monkeypatch):
    """Both kernels: the one-tile-per-CTA kernel (default) and the persistent
    warp-specialised one (FS_CONV=v2, where it fits)."""
    if request.param == "persistent":
        monkeypatch.setenv("FS_CONV", "v2")
    else:
        monkeypatch.delenv("FS_CONV", raising=False)
    return request.param


def _padded(x):
    """(B, X, Y, Z, C) -> zero-halo (B, X+2, Y+2, Z+2, C)."""
    import torch
    B, X, Y, Z, C = x.shape
    out = torch.zeros((B, X + 2, Y + 2, Z + 2, C), dtype=x.dtype)
    out[:, 1:-1, 1:-1, 1:-1] = x
    return out


def _ref_conv(x, w, bias, relu):
    import torch
    import torch.nn.functional as F
    # x (B, X, Y, Z, Cin) float64; w[27][co][ci] -> torch (co, ci, 3, 3, 3)
    co, ci = w.shape[1], w.shape[2]
    wt = w.reshape(3, 3, 3, co, ci).permute(3, 4, 0, 1, 2)
    y = F.conv3d(x.permute(0, 4, 1, 2, 3), wt, bias=bias, padding=1)
    y = y.permute(0, 2, 3, 4, 1)
    return torch.relu(y) if relu else y


def _run(cuda, xpad_bf16, ctot_in, cin_off, cin, w, bias, ctot_out, cout_off, cout, dims,
         relu=0, mask=None, ctot_mask=0, mask_off=0, y0=None, flip=0):
    import torch
    from fieldspice_b200 import _lib as L
    lib = L.lib()
    B, X, Y, Z = dims
    wd = torch.as_tensor(w, dtype=torch.float32, device=cuda).contiguous()
    wp = torch.empty(w.size, dtype=torch.int16, device=cuda)
    kin, kout = (cout, cin) if flip else (cin, cout)
    L.check("pack", lib.fs_conv3d_pack_weights(L.ptr(wd), kin, kout, flip, L.ptr(wp), L.stream_ptr()))
    xd = xpad_bf16.to(cuda).contiguous()
    yd = (y0.to(cuda).contiguous() if y0 is not None else
          torch.full((B, X + 2, Y + 2, Z + 2, ctot_out), 7.0, dtype=torch.bfloat16, device=cuda))
    bd = torch.as_tensor(bias, dtype=torch.float32, device=cuda) if bias is not None else None
    md = mask.to(cuda).contiguous() if mask is not None else None
    err = torch.zeros(1, dtype=torch.int32, device=cuda)
    st = lib.fs_conv3d_bf16(L.ptr(xd), ctot_in, cin_off, cin, L.ptr(wp), L.ptr(bd), L.ptr(yd),
                            ctot_out, cout_off, cout, L.ptr(md), ctot_mask, mask_off, B, X, Y, Z,
                            relu, 1 if y0 is not None else 0, L.ptr(err), L.stream_ptr())
    L.check("fs_conv3d_bf16", st)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return yd.cpu()


def _bf(a):
    import torch
    return torch.as_tensor(a).to(torch.bfloat16)


def _close(got, want):
    import torch
    got = got.to(torch.float64)
    scale = want.abs().max().item()
    err = (got - want).abs()
    assert (err <= 2.0 ** -7 * want.abs() + 2e-3 * scale).all(), err.max().item()


@pytest.mark.parametrize("dims,cin,cout", [((2, 7, 9, 11), 16, 16), ((1, 12, 10, 9), 32, 48),
                                           ((3, 5, 6, 4), 64, 64), ((1, 6, 6, 30), 112, 48),
                                           ((2, 4, 4, 70), 16, 32), ((4, 20, 18, 16), 16, 16),
                                           ((8, 24, 24, 30), 16, 32)])
def test_conv_forward_matches_fp64(cuda, variant, dims, cin, cout):
    import torch
    rng = np.random.default_rng(cin * 100 + cout)
    B, X, Y, Z = dims
    x = _bf(rng.standard_normal((B, X, Y, Z, cin)).astype(np.float32))
    w = _bf(rng.standard_normal((27, cout, cin)).astype(np.float32) / np.sqrt(27 * cin))
    bias = rng.standard_normal(cout).astype(np.float32)
    got = _run(cuda, _padded(x), cin, 0, cin, w.float().numpy(), bias, cout, 0, cout, dims, relu=1)
    want = _ref_conv(x.double(), w.double(), torch.as_tensor(bias, dtype=torch.float64), True)
    _close(got[:, 1:-1, 1:-1, 1:-1], want)
    halo = got.clone()
    halo[:, 1:-1, 1:-1, 1:-1] = 0
    assert halo.abs().max().item() == 0.0


def test_conv_channel_slices_mask_and_accumulate(cuda):
    import torch
    rng = np.random.default_rng(5)
    dims = (2, 6, 7, 8)
    B, X, Y, Z = dims
    full = _bf(rng.standard_normal((B, X, Y, Z, 64)).astype(np.float32))
    w = _bf(rng.standard_normal((27, 16, 48)).astype(np.float32) / 30)
    m = _bf(rng.standard_normal((B, X, Y, Z, 32)).astype(np.float32))
    y0 = _bf(rng.standard_normal((B, X, Y, Z, 48)).astype(np.float32))
    got = _run(cuda, _padded(full), 64, 16, 48, w.float().numpy(), None, 48, 32, 16, dims,
               mask=_padded(m), ctot_mask=32, mask_off=16, y0=_padded(y0))
    ref = _ref_conv(full[..., 16:].double(), w.double(), None, False)
    ref = ref * (m[..., 16:32].double() > 0)
    want = y0.double().clone()
    want[..., 32:48] += ref
    _close(got[:, 1:-1, 1:-1, 1:-1], want)


@pytest.mark.parametrize("cin,cout", [(16, 32), (112, 48)])
def test_conv_data_gradient_matches_autograd(cuda, variant, cin, cout):
    """The flipped pack turns the kernel into dL/dx of the forward conv."""
    import torch
    import torch.nn.functional as F
    rng = np.random.default_rng(cin + cout)
    dims = (2, 5, 6, 9)
    B, X, Y, Z = dims
    x = torch.zeros((B, X, Y, Z, cin), dtype=torch.float64, requires_grad=True)
    w = _bf(rng.standard_normal((27, cout, cin)).astype(np.float32) / 20)
    dy = _bf(rng.standard_normal((B, X, Y, Z, cout)).astype(np.float32))
    y = _ref_conv(x, w.double(), None, False)
    y.backward(dy.double())
    want = x.grad
    got = _run(cuda, _padded(dy), cout, 0, cout, w.float().numpy(), None, cin, 0, cin, dims, flip=1)
    _close(got[:, 1:-1, 1:-1, 1:-1], want)


@pytest.mark.parametrize("dims,cin,cout,slices", [
    ((2, 5, 6, 9), 16, 32, False), ((1, 7, 6, 20), 48, 48, False),
    ((2, 4, 5, 6), 112, 48, True), ((1, 6, 6, 30), 64, 64, False),
    ((3, 9, 8, 7), 80, 32, True), ((1, 20, 18, 16), 16, 16, False)])
def test_conv_weight_gradient_matches_autograd(cuda, dims, cin, cout, slices):
    """fs_conv3d_wgrad_bf16 (tensor cores, voxels as the reduction index) is
    dL/dW and dL/db of the forward conv: FP64 autograd on the same BF16
    inputs, FP32 accumulation differences only (channel slices of wider
    volumes where ``slices``)."""
    import torch
    from fieldspice_b200 import _lib as L
    lib = L.lib()
    rng = np.random.default_rng(cin * 7 + cout)
    B, X, Y, Z = dims
    x = _bf(rng.standard_normal((B, X, Y, Z, cin)).astype(np.float32))
    dy = _bf(rng.standard_normal((B, X, Y, Z, cout)).astype(np.float32))
    w = torch.zeros((27, cout, cin), dtype=torch.float64, requires_grad=True)
    b = torch.zeros(cout, dtype=torch.float64, requires_grad=True)
    y = _ref_conv(x.double(), w, b, False)
    y.backward(dy.double())
    xo, yo = (8, 16) if slices else (0, 0)
    ctx, cty = cin + xo + (8 if slices else 0), cout + yo
    xp = torch.zeros((B, X + 2, Y + 2, Z + 2, ctx), dtype=torch.bfloat16)
    xp[..., xo:xo + cin] = _padded(x)
    yp = torch.zeros((B, X + 2, Y + 2, Z + 2, cty), dtype=torch.bfloat16)
    yp[..., yo:yo + cout] = _padded(dy)
    xd, yd = xp.to(cuda).contiguous(), yp.to(cuda).contiguous()
    nb = __import__("ctypes").c_size_t()
    L.check("ws", lib.fs_conv3d_wgrad_workspace_bytes(cin, cout, __import__("ctypes").byref(nb)))
    ws = torch.empty(nb.value, dtype=torch.uint8, device=cuda)
    dw = torch.full((27, cout, cin), np.nan, dtype=torch.float32, device=cuda)
    db = torch.full((cout,), np.nan, dtype=torch.float32, device=cuda)
    err = torch.zeros(1, dtype=torch.int32, device=cuda)
    L.check("fs_conv3d_wgrad_bf16", lib.fs_conv3d_wgrad_bf16(
        L.ptr(xd), ctx, xo, cin, L.ptr(yd), cty, yo, cout, B, X, Y, Z, L.ptr(dw), L.ptr(db),
        L.ptr(ws), nb.value, L.ptr(err), L.stream_ptr()))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    gw, gb = dw.cpu().double(), db.cpu().double()
    # FP32 sums of up to ~1e4 products of unit-scale BF16 values
    assert (gw - w.grad).abs().max().item() <= 2e-5 * w.grad.abs().max().item() + 1e-3
    assert (gb - b.grad).abs().max().item() <= 2e-5 * b.grad.abs().max().item() + 1e-3
