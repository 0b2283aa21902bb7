"""The learned preconditioner's U-Net on the GPU against the CPU FP64 oracle.

The network runs on this library's kernels: fourteen 3x3x3 convolutions and
their data gradients on tcgen05 tensor cores (BF16 operands, FP32
accumulation), weight gradients, pooling, upsampling, head and Adam on CUDA
cores.  oracle/fs_unet_oracle.py restates the same network in PyTorch CPU
FP64 with autograd.  BF16 activations give ~1% relative differences, so the
forward output is compared in relative L2 norm (<= 3%) and the gradient by
direction (cosine >= 0.99) and size (relative norm <= 5%).
"""

import ctypes

import numpy as np
import pytest

from oracle import fs_unet_oracle as UO

pytestmark = pytest.mark.gpu


def _net(cuda, dims, batch, theta, train=1):
    import torch
    from fieldspice_b200 import _lib as L
    lib = L.lib()
    nb = ctypes.c_size_t()
    L.check("ws", lib.fs_unet_workspace_bytes(*dims, batch, train, ctypes.byref(nb)))
    ws = torch.empty(nb.value, dtype=torch.uint8, device=cuda)
    th = torch.as_tensor(theta, dtype=torch.float32, device=cuda).contiguous()
    net = ctypes.c_void_p()
    L.check("fs_unet_create", lib.fs_unet_create(*dims, batch, train, L.ptr(th), L.ptr(ws),
                                                 nb.value, ctypes.byref(net), L.stream_ptr()))
    return net, th, ws


def _data(dims, batch, seed):
    rng = np.random.default_rng(seed)
    N = int(np.prod(dims))
    rhs = rng.standard_normal((batch, N)).astype(np.float32) * 1e-3
    em = rng.uniform(0.0, 0.18, (batch, 3, N)).astype(np.float32)
    lab = (rng.random((batch, N)) < 0.08).astype(np.uint8)
    tgt = rng.standard_normal((batch, N)).astype(np.float32) * 1e-2
    return rhs, em, lab, tgt


def _dev(cuda, *arrs):
    import torch
    return [torch.as_tensor(a, device=cuda).contiguous() for a in arrs]


@pytest.mark.parametrize("dims", [(12, 10, 9), (20, 16, 12)])
def test_unet_forward_matches_oracle(cuda, dims):
    import torch
    from fieldspice_b200 import _lib as L
    lib = L.lib()
    B = 2
    theta = UO.init_theta(7)
    net, th, ws = _net(cuda, dims, B, theta, train=0)
    rhs, em, lab, _ = _data(dims, B, 1)
    N = int(np.prod(dims))
    r, e, l = _dev(cuda, rhs, em, lab)
    out = torch.zeros((B, N), dtype=torch.float32, device=cuda)
    L.check("fwd", lib.fs_unet_forward(net, L.ptr(r), 1, N, L.ptr(e), 3 * N, L.ptr(l), N,
                                       L.ptr(out), 1, N, L.stream_ptr()))
    got = out.cpu().numpy().astype(np.float64)
    want, _ = UO.forward(torch.as_tensor(theta, dtype=torch.float64), rhs, em, lab, dims,
                         normalised=False)
    want = want.numpy()
    assert np.all(got[lab == 1] == 0.0)
    assert np.linalg.norm(got - want) <= 3e-2 * np.linalg.norm(want)
    flag = ctypes.c_int(1)
    L.check("err", lib.fs_unet_error(net, ctypes.byref(flag), L.stream_ptr()))
    assert flag.value == 0
    lib.fs_unet_destroy(net)


def test_unet_gradient_matches_oracle(cuda):
    import torch
    from fieldspice_b200 import _lib as L
    lib = L.lib()
    dims, B = (12, 10, 9), 2
    theta = UO.init_theta(11)
    net, th, ws = _net(cuda, dims, B, theta)
    rhs, em, lab, tgt = _data(dims, B, 2)
    r, e, l, t = _dev(cuda, rhs, em, lab, tgt)
    grad = torch.zeros(theta.size, dtype=torch.float32, device=cuda)
    loss = torch.zeros(1, dtype=torch.float32, device=cuda)
    L.check("grad", lib.fs_unet_gradient(net, L.ptr(r), L.ptr(e), L.ptr(l), L.ptr(t),
                                         L.ptr(grad), L.ptr(loss), L.stream_ptr()))
    g = grad.cpu().numpy().astype(np.float64)
    lw, gw = UO.loss_and_grad(theta, rhs, em, lab, tgt, dims)
    assert abs(float(loss.item()) - lw) <= 2e-2 * lw
    cos = g @ gw / (np.linalg.norm(g) * np.linalg.norm(gw))
    assert cos >= 0.99, cos
    assert abs(np.linalg.norm(g) - np.linalg.norm(gw)) <= 5e-2 * np.linalg.norm(gw)
    # every layer's weight gradient, not only the dominant ones
    offs, head = UO.layer_offsets()
    for li, (wo, bo) in enumerate(offs):
        a, b = g[wo:bo], gw[wo:bo]
        c = a @ b / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-300)
        assert c >= 0.97, (li, c)
    lib.fs_unet_destroy(net)


def test_unet_training_reduces_the_loss(cuda):
    """Adam on the library's gradients: a fixed batch whose target is a
    smooth function of the input is fitted (loss falls at least 4x)."""
    import torch
    from fieldspice_b200 import _lib as L
    lib = L.lib()
    dims, B = (16, 16, 12), 4
    theta = UO.init_theta(3)
    net, th, ws = _net(cuda, dims, B, theta)
    rhs, em, lab, _ = _data(dims, B, 5)
    # target: a blurred copy of the input (a smooth, learnable map)
    v = rhs.reshape(B, *dims).astype(np.float64)
    for ax in (1, 2, 3):
        v = 0.25 * np.roll(v, 1, ax) + 0.5 * v + 0.25 * np.roll(v, -1, ax)
    tgt = (v.reshape(B, -1) * (lab == 0)).astype(np.float32)
    r, e, l, t = _dev(cuda, rhs, em, lab, tgt)
    loss = torch.zeros(1, dtype=torch.float32, device=cuda)
    hist = []
    for it in range(60):
        L.check("step", lib.fs_unet_train_step(net, L.ptr(r), L.ptr(e), L.ptr(l), L.ptr(t),
                                               ctypes.c_float(2e-3), L.ptr(loss), L.stream_ptr()))
        hist.append(float(loss.item()))
    assert np.all(np.isfinite(hist))
    assert hist[-1] < hist[0] / 4, hist[::10]
    lib.fs_unet_destroy(net)


def test_gradient_then_adam_step_equals_train_step(cuda):
    """The data-parallel training primitive: fs_unet_gradient followed by
    fs_unet_adam_step on that gradient gives bit for bit the theta of
    fs_unet_train_step (three steps on the same batches), and an averaged
    gradient of two half batches drives the same update path."""
    import torch
    from fieldspice_b200 import _lib as L
    lib = L.lib()
    dims, B = (12, 10, 9), 4
    theta = UO.init_theta(7)
    net_a, th_a, ws_a = _net(cuda, dims, B, theta)
    net_b, th_b, ws_b = _net(cuda, dims, B, theta)
    r, e, l, t = _dev(cuda, *_data(dims, B, 8))
    loss = torch.zeros(1, dtype=torch.float32, device=cuda)
    grad = torch.empty_like(th_b)
    for it in range(3):
        lr = ctypes.c_float(1e-3 * (it + 1))
        L.check("step", lib.fs_unet_train_step(net_a, L.ptr(r), L.ptr(e), L.ptr(l), L.ptr(t),
                                               lr, L.ptr(loss), L.stream_ptr()))
        L.check("grad", lib.fs_unet_gradient(net_b, L.ptr(r), L.ptr(e), L.ptr(l), L.ptr(t),
                                             L.ptr(grad), L.ptr(loss), L.stream_ptr()))
        L.check("adam", lib.fs_unet_adam_step(net_b, L.ptr(grad), lr, L.stream_ptr()))
    torch.cuda.synchronize()
    assert torch.equal(th_a, th_b)
    assert not torch.equal(th_a, torch.as_tensor(theta, dtype=torch.float32, device=cuda))
    assert lib.fs_unet_adam_step(net_b, None, ctypes.c_float(1e-3), L.stream_ptr()) == L.FS_BAD_ARG
    lib.fs_unet_destroy(net_a)
    lib.fs_unet_destroy(net_b)
