"""The U-Net's parameter layout: library and CPU oracle agree (CPU only).

``fs_unet_param_count`` and ``fs_unet_layer`` are host-only queries of the
C library; the oracle restates the same layout.
"""

import ctypes

import numpy as np

from fieldspice_b200 import _lib as L
from fieldspice_b200._build import build
from oracle import fs_unet_oracle as UO


def test_parameter_layout_matches_oracle():
    build()
    lib = L.load_library()
    n = ctypes.c_longlong()
    assert lib.fs_unet_param_count(ctypes.byref(n)) == L.FS_OK
    assert n.value == UO.param_count()
    offs, head = UO.layer_offsets()
    ci, co, wo, bo = ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong(), ctypes.c_longlong()
    for l in range(14):
        assert lib.fs_unet_layer(l, ctypes.byref(ci), ctypes.byref(co), ctypes.byref(wo),
                                 ctypes.byref(bo)) == L.FS_OK
        assert (ci.value, co.value) == (UO.CIN[l], UO.COUT[l])
        assert (wo.value, bo.value) == offs[l]
    assert lib.fs_unet_layer(14, ctypes.byref(ci), ctypes.byref(co), ctypes.byref(wo),
                             ctypes.byref(bo)) == L.FS_OK
    assert (wo.value, bo.value) == (head, head + 16)
    assert lib.fs_unet_layer(15, ctypes.byref(ci), ctypes.byref(co), ctypes.byref(wo),
                             ctypes.byref(bo)) == L.FS_BAD_ARG
    nb = ctypes.c_size_t()
    assert lib.fs_unet_workspace_bytes(32, 32, 32, 8, 1, ctypes.byref(nb)) == L.FS_OK
    nb0 = ctypes.c_size_t()
    assert lib.fs_unet_workspace_bytes(32, 32, 32, 8, 0, ctypes.byref(nb0)) == L.FS_OK
    assert nb.value > nb0.value > 34 ** 3 * 8 * 16 * 2
    assert lib.fs_unet_workspace_bytes(32, 32, 32, 65, 0, ctypes.byref(nb0)) == L.FS_BAD_ARG


def test_oracle_gradient_is_a_derivative():
    """Central differences of the oracle loss along a random direction."""
    rng = np.random.default_rng(3)
    dims = (6, 5, 4)
    N = int(np.prod(dims))
    th = UO.init_theta(1).astype(np.float64)
    rhs = rng.standard_normal((1, N))
    em = rng.uniform(0, 0.2, (1, 3, N))
    lab = (rng.random((1, N)) < 0.1).astype(np.uint8)
    tgt = rng.standard_normal((1, N))
    # perturb only the head and the biases (the BF16-rounded convolution
    # weights are piecewise constant)
    offs, head = UO.layer_offsets()
    mask = np.zeros_like(th)
    mask[head:] = 1.0
    for (wo, bo), co in zip(offs, UO.COUT):
        mask[bo:bo + co] = 1.0
    d = rng.standard_normal(th.size) * mask
    _, g = UO.loss_and_grad(th, rhs, em, lab, tgt, dims)
    h = 1e-8
    lp, _ = UO.loss_and_grad(th + h * d, rhs, em, lab, tgt, dims)
    lm, _ = UO.loss_and_grad(th - h * d, rhs, em, lab, tgt, dims)
    fd = (lp - lm) / (2 * h)
    assert abs(fd - g @ d) <= 1e-5 * max(1.0, abs(fd))
