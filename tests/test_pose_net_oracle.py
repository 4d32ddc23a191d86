"""CPU: the pose-network oracle's manual backward against float64 torch autograd."""

import numpy as np

from oracle import pose_net_oracle as PO


def _setup(image_size=64, n_classes=768, B=4, seed=0):
    rng = np.random.default_rng(seed)
    layers, n = PO.layer_table(image_size, n_classes)
    p = np.zeros(n, np.float32)
    for i, L in enumerate(layers):
        std = np.sqrt((2.0 if i < len(layers) - 1 else 1.0) / L["K"])
        p[L["w_off"]:L["w_off"] + L["K"] * L["cout"]] = rng.standard_normal(L["K"] * L["cout"]) * std
        p[L["b_off"]:L["b_off"] + L["cout"]] = rng.standard_normal(L["cout"]) * 0.1
    x = rng.standard_normal((B, image_size, image_size))
    labels = rng.integers(0, n_classes, B)
    nb = rng.integers(0, n_classes, (n_classes, 8)).astype(np.int32)
    return p, x, labels, nb


def test_manual_backward_matches_autograd():
    p, x, labels, nb = _setup()
    for kw in (dict(), dict(neighbours=nb, smoothing=0.2), dict(smoothing=0.1)):
        lo, lr, g = PO.forward_backward(p, x, labels, image_size=64, emulate_bf16=False, **kw)
        lo2, lr2, g2 = PO.autograd_reference(p, x, labels, image_size=64, **kw)
        np.testing.assert_allclose(lo, lo2, rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(lr, lr2, rtol=1e-12)
        np.testing.assert_allclose(g, g2, rtol=1e-9, atol=1e-12 * np.abs(g2).max())


def test_im2col_col2im_adjoint():
    import torch

    rng = np.random.default_rng(1)
    x = torch.as_tensor(rng.standard_normal((2, 8, 8, 3)))
    y = torch.as_tensor(rng.standard_normal((2 * 4 * 4, 27)))
    lhs = float((PO.im2col(x) * y).sum())
    rhs = float((x * PO.col2im(y, 2, 8, 8, 3)).sum())
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
    # K ordering: (ky, kx, c) with pad 1, stride 2
    col = PO.im2col(x)
    assert float(col[5, (3 * 1 + 2) * 3 + 1]) == float(x[0, 2 * 1 + 1 - 1, 2 * 1 + 2 - 1, 1])


def test_layer_table_parameter_count():
    layers, n = PO.layer_table(128, 768)
    assert layers[6]["K"] == 1024 and layers[7]["cout"] == 768
    assert 2.0e6 < n < 2.1e6
