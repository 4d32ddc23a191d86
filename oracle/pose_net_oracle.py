"""Test infrastructure only: CPU float64 restatement of the pose-proposal
network (forward, softmax cross entropy, manual backward).

The reference has no learned component, so this oracle restates the
network as the device builds it (cryojax_b200/pose_net.py): NHWC
activations, 3x3 stride-2 pad-1 convolutions as im2col with K ordered
(ky, kx, c), weights stored [K][out] in one flat vector (per layer: weight,
then bias), ReLU after every layer but the last, and the loss
-sum_j t_j log softmax_j with t = (1 - eps) at the label plus eps spread
over the label's listed neighbours (or over all classes).

With ``emulate_bf16`` the oracle rounds to BF16 exactly where the device
stores BF16 (weights, every activation, dlogits, every activation
gradient), so the remaining difference is FP32 versus float64 summation;
without it only the weights are BF16 and everything else is float64.
The manual backward is checked against torch autograd (float64, CPU).
"""

from __future__ import annotations

import numpy as np
import torch

CONV_CHANNELS = (1, 32, 64, 128, 128, 256, 256)
HIDDEN = 512


def layer_table(image_size=128, n_classes=768):
    layers, s = [], image_size
    for cin, cout in zip(CONV_CHANNELS[:-1], CONV_CHANNELS[1:]):
        layers.append(dict(kind="conv", cin=cin, cout=cout, h=s, K=9 * cin))
        s //= 2
    feat = CONV_CHANNELS[-1] * s * s
    layers.append(dict(kind="fc", cin=feat, cout=HIDDEN, K=feat))
    layers.append(dict(kind="fc", cin=HIDDEN, cout=n_classes, K=HIDDEN))
    off = 0
    for L in layers:
        L["w_off"] = off
        off += L["K"] * L["cout"]
        L["b_off"] = off
        off += L["cout"]
    return layers, off


def _bf16(t):
    return t.to(torch.bfloat16).to(torch.float64)


def im2col(x):
    """x [B][H][W][C] -> col [B*(H/2)*(W/2)][9C], K = (3 ky + kx) C + c."""
    B, H, W, C = x.shape
    xp = torch.nn.functional.pad(x, (0, 0, 1, 1, 1, 1))
    taps = [xp[:, ky:ky + H:2, kx:kx + W:2, :] for ky in range(3) for kx in range(3)]
    return torch.stack(taps, dim=3).reshape(B * (H // 2) * (W // 2), 9 * C)


def col2im(dcol, B, H, W, C):
    """Adjoint of im2col."""
    d = dcol.reshape(B, H // 2, W // 2, 9, C)
    dxp = torch.zeros((B, H + 2, W + 2, C), dtype=dcol.dtype)
    for ky in range(3):
        for kx in range(3):
            dxp[:, ky:ky + H:2, kx:kx + W:2, :] += d[:, :, :, 3 * ky + kx, :]
    return dxp[:, 1:H + 1, 1:W + 1, :]


def targets(labels, n_classes, neighbours=None, smoothing=0.0):
    B = len(labels)
    t = np.zeros((B, n_classes))
    for r, lab in enumerate(labels):
        t[r, lab] += 1.0 - smoothing
        if smoothing > 0:
            if neighbours is not None and neighbours.shape[1] > 0:
                for q in neighbours[lab]:
                    t[r, q] += smoothing / neighbours.shape[1]
            else:
                t[r] += smoothing / n_classes
    return torch.as_tensor(t)


def forward_backward(params, x, labels, *, image_size=128, n_classes=768, neighbours=None, smoothing=0.0,
                     emulate_bf16=True, trace=None):
    """(logits [B][C], per-row loss [B], grads flat) for the mean loss over the batch.

    params: flat FP32 parameter vector (numpy); x: [B][S][S] network input
    (already BF16 values); labels: [B] ints.
    """
    layers, n = layer_table(image_size, n_classes)
    p = torch.as_tensor(np.asarray(params, np.float32)).to(torch.float64)
    rnd = _bf16 if emulate_bf16 else (lambda t: t)
    W = [_bf16(p[L["w_off"]:L["w_off"] + L["K"] * L["cout"]].reshape(L["K"], L["cout"])) for L in layers]
    b = [p[L["b_off"]:L["b_off"] + L["cout"]] for L in layers]
    B = x.shape[0]
    a = torch.as_tensor(np.asarray(x, np.float64)).reshape(B, image_size, image_size, 1)
    acts, cols = [a], []
    for i, L in enumerate(layers[:6]):
        col = im2col(acts[-1])
        cols.append(col)
        ho = L["h"] // 2
        acts.append(rnd(torch.relu(col @ W[i] + b[i])).reshape(B, ho, ho, L["cout"]))
    feat = acts[6].reshape(B, -1)
    h1 = rnd(torch.relu(feat @ W[6] + b[6]))
    logits = h1 @ W[7] + b[7]
    t = targets(labels, n_classes, neighbours, smoothing)
    logp = torch.log_softmax(logits, dim=1)
    loss = -(t * logp).sum(1)
    g = np.zeros(n)

    def put_w(i, val):
        L = layers[i]
        g[L["w_off"]:L["w_off"] + L["K"] * L["cout"]] = val.reshape(-1).numpy()

    def put_b(i, val):
        L = layers[i]
        g[L["b_off"]:L["b_off"] + L["cout"]] = val.numpy()

    if trace is not None:
        trace["acts"] = [t_.numpy() for t_ in acts]
        trace["h1"] = h1.numpy()
        trace["dy"] = {}
    dl = rnd((torch.exp(logp) - t) / B)
    put_w(7, h1.T @ dl)
    put_b(7, dl.sum(0))
    dh1 = rnd((dl @ W[7].T) * (h1 > 0))
    put_w(6, feat.T @ dh1)
    put_b(6, dh1.sum(0))
    dy = rnd((dh1 @ W[6].T) * (feat > 0))
    for i in range(5, -1, -1):
        L = layers[i]
        dyv = dy.reshape(-1, L["cout"])
        if trace is not None:
            trace["dy"][i] = dyv.numpy()
        put_w(i, cols[i].T @ dyv)
        put_b(i, dyv.sum(0))
        if i == 0:
            break
        dcol = dyv @ W[i].T
        dx = col2im(dcol, B, L["h"], L["h"], L["cin"])
        dy = rnd(dx * (acts[i] > 0))
    return logits.numpy(), loss.numpy(), g


def autograd_reference(params, x, labels, *, image_size=128, n_classes=768, neighbours=None, smoothing=0.0):
    """Float64 torch autograd of the same network (BF16 weights, float64 activations)."""
    layers, n = layer_table(image_size, n_classes)
    p = torch.as_tensor(np.asarray(params, np.float32)).to(torch.float64)
    wb = []
    for L in layers:
        w = _bf16(p[L["w_off"]:L["w_off"] + L["K"] * L["cout"]].reshape(L["K"], L["cout"])).requires_grad_(True)
        bb = p[L["b_off"]:L["b_off"] + L["cout"]].clone().requires_grad_(True)
        wb.append((w, bb))
    B = x.shape[0]
    a = torch.as_tensor(np.asarray(x, np.float64)).reshape(B, image_size, image_size, 1)
    for i, L in enumerate(layers[:6]):
        ho = L["h"] // 2
        a = torch.relu(im2col(a) @ wb[i][0] + wb[i][1]).reshape(B, ho, ho, L["cout"])
    h1 = torch.relu(a.reshape(B, -1) @ wb[6][0] + wb[6][1])
    logits = h1 @ wb[7][0] + wb[7][1]
    t = targets(labels, n_classes, neighbours, smoothing)
    loss = -(t * torch.log_softmax(logits, 1)).sum(1)
    loss.mean().backward()
    g = np.zeros(n)
    for L, (w, bb) in zip(layers, wb):
        g[L["w_off"]:L["w_off"] + L["K"] * L["cout"]] = w.grad.reshape(-1).numpy()
        g[L["b_off"]:L["b_off"] + L["cout"]] = bb.grad.numpy()
    return logits.detach().numpy(), loss.detach().numpy(), g


def adamw_reference(p, g, m, v, step, lr, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0, decay_mask=None):
    """One AdamW step (Loshchilov & Hutter, decoupled weight decay) in float64."""
    p, g, m, v = (np.asarray(a, np.float64) for a in (p, g, m, v))
    m = beta1 * m + (1 - beta1) * g
    v = beta2 * v + (1 - beta2) * g * g
    mh = m / (1 - beta1**step)
    vh = v / (1 - beta2**step)
    wd = weight_decay * (decay_mask if decay_mask is not None else 1.0)
    p = p - lr * (mh / (np.sqrt(vh) + eps) + wd * p)
    return p, m, v
