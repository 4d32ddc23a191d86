"""Pose-proposal network: a small CNN that maps a noisy particle image to a
distribution over the HEALPix viewing directions of the orientation grid.

Architecture (about 2.05 M parameters): six 3x3 stride-2 convolutions with
ReLU, channels 1 -> 32 -> 64 -> 128 -> 128 -> 256 -> 256 (a 128^2 image ends
at 2 x 2 x 256 = 1024 features), then dense 1024 -> 512 (ReLU) -> 768
logits, one per direction.  Weights and activations are BF16, accumulation
is FP32 on the tensor cores (cjx_gemm: TMA + tcgen05.mma + TMEM); the FP32
master weights, gradients and AdamW moments live in one flat vector.

Every layer is an implicit GEMM over NHWC activations:
  forward   col = im2col(x);  y = relu(col W^T + b)           (bias+ReLU fused)
  backward  dWt = col^T dY      (split-K, FP32 atomics)
            db  = colsum(dY)
            dx  = col2im(dY Wt^T) * (x > 0)                    (ReLU mask fused)
with W the BF16 copy [out][K] and Wt = W^T [K][out] refreshed by the AdamW
kernel.  K is ordered (ky, kx, c), matching the NHWC im2col.

The reference has no learned component (its pose search is a plain grid
search, cryojax/jax_util/_grid_search/search_loop.py:24-158); this network
only proposes candidates that the grid search's scorer rescores.
"""

from __future__ import annotations

import numpy as np

from . import _native as nat


def _torch():
    import torch

    return torch


CONV_CHANNELS = (1, 32, 64, 128, 128, 256, 256)
HIDDEN = 512
INFER_BATCH = 2048  # largest batch of one proposal forward pass


def _round8(x):
    return (x + 7) // 8 * 8


class PoseProposalNet:
    """Parameters, buffers and the forward / backward / AdamW launches.

    ``max_batch`` fixes the activation buffers (rounded up to a multiple of
    8, the GEMM operand pitch); calls may use any batch up to it.
    """

    def __init__(self, image_size: int = 128, n_classes: int = 768, *, max_batch: int = 256, seed: int = 0,
                 device="cuda"):
        torch = _torch()
        if image_size % 64:
            raise ValueError("image_size must be a multiple of 64 (six stride-2 layers)")
        self.image_size = image_size
        self.n_classes = n_classes
        self.device = torch.device(device)
        self.max_batch = _round8(max_batch)
        # layer table
        self.layers = []
        s = image_size
        for cin, cout in zip(CONV_CHANNELS[:-1], CONV_CHANNELS[1:]):
            k = 9 * cin
            self.layers.append(dict(kind="conv", cin=cin, cout=cout, h=s, w=s, K=k, ldk=_round8(k)))
            s //= 2
        feat = CONV_CHANNELS[-1] * s * s
        self.final_spatial = s
        self.layers.append(dict(kind="fc", cin=feat, cout=HIDDEN, K=feat, ldk=feat))
        self.layers.append(dict(kind="fc", cin=HIDDEN, cout=n_classes, K=HIDDEN, ldk=HIDDEN))
        # flat parameter vector: per layer weight [K][cout] then bias [cout]
        off = 0
        for L in self.layers:
            L["w_off"] = off
            off += L["K"] * L["cout"]
            L["b_off"] = off
            off += L["cout"]
        self.n_params = off
        f32 = dict(device=self.device, dtype=torch.float32)
        self.params = torch.zeros(off, **f32)
        self.grads = torch.zeros(off, **f32)
        self.m = torch.zeros(off, **f32)
        self.v = torch.zeros(off, **f32)
        g = torch.Generator(device="cpu")
        g.manual_seed(seed)
        for i, L in enumerate(self.layers):
            std = np.sqrt((2.0 if i < len(self.layers) - 1 else 1.0) / L["K"])  # He init; plain for the logits
            w = torch.randn((L["K"], L["cout"]), generator=g, dtype=torch.float32) * std
            self.params[L["w_off"]:L["w_off"] + w.numel()] = w.reshape(-1).to(self.device)
        for L in self.layers:
            L["W"] = torch.zeros((L["cout"], L["ldk"]), device=self.device, dtype=torch.bfloat16)
            L["Wt"] = torch.zeros((L["K"], L["cout"]), device=self.device, dtype=torch.bfloat16)
        self._segments = self._make_segments()
        self.refresh_bf16_weights()
        self.step_count = 0
        self._alloc(self.max_batch)

    # ---- parameter views ------------------------------------------------
    def weight(self, i):
        L = self.layers[i]
        return self.params[L["w_off"]:L["w_off"] + L["K"] * L["cout"]].view(L["K"], L["cout"])

    def bias(self, i):
        L = self.layers[i]
        return self.params[L["b_off"]:L["b_off"] + L["cout"]]

    def weight_grad(self, i):
        L = self.layers[i]
        return self.grads[L["w_off"]:L["w_off"] + L["K"] * L["cout"]].view(L["K"], L["cout"])

    def bias_grad(self, i):
        L = self.layers[i]
        return self.grads[L["b_off"]:L["b_off"] + L["cout"]]

    def _make_segments(self):
        segs = (nat.ParamSegment * (2 * len(self.layers)))()
        for i, L in enumerate(self.layers):
            w = segs[2 * i]
            w.offset, w.count, w.cols, w.ldk = L["w_off"], L["K"] * L["cout"], L["cout"], L["ldk"]
            w.w_bf16, w.wt_bf16, w.weight_decay = L["W"].data_ptr(), L["Wt"].data_ptr(), 1
            b = segs[2 * i + 1]
            b.offset, b.count, b.cols, b.ldk, b.weight_decay = L["b_off"], L["cout"], 0, 0, 0
        return segs

    def refresh_bf16_weights(self):
        """BF16 copies W [out][ldk] and Wt [K][out] of the FP32 master weights."""
        for i, L in enumerate(self.layers):
            w = self.weight(i)
            nat.transpose_to_bf16(w, L["K"], L["cout"], L["cout"], L["W"], L["ldk"])
            L["Wt"].copy_(w.to(_torch().bfloat16))

    def state_dict(self):
        return {"params": self.params.detach().cpu().numpy().copy(), "image_size": self.image_size,
                "n_classes": self.n_classes, "step": self.step_count}

    def load_state_dict(self, sd):
        torch = _torch()
        if sd["params"].shape != (self.n_params,):
            raise ValueError("parameter vector size mismatch")
        self.params.copy_(torch.as_tensor(sd["params"], device=self.device))
        self.refresh_bf16_weights()
        self.step_count = int(sd.get("step", 0))

    # ---- buffers ----------------------------------------------------------
    def _forward_buffers(self, B):
        """Input, im2col, activation and logit buffers of a forward pass over up to B images."""
        torch = _torch()
        bf, f32 = dict(device=self.device, dtype=torch.bfloat16), dict(device=self.device, dtype=torch.float32)
        S = self.image_size
        x0 = torch.empty((B, S, S), **bf)
        acts, cols = [x0], []
        for L in self.layers[:6]:
            ho = L["h"] // 2
            cols.append(torch.empty((B * ho * ho, L["ldk"]), **bf))
            acts.append(torch.empty((B, ho, ho, L["cout"]), **bf))
        return dict(B=B, x0=x0, acts=acts, cols=cols, h1=torch.empty((B, HIDDEN), **bf),
                    logits=torch.empty((B, self.n_classes), **f32))

    def _alloc(self, B):
        torch = _torch()
        bf, f32 = dict(device=self.device, dtype=torch.bfloat16), dict(device=self.device, dtype=torch.float32)
        self._fwd = self._forward_buffers(B)
        self.x0, self.acts, self.cols = self._fwd["x0"], self._fwd["acts"], self._fwd["cols"]
        self.h1, self.logits = self._fwd["h1"], self._fwd["logits"]
        self._infer = None  # forward-only buffers for larger inference batches (propose)
        # backward scratch (sized for the largest layer)
        self.dlogits = torch.empty((B, self.n_classes), **bf)
        self.loss_rows = torch.empty(B, **f32)
        max_pix_k = max(c.numel() for c in self.cols)
        self.t_col = torch.empty(max_pix_k, **bf)                          # col^T
        self.t_dy = torch.empty(max(a.numel() for a in self.acts[1:]) + B * self.n_classes, **bf)  # dY^T
        self.dcol = torch.empty(max_pix_k, **f32)                          # dY Wt^T (FP32)
        self.dy_a = torch.empty(max(a.numel() for a in self.acts), **bf)   # dY ping
        self.dy_b = torch.empty(max(a.numel() for a in self.acts), **bf)   # dY pong
        self.g32 = torch.empty(B * max(1024, self.layers[6]["cin"]), **f32)
        self._B = B

    # ---- forward ----------------------------------------------------------
    def forward(self, x_bf16=None, *, B=None, stream=None, buffers=None, direct_first_layer=False,
                implicit_convs=False):
        """Logits [B][n_classes] (FP32) for the images in x0[:B] (or x_bf16 copied there) of `buffers`
        (default: the training buffers, which backward reads).  ``direct_first_layer`` computes the first
        convolution and ``implicit_convs`` the others without their im2col matrices (inference only:
        backward reads those matrices)."""
        buf = self._fwd if buffers is None else buffers
        cap = buf["B"]
        B = cap if B is None else B
        if B > cap or B % 8:
            raise ValueError(f"batch {B} must be a multiple of 8 and <= {cap}")
        x0, acts, cols = buf["x0"], buf["acts"], buf["cols"]
        if x_bf16 is not None:
            x0[:B].copy_(x_bf16.reshape(B, self.image_size, self.image_size))
        for i, L in enumerate(self.layers[:6]):
            ho = L["h"] // 2
            npix = B * ho * ho
            if i == 0 and direct_first_layer and L["cin"] == 1 and L["cout"] == 32:
                nat.cnn_conv0(acts[0], B, L["h"], L["w"], L["W"], L["ldk"], L["cout"], self.bias(0), acts[1],
                              stream=stream)
                continue
            if i > 0 and implicit_convs:
                nat.cnn_conv_s2(acts[i], B, L["h"], L["w"], L["cin"], L["W"], L["ldk"], L["cout"], self.bias(i),
                                acts[i + 1], stream=stream)
                continue
            nat.cnn_im2col(acts[i], B, L["h"], L["w"], L["cin"], cols[i], L["ldk"], stream=stream)
            nat.gemm(cols[i], L["W"], acts[i + 1].view(-1, L["cout"]), m=npix, n=L["cout"], k=L["K"],
                     bias=self.bias(i),
                     flags=nat.CJX_GEMM_RELU | nat.CJX_GEMM_OUT_BF16, stream=stream)
        L6, L7 = self.layers[6], self.layers[7]
        feat = acts[6].view(cap, -1)
        nat.gemm(feat, L6["W"], buf["h1"], m=B, n=HIDDEN, k=L6["K"], bias=self.bias(6),
                 flags=nat.CJX_GEMM_RELU | nat.CJX_GEMM_OUT_BF16, stream=stream)
        nat.gemm(buf["h1"], L7["W"], buf["logits"], m=B, n=self.n_classes, k=L7["K"], bias=self.bias(7),
                 stream=stream)
        return buf["logits"][:B]

    # ---- backward -----------------------------------------------------------
    def backward(self, labels, *, B=None, neighbours=None, smoothing=0.0, stream=None):
        """Accumulate d(mean loss)/d(params) into self.grads (zeroed here); returns per-row losses."""
        torch = _torch()
        B = self._B if B is None else B
        self.grads.zero_()
        nat.softmax_xent(self.logits, labels, neighbours=neighbours, smoothing=smoothing, grad_scale=1.0 / B,
                         loss=self.loss_rows, dlogits=self.dlogits, B=B, stream=stream)
        # dense 2: dWt [512][C] = h1^T dlogits
        L7 = self.layers[7]
        C = self.n_classes
        h1T = self.t_col[:HIDDEN * B].view(HIDDEN, B)
        dlT = self.t_dy[:C * B].view(C, B)
        nat.transpose_to_bf16(self.h1, B, HIDDEN, HIDDEN, h1T, B, stream=stream)
        nat.transpose_to_bf16(self.dlogits, B, C, C, dlT, B, stream=stream)
        nat.gemm(h1T, dlT, self.weight_grad(7), m=HIDDEN, n=C, k=B, stream=stream)
        nat.colsum(self.dlogits, B, C, C, self.bias_grad(7), stream=stream)
        g = self.g32[:B * HIDDEN].view(B, HIDDEN)
        nat.gemm(self.dlogits, L7["Wt"], g, m=B, n=HIDDEN, k=C, stream=stream)
        dh1 = self.dy_a[:B * HIDDEN].view(B, HIDDEN)
        nat.relu_mask(g, self.h1, B * HIDDEN, dh1, stream=stream)
        # dense 1: dWt [feat][512] = a6^T dh1
        L6 = self.layers[6]
        F = L6["K"]
        feat = self.acts[6].view(self._B, -1)
        aT = self.t_col[:F * B].view(F, B)
        dT = self.t_dy[:HIDDEN * B].view(HIDDEN, B)
        nat.transpose_to_bf16(feat, B, F, F, aT, B, stream=stream)
        nat.transpose_to_bf16(dh1, B, HIDDEN, HIDDEN, dT, B, stream=stream)
        nat.gemm(aT, dT, self.weight_grad(6), m=F, n=HIDDEN, k=B, stream=stream)
        nat.colsum(dh1, B, HIDDEN, HIDDEN, self.bias_grad(6), stream=stream)
        g = self.g32[:B * F].view(B, F)
        nat.gemm(dh1, L6["Wt"], g, m=B, n=F, k=HIDDEN, stream=stream)
        dy = self.dy_b
        nat.relu_mask(g, feat, B * F, dy, stream=stream)
        # convolutions, last to first; dy holds dL/d(output of layer i) (ReLU applied)
        for i in range(5, -1, -1):
            L = self.layers[i]
            ho = L["h"] // 2
            npix = B * ho * ho
            K, cout = L["K"], L["cout"]
            dyv = dy[:npix * cout].view(npix, cout)
            colT = self.t_col[:K * npix].view(K, npix)
            dyT = self.t_dy[:cout * npix].view(cout, npix)
            nat.transpose_to_bf16(self.cols[i], npix, K, L["ldk"], colT, npix, stream=stream)
            nat.transpose_to_bf16(dyv, npix, cout, cout, dyT, npix, stream=stream)
            tiles = ((K + 127) // 128) * ((cout + 127) // 128)
            nk = (npix + 63) // 64
            split = int(max(1, min(nk // 4, (2 * 148) // max(tiles, 1))))
            nat.gemm(colT, dyT, self.weight_grad(i), m=K, n=cout, k=npix, flags=nat.CJX_GEMM_ACCUMULATE,
                     split_k=split, stream=stream)
            nat.colsum(dyv, npix, cout, cout, self.bias_grad(i), stream=stream)
            if i == 0:
                break
            dcol = self.dcol[:npix * L["ldk"]].view(npix, L["ldk"])
            nat.gemm(dyv, L["Wt"], dcol, m=npix, n=K, k=cout, stream=stream)
            nxt = self.dy_a if dy is self.dy_b else self.dy_b
            nat.cnn_col2im(dcol, L["ldk"], self.acts[i], B, L["h"], L["w"], L["cin"], nxt, stream=stream)
            dy = nxt
        return self.loss_rows[:B]

    def adam_step(self, lr, *, weight_decay=0.0, beta1=0.9, beta2=0.999, eps=1e-8, stream=None):
        self.step_count += 1
        nat.adamw(self.params, self.grads, self.m, self.v, self._segments, lr=lr, beta1=beta1, beta2=beta2, eps=eps,
                  weight_decay=weight_decay, step=self.step_count, stream=stream)

    # ---- inference ------------------------------------------------------------
    def propose(self, images, k=16, n_inplane=48, *, batch=None, stream=None):
        """Top-k directions (n, k) and candidate orientations (n, k * n_inplane), int32 CUDA tensors.

        images: float32 CUDA tensor (n, S, S) of real-space images; each is
        normalised (zero mean, unit std) on the device before the network.
        """
        torch = _torch()
        n = images.shape[0]
        # batches beyond the training buffers' size use forward-only buffers of up to INFER_BATCH images
        # (about 1.7 MB each at 128^2), allocated once: fewer, larger GEMMs per layer
        want = _round8(min(max(n, 1), INFER_BATCH)) if batch is None else _round8(batch)
        if want <= self._B:
            buf = self._fwd
        else:
            if self._infer is None or self._infer["B"] < want:
                self._infer = None
                self._infer = self._forward_buffers(want)
            buf = self._infer
        batch = buf["B"] if batch is None else min(batch, buf["B"])
        x0 = buf["x0"]
        dirs = torch.empty((n, k), dtype=torch.int32, device=self.device)
        cand = torch.empty((n, k * n_inplane), dtype=torch.int32, device=self.device)
        for s in range(0, n, batch):
            cnt = min(batch, n - s)
            b8 = _round8(cnt)
            nat.cnn_noisy_normalize(images[s:s + cnt].contiguous(), x0, n=cnt, stream=stream)
            if b8 > cnt:
                x0[cnt:b8].zero_()
            logits = self.forward(B=b8, stream=stream, buffers=buf, direct_first_layer=True, implicit_convs=True)
            nat.topk_candidates(logits, k, n_inplane, dirs=dirs[s:s + cnt], candidates=cand[s:s + cnt], B=cnt,
                                stream=stream)
        return dirs, cand
