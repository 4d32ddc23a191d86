"""GPU: the pose-proposal network's own kernels against the CPU float64 oracle.

Forward + backward are compared with oracle/pose_net_oracle.py in two
modes.  Emulating the device's BF16 storage points, the only differences are
FP32-versus-float64 sums that flip a BF16 rounding now and then; the flips
cascade through the layers (a few percent of the last activations differ by
an ulp), so the tolerances are: logits and losses rel 3e-3, every
parameter-gradient tensor rel L2 3e-2.  Against pure float64 activations
the device must be no farther than the BF16-emulating oracle itself
(1.5x its distance + 0.02 per tensor): BF16 activations alone move the
gradients by about 5-15 % in these random-weight networks.
"""

import numpy as np
import pytest

from oracle import pose_net_oracle as PO

pytestmark = pytest.mark.gpu

EMU_LOGIT_TOL = 3e-3
EMU_GRAD_TOL = 3e-2


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a - b)) / max(np.linalg.norm(np.ravel(b)), 1e-30))


def _net_and_batch(image_size=64, B=16, seed=0):
    import torch

    from cryojax_b200 import _native as nat
    from cryojax_b200.pose_net import PoseProposalNet

    net = PoseProposalNet(image_size, 768, max_batch=B, seed=seed)
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    with torch.no_grad():  # nonzero biases exercise the bias paths
        for i in range(len(net.layers)):
            net.bias(i).copy_(torch.randn(net.layers[i]["cout"], generator=g, device="cuda") * 0.05)
    imgs = torch.randn((B, image_size, image_size), generator=g, device="cuda")
    nat.cnn_noisy_normalize(imgs, net.x0, n=B)
    labels = torch.randint(0, 768, (B,), generator=g, device="cuda", dtype=torch.int32)
    return net, labels


def _grad_tensors(net, g):
    out = []
    for L in net.layers:
        out.append(g[L["w_off"]:L["w_off"] + L["K"] * L["cout"]])
        out.append(g[L["b_off"]:L["b_off"] + L["cout"]])
    return out


@pytest.mark.parametrize("smoothing,use_nb", [(0.0, False), (0.2, True)])
def test_forward_backward_against_oracle(cuda_device, smoothing, use_nb):
    import torch

    from cryojax_b200 import _native as nat

    B, S = 16, 64
    net, labels = _net_and_batch(S, B)
    nb = torch.randint(0, 768, (768, 8), device="cuda", dtype=torch.int32) if use_nb else None
    logits = net.forward(B=B).cpu().numpy().copy()
    loss = net.backward(labels, B=B, neighbours=nb, smoothing=smoothing).cpu().numpy().copy()
    assert nat.device_status() == 0
    grads = net.grads.cpu().numpy()
    x = net.x0[:B].float().cpu().numpy()
    params = net.params.cpu().numpy()
    lab = labels.cpu().numpy()
    nbn = None if nb is None else nb.cpu().numpy()
    lo, lr, g = PO.forward_backward(params, x, lab, image_size=S, neighbours=nbn, smoothing=smoothing,
                                    emulate_bf16=True)
    assert _rel(logits, lo) <= EMU_LOGIT_TOL
    assert _rel(loss, lr) <= EMU_LOGIT_TOL
    for k, (got, ref) in enumerate(zip(_grad_tensors(net, grads), _grad_tensors(net, g))):
        assert _rel(got, ref) <= EMU_GRAD_TOL, (k, _rel(got, ref))
    lo64, lr64, g64 = PO.forward_backward(params, x, lab, image_size=S, neighbours=nbn, smoothing=smoothing,
                                          emulate_bf16=False)
    assert _rel(logits, lo64) <= 1.5 * _rel(lo, lo64) + 0.02
    for k, (got, emu, ref) in enumerate(zip(_grad_tensors(net, grads), _grad_tensors(net, g),
                                            _grad_tensors(net, g64))):
        assert _rel(got, ref) <= 1.5 * _rel(emu, ref) + 0.02, (k, _rel(got, ref), _rel(emu, ref))


def test_full_size_forward_backward_runs_and_matches(cuda_device):
    """128^2 inputs (the benchmark's network), batch 8, emulated-BF16 oracle."""
    from cryojax_b200 import _native as nat

    net, labels = _net_and_batch(128, 8, seed=3)
    logits = net.forward(B=8).cpu().numpy().copy()
    net.backward(labels, B=8)
    assert nat.device_status() == 0
    lo, lr, g = PO.forward_backward(net.params.cpu().numpy(), net.x0[:8].float().cpu().numpy(),
                                    labels.cpu().numpy(), image_size=128, emulate_bf16=True)
    assert _rel(logits, lo) <= EMU_LOGIT_TOL
    for k, (got, ref) in enumerate(zip(_grad_tensors(net, net.grads.cpu().numpy()), _grad_tensors(net, g))):
        assert _rel(got, ref) <= EMU_GRAD_TOL, (k, _rel(got, ref))


def test_adamw_step_and_bf16_copies(cuda_device):
    import torch

    net, labels = _net_and_batch(64, 8, seed=5)
    net.forward(B=8)
    net.backward(labels, B=8)
    p0 = net.params.cpu().numpy().astype(np.float64)
    g0 = net.grads.cpu().numpy().astype(np.float64)
    decay = np.zeros_like(p0)
    for L in net.layers:
        decay[L["w_off"]:L["w_off"] + L["K"] * L["cout"]] = 1.0
    for step in (1, 2):
        m0, v0 = net.m.cpu().numpy().astype(np.float64), net.v.cpu().numpy().astype(np.float64)
        net.adam_step(1e-3, weight_decay=0.05)
        p_ref, m_ref, v_ref = PO.adamw_reference(p0, g0, m0, v0, step, 1e-3, weight_decay=0.05, decay_mask=decay)
        np.testing.assert_allclose(net.params.cpu().numpy(), p_ref, rtol=1e-5, atol=1e-7)
        np.testing.assert_allclose(net.m.cpu().numpy(), m_ref, rtol=1e-5, atol=1e-10)
        p0 = net.params.cpu().numpy().astype(np.float64)
    for i, L in enumerate(net.layers):
        w = net.weight(i).to(torch.bfloat16)
        assert torch.equal(L["Wt"], w)
        assert torch.equal(L["W"][:, :L["K"]], w.T)
        assert torch.count_nonzero(L["W"][:, L["K"]:]) == 0


def test_topk_candidates(cuda_device):
    import torch

    from cryojax_b200 import _native as nat

    g = torch.Generator(device="cuda")
    g.manual_seed(0)
    logits = torch.randn((37, 768), generator=g, device="cuda")
    logits[3, 10] = logits[3, 20] = 50.0  # a tie: the lower index first
    dirs = torch.empty((37, 16), dtype=torch.int32, device="cuda")
    cand = torch.empty((37, 16 * 48), dtype=torch.int32, device="cuda")
    nat.topk_candidates(logits, 16, 48, dirs=dirs, candidates=cand)
    ref = np.argsort(-logits.cpu().numpy(), axis=1, kind="stable")[:, :16]
    np.testing.assert_array_equal(dirs.cpu().numpy(), ref)
    c = cand.cpu().numpy().reshape(37, 16, 48)
    np.testing.assert_array_equal(c, ref[:, :, None] * 48 + np.arange(48))


def test_noisy_normalize(cuda_device):
    import torch

    from cryojax_b200 import _native as nat

    g = torch.Generator(device="cuda")
    g.manual_seed(1)
    imgs = torch.randn((6, 128, 128), generator=g, device="cuda") * 3.0 + 7.0
    out = torch.empty((6, 128, 128), dtype=torch.bfloat16, device="cuda")
    nat.cnn_noisy_normalize(imgs, out)
    x = imgs.double().cpu().numpy()
    ref = (x - x.mean(axis=(1, 2), keepdims=True)) / x.std(axis=(1, 2), keepdims=True)
    np.testing.assert_allclose(out.double().cpu().numpy(), ref, atol=2e-2, rtol=1e-2)
    # with noise at SNR s: deterministic in the seed, zero mean, unit std, correlation sqrt(s / (1 + s))
    idx = torch.tensor([2, 0, 5, 5], dtype=torch.int64, device="cuda")
    o1 = torch.empty((4, 128, 128), dtype=torch.bfloat16, device="cuda")
    o2 = torch.empty_like(o1)
    nat.cnn_noisy_normalize(imgs, o1, index=idx, snr=0.25, seed=11, n=4)
    nat.cnn_noisy_normalize(imgs, o2, index=idx, snr=0.25, seed=11, n=4)
    assert torch.equal(o1, o2)
    a = o1.double().cpu().numpy()
    assert np.all(np.abs(a.mean(axis=(1, 2))) < 1e-2) and np.all(np.abs(a.std(axis=(1, 2)) - 1) < 2e-2)
    r = [np.corrcoef(a[k].ravel(), ref[s].ravel())[0, 1] for k, s in enumerate([2, 0, 5, 5])]
    np.testing.assert_allclose(r, np.sqrt(0.25 / 1.25), atol=0.03)
    nat.cnn_noisy_normalize(imgs, o2, index=idx, snr=0.25, seed=12, n=4)
    assert not torch.equal(o1, o2)


def test_direct_first_layer_matches_im2col_gemm(cuda_device):
    """The inference path's first layer without im2col (cjx_cnn_conv0) gives the im2col + tensor-core GEMM
    layer's BF16 activations (equal on >= 99.9 %, else one BF16 step apart where the FP32 sums of the 9 taps
    round differently), and the proposals of a forward pass built on either agree."""
    import torch

    from cryojax_b200.pose_net import PoseProposalNet

    net = PoseProposalNet(128, 768, max_batch=64, seed=3)
    g = torch.Generator(device="cuda").manual_seed(4)
    x = torch.randn((64, 128, 128), generator=g, device="cuda").to(torch.bfloat16)
    a = net.forward(x, B=64).clone()
    act_gemm = net.acts[1].clone()
    b = net.forward(x, B=64, direct_first_layer=True).clone()
    act_direct = net.acts[1].clone()
    ra, rd = act_gemm.float(), act_direct.float()
    # one BF16 step of the larger value, or (near zero, where the ReLU cuts a sum that cancels) a tiny
    # fraction of the layer's scale
    tol = torch.maximum(ra.abs(), rd.abs()) * 2.0 ** -7 + 1e-4 * ra.abs().max()
    assert ((ra - rd).abs() <= tol).all(), (ra - rd).abs().max()
    assert (ra == rd).float().mean().item() >= 0.999
    torch.testing.assert_close(b, a, rtol=2e-2, atol=2e-2 * a.abs().max().item())
    top_a = torch.topk(a, 16, dim=1).indices.sort(dim=1).values
    top_b = torch.topk(b, 16, dim=1).indices.sort(dim=1).values
    assert (top_a == top_b).all(dim=1).float().mean().item() >= 0.9


def test_implicit_convolutions_match_im2col_gemm(cuda_device):
    """The inference path's later layers without im2col (cjx_cnn_conv_s2, implicit GEMM on the tensor cores)
    give each layer's im2col + GEMM BF16 activations from the same input (equal on >= 99 %, else within one
    BF16 step or a tiny fraction of the layer's scale), and the network's logits agree."""
    import torch

    from cryojax_b200 import _native as nat
    from cryojax_b200.pose_net import PoseProposalNet

    net = PoseProposalNet(128, 768, max_batch=64, seed=5)
    g = torch.Generator(device="cuda").manual_seed(6)
    x = torch.randn((64, 128, 128), generator=g, device="cuda").to(torch.bfloat16)
    a = net.forward(x, B=64).clone()
    ref = [t.clone() for t in net.acts]
    for i, L in enumerate(net.layers[1:6], start=1):
        out = torch.empty_like(ref[i + 1])
        nat.cnn_conv_s2(ref[i], 64, L["h"], L["w"], L["cin"], L["W"], L["ldk"], L["cout"], net.bias(i), out)
        ra, rd = ref[i + 1].float(), out.float()
        tol = torch.maximum(ra.abs(), rd.abs()) * 2.0 ** -7 + 1e-4 * ra.abs().max()
        assert ((ra - rd).abs() <= tol).all(), (i, (ra - rd).abs().max())
        assert (ra == rd).float().mean().item() >= 0.99, i
    b = net.forward(x, B=64, direct_first_layer=True, implicit_convs=True).clone()
    torch.testing.assert_close(b, a, rtol=2e-2, atol=2e-2 * a.abs().max().item())
