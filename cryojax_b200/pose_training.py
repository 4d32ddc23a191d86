"""Training the pose-proposal network on images the simulator generates.

Data: N poses uniform on SO(3) (no in-plane offsets), per-image defocus
uniform in a range, simulated by the batched Fourier-slice + CTF kernels and
brought to real space; the label is the HEALPix direction nearest to the
pose's viewing direction R[:, 2] (the orientation grid's direction index).
Every epoch draws fresh white noise at the target SNR inside the input
kernel (cjx_cnn_noisy_normalize), so the clean set is stored once on the
device.  The loss is softmax cross entropy with label smoothing spread over
each direction's nearest HEALPix neighbours.
"""

from __future__ import annotations

import math
import time

import numpy as np

from . import _native as nat
from . import rotations as rot
from . import simulator as S
from .healpix import OrientationGrid, pixel_directions


def _torch():
    import torch

    return torch


def direction_neighbours(nside: int, k: int = 8) -> np.ndarray:
    """(n_dir, k) int32: the k HEALPix pixels nearest to each pixel centre (itself excluded)."""
    d = pixel_directions(nside)
    cos = d @ d.T
    np.fill_diagonal(cos, -2.0)
    return np.argsort(-cos, axis=1, kind="stable")[:, :k].astype(np.int32)


def simulate_clean_images(volume, image_config, wxyz, defocus, *, chunk=8192, amplitude_contrast=0.1, out_size=None):
    """Real-space float32 CUDA images (n, P, P) at the given poses and defoci (no offsets, no noise).

    With ``out_size`` each image is area-downsampled to out_size x out_size
    on the device (cjx_area_downsample) as it is made, so only the small
    images are kept.
    """
    torch = _torch()
    n = len(wxyz)
    py, px = image_config.padded_shape
    oy, ox = (py, px) if out_size is None else (out_size, out_size)
    out = torch.empty((n, oy, ox), dtype=torch.float32, device=volume.device)
    from . import _postprocess

    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        m = e - s
        ctf = S.AstigmaticCTF(defocus_in_angstroms=np.asarray(defocus[s:e], np.float64),
                              astigmatism_in_angstroms=np.zeros(m), astigmatism_angle=np.zeros(m))
        tt = S.ContrastTransferTheory(ctf, amplitude_contrast_ratio=amplitude_contrast)
        pose = S.QuaternionPose(np.zeros(m), np.zeros(m), wxyz=np.asarray(wxyz[s:e], np.float64))
        model = S.make_image_model(volume, image_config, pose, tt)
        f = model.compute_fourier_image()
        img = _postprocess.irfftn(f, (py, px)).float().contiguous()
        if out_size is None:
            out[s:e] = img
        else:
            nat.area_downsample(img, out[s:e])
    return out


class TrainingSet:
    def __init__(self, volume, image_config, n, *, seed=0, defocus_range=(8000.0, 20000.0), nside=8, out_size=None):
        rng = np.random.default_rng(seed)
        self.wxyz = rot.sample_uniform_quaternions(rng, n)
        self.defocus = rng.uniform(*defocus_range, n)
        self.grid = OrientationGrid(nside, 1)
        R = rot.quat_to_matrix(self.wxyz)
        self.labels_np = self.grid.direction_of(R).astype(np.int32)
        torch = _torch()
        dev = volume.device
        self.labels = torch.as_tensor(self.labels_np, device=dev)
        self.images = simulate_clean_images(volume, image_config, self.wxyz, self.defocus, out_size=out_size)
        self.n = n


def snr_at(progress, snr, snr_start=None, ramp=0.5):
    """Curriculum: SNR falls geometrically from snr_start to snr over the first `ramp` of training."""
    if snr_start is None or progress >= ramp:
        return snr
    return float(snr_start * (snr / snr_start) ** (progress / ramp))


def train_pose_net(net, data: TrainingSet, *, epochs=8, batch=256, lr=2e-3, min_lr_frac=0.02, warmup=200,
                   weight_decay=0.01, snr=0.05, snr_start=None, snr_ramp=0.5, smoothing=0.2, n_neighbours=8, seed=0,
                   log=None):
    """AdamW with linear warm-up and cosine decay; fresh noise every step.  Returns a history dict."""
    torch = _torch()
    if batch > net.max_batch or batch % 8:
        raise ValueError("batch must be a multiple of 8 and <= net.max_batch")
    dev = net.device
    nb = torch.as_tensor(direction_neighbours(data.grid.nside, n_neighbours), device=dev) if n_neighbours else None
    steps_per_epoch = data.n // batch
    total = epochs * steps_per_epoch
    rng = np.random.default_rng(seed)
    hist = {"loss": [], "step": [], "seconds": 0.0, "steps": total}
    t0 = time.perf_counter()
    step = 0
    labels_b = torch.empty(batch, dtype=torch.int32, device=dev)
    for ep in range(epochs):
        perm = torch.as_tensor(rng.permutation(data.n)[:steps_per_epoch * batch].astype(np.int64), device=dev)
        ep_loss = torch.zeros((), dtype=torch.float32, device=dev)
        for it in range(steps_per_epoch):
            idx = perm[it * batch:(it + 1) * batch]
            cur_snr = snr_at(step / total, snr, snr_start, snr_ramp)
            nat.cnn_noisy_normalize(data.images, net.x0, index=idx, snr=cur_snr, seed=seed * 1000003 + step, n=batch)
            torch.index_select(data.labels, 0, idx, out=labels_b)
            net.forward(B=batch)
            loss = net.backward(labels_b, B=batch, neighbours=nb, smoothing=smoothing)
            ep_loss += loss.sum()
            if step < warmup:
                cur = lr * (step + 1) / warmup
            else:
                t = (step - warmup) / max(1, total - warmup)
                cur = lr * (min_lr_frac + (1 - min_lr_frac) * 0.5 * (1 + math.cos(math.pi * t)))
            net.adam_step(cur, weight_decay=weight_decay)
            step += 1
        mean_loss = float(ep_loss) / (steps_per_epoch * batch)
        hist["loss"].append(mean_loss)
        hist["step"].append(step)
        if log:
            log(f"epoch {ep + 1}/{epochs} loss {mean_loss:.4f} snr {cur_snr:.3g} ({time.perf_counter() - t0:.1f} s)")
    torch.cuda.synchronize()
    hist["seconds"] = time.perf_counter() - t0
    return hist


def top_k_hit_rate(net, images, true_dirs, k=16, *, batch=None):
    """Fraction of images whose true direction is among the network's top-k."""
    dirs, _ = net.propose(images, k=k, n_inplane=1, batch=batch)
    d = dirs.cpu().numpy()
    return float(np.mean(np.any(d == np.asarray(true_dirs)[:, None], axis=1)))
