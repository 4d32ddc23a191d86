#!/usr/bin/env python
"""Benchmark: batched Fourier-slice + CTF image simulation on B200.

Workload (default): a 256^3 Gaussian-sum volume (6000 Gaussians, sigma 1-3
voxels, seeded) prepared as a FourierVoxelGridVolume with pad factor 2
(N = 512, complex64, 1.07 GB), and 16384 images of 320 x 320 at 2 A / 300 kV,
each with its own uniform SO(3) pose, +-20 A offsets and AstigmaticCTF
(defocus U(5000, 25000) A, astigmatism U(0, 500) A, angle U(0, 180) deg).
One step = simulate the whole batch (rfft half-plane output, complex64
[16384, 320, 161]) through one cjx_slice_ctf_forward call.  Inputs (volume,
per-image parameters) are resident in HBM; the volume (1.07 GB) and the
output (6.75 GB) both exceed L2, so no flush is needed between steps.

Under torchrun each rank simulates its own 16384 images from its own
replica of the volume (images shard with no collective: weak scaling).

``--impl reference`` times the reference path's CPU restatement (the
float64 NumPy oracle; JAX is not installed, so the reference itself cannot
run) on all host cores, on a bounded sample of the same workload.
"""

from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "slice+CTF images/s at 320^2 (256^3 volume, pad 2)"
UNIT = "images/s"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--images", type=int, default=16384)
    ap.add_argument("--box", type=int, default=256)
    ap.add_argument("--gaussians", type=int, default=6000)
    ap.add_argument("--image", type=int, default=320)
    ap.add_argument("--pad-scale", type=float, default=2.0)
    ap.add_argument("--chunk", type=int, default=0, help="images per workspace chunk (0 = library default)")
    ap.add_argument("--ilp", type=int, default=0, help="gather ILP (1, 2, 4; 0 = library default)")
    ap.add_argument("--gather-mode", type=int, default=-1, help="CJX_TUNE_GATHER_MODE (-1 = library default)")
    ap.add_argument("--scatter-mode", type=int, default=-1, help="CJX_TUNE_SCATTER_VEC (-1 = library default)")
    ap.add_argument("--layout", choices=["pairs", "bricked", "linear"], default="pairs",
                    help="device layout of the volume the gather reads")
    ap.add_argument("--order", choices=["orientation", "none"], default="orientation",
                    help="image processing order (orientation-sorted for L2 reuse, or as given)")
    ap.add_argument("--cpu-sample", type=int, default=6, help="images in the bounded CPU sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--no-batched", action="store_true", help="skip the mixed-size batch measurement")
    ap.add_argument("--no-grad", action="store_true", help="skip the loss-gradient measurement")
    ap.add_argument("--no-search", action="store_true", help="skip the pose-search (learned vs grid) measurement")
    ap.add_argument("--probe", choices=["gemm", "search", "cnn", "spline", "ewald", "render", "ncc"], default=None,
                    help="run one small workload of that kernel family (for a profiler), print its timing, exit")
    ap.add_argument("--no-refine", action="store_true",
                    help="skip the search + refinement measurement (320^2 images, N=512)")
    ap.add_argument("--refine-images", type=int, default=512, help="images in the learned arm of that measurement")
    ap.add_argument("--refine-exhaustive-images", type=int, default=512,
                    help="images in its exhaustive arm (36,864 simulations each)")
    ap.add_argument("--no-spline", action="store_true", help="skip the spline-volume measurement")
    ap.add_argument("--no-ewald", action="store_true", help="skip the Ewald-sphere measurement")
    ap.add_argument("--no-relion", action="store_true", help="skip the RELION particle-stack measurement")
    ap.add_argument("--no-render", action="store_true", help="skip the Gaussian-mixture rendering measurement")
    ap.add_argument("--search-images", type=int, default=4096,
                    help="observed images in the pose-search measurement (the configuration's 4096)")
    return ap.parse_args()


def config_dict(args, world):
    n = int(args.box * args.pad_scale)
    return {
        "workload": f"{args.images} images {args.image}x{args.image} from a {args.box}^3 volume "
                    f"(N={n} padded grid), per-image pose+CTF, rfft output",
        "volume_box": args.box, "padded_volume_side": n, "gaussians": args.gaussians,
        "image_shape": [args.image, args.image], "images_per_gpu": args.images,
        "global_batch": args.images * world, "pixel_size_A": 2.0, "voltage_kV": 300.0,
        "l2_flush": "not needed: volume (1.07 GB) and output (6.75 GB per step) exceed the 126 MB L2",
        "parallelism": f"replicas x{world} (images sharded, no collective)",
        "processing_order": args.order,
        "volume_layout": {"pairs": "x-pair bricked (16-byte entries g(x), g(x+1))",
                          "bricked": "bricked (8^3 blocks, Morton order inside)",
                          "linear": "C-order [z][y][x]"}[args.layout],
    }


# ---------------------------------------------------------------------------
# clocks sampling
# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi samples of SM clock, power and throttle reasons during the timed region.

    Every sample carries nvidia-smi's own timestamp, and only samples taken at or after ``mark()``
    count, so samples that nvidia-smi took before the region but flushed to its output file later
    (block-buffered output) are never attributed to the region.  nvidia-smi runs line-buffered
    through ``stdbuf -oL`` where that exists, so ``start()`` sees the first sample promptly."""

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu_index = gpu_index
        self.proc = None
        self.path = None
        self.mark_time = None

    def _lines(self):
        try:
            with open(self.path) as f:
                return sum(1 for _ in f)
        except Exception:
            return 0

    @staticmethod
    def _epoch(stamp):
        """nvidia-smi's timestamp (local time, "YYYY/MM/DD HH:MM:SS.mmm") as seconds since the epoch."""
        import datetime

        return datetime.datetime.strptime(stamp.strip(), "%Y/%m/%d %H:%M:%S.%f").timestamp()

    def start(self):
        """Start nvidia-smi and wait (at most 5 s) for its first sample, so that a short timed region
        that begins after this call is sampled from its start."""
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                   "-i", str(self.gpu_index)]
            if shutil.which("stdbuf"):
                cmd = ["stdbuf", "-oL"] + cmd
            self.proc = subprocess.Popen(cmd, stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            t0 = time.time()
            while time.time() - t0 < 5.0 and self._lines() == 0 and self.proc.poll() is None:
                time.sleep(0.02)
        except Exception:
            self.proc = None

    def mark(self):
        """Call when the timed region starts: samples taken before this moment are not part of it."""
        self.mark_time = time.time()

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 10:
                continue
            try:
                rows.append((self._epoch(parts[0]), float(parts[2]), float(parts[3]), parts[6:10]))
            except ValueError:
                continue
        os.unlink(self.path)
        mark = self.mark_time if self.mark_time is not None else float("-inf")
        region = [r for r in rows if r[0] >= mark]
        note = None
        if not region and rows:  # region shorter than one sampling period: the last sample before it
            region, note = rows[-1:], "no sample fell inside the timed region; last sample before it"
        if not region:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, _, r in region for i, v in enumerate(r) if v.lower() == "active"})
        out = {"sm_mhz": statistics.median(r[1] for r in region), "sm_min_mhz": min(r[1] for r in region),
               "sm_max_mhz": max(r[2] for r in region), "reasons": reasons, "samples": len(region)}
        if note:
            out["note"] = note
        return out


# ---------------------------------------------------------------------------
# reference arm / CPU baseline: the float64 oracle on host cores
# ---------------------------------------------------------------------------
def _cpu_worker(args_tuple):
    path, specs = args_tuple
    import numpy as np

    from oracle import cryojax_oracle as O

    grid = np.load(path, mmap_mode="r")
    fs = O.make_frequency_slice((grid.shape[0], grid.shape[0]), outputs_rfftfreqs=False)
    t0 = time.perf_counter()
    for s in specs:
        O.compute_fourier_image(grid, fs, s)
    return len(specs), time.perf_counter() - t0


def cpu_oracle_throughput(grid_c128, batch, n_images, image, pixel_size, voltage, workers):
    """images/s of the float64 oracle over `n_images` images.

    workers == 1: in this process.  workers > 1: a spawn pool whose workers
    map the grid read-only from a temporary .npy file (shared page cache).
    Throughput = images / the slowest worker's busy time.
    """
    from oracle import cryojax_oracle as O

    specs = []
    for b in range(n_images):
        specs.append(O.ImageSpec(shape=(image, image), pixel_size=pixel_size, voltage_in_kilovolts=voltage,
                                 wxyz=batch.wxyz[b], offset_in_angstroms=batch.offsets[b],
                                 defocus_in_angstroms=batch.defocus[b], astigmatism_in_angstroms=batch.astigmatism[b],
                                 astigmatism_angle=batch.astigmatism_angle[b]))
    t0 = time.perf_counter()
    if workers == 1:
        fs = O.make_frequency_slice((grid_c128.shape[0], grid_c128.shape[0]), outputs_rfftfreqs=False)
        t1 = time.perf_counter()
        for s in specs:
            O.compute_fourier_image(grid_c128, fs, s)
        busy = time.perf_counter() - t1
        return len(specs) / busy, len(specs), time.perf_counter() - t0
    import multiprocessing as mp

    import numpy as np

    fd, path = tempfile.mkstemp(suffix=".npy")
    os.close(fd)
    try:
        np.save(path, grid_c128)
        per = [p for p in (specs[i::workers] for i in range(workers)) if p]
        with mp.get_context("spawn").Pool(len(per)) as pool:
            res = pool.map(_cpu_worker, [(path, p) for p in per])
    finally:
        os.unlink(path)
    done = sum(r[0] for r in res)
    busy = max(r[1] for r in res)
    return done / busy, done, time.perf_counter() - t0


PARITY_IMAGES = 8  # timed images per leg checked against the float64 oracle after all timed regions
PARITY_TOL = 1e-5  # relative L2 per image, the tolerance of the parity tests


def oracle_specs(batch, idx, shape, pixel_size=2.0, voltage=300.0):
    """Oracle parameter records of images `idx` of a synthetic batch (the same pose / CTF the device saw)."""
    from oracle import cryojax_oracle as O

    return [O.ImageSpec(shape=shape, pixel_size=pixel_size, voltage_in_kilovolts=voltage, wxyz=batch.wxyz[b],
                        offset_in_angstroms=batch.offsets[b], defocus_in_angstroms=batch.defocus[b],
                        astigmatism_in_angstroms=batch.astigmatism[b], astigmatism_angle=batch.astigmatism_angle[b])
            for b in idx]


def oracle_parity(grid, got, specs, n=None, grid_source="float64 FFT of the same real volume", **kw):
    """Per-image relative L2 of the device's images `got` (host complex64) against the float64 oracle
    (cryojax_oracle.compute_fourier_image with keyword options `kw`) fed `grid`."""
    from oracle import cryojax_oracle as O

    n = grid.shape[0] if n is None else n
    fs = O.make_frequency_slice((n, n), outputs_rfftfreqs=False)
    t0 = time.perf_counter()
    errs = [float(O.relative_l2(g, O.compute_fourier_image(grid, fs, s, **kw))) for g, s in zip(got, specs)]
    return {"max_rel_l2": max(errs), "median_rel_l2": statistics.median(errs), "images": len(errs),
            "tolerance": PARITY_TOL, "pass": max(errs) <= PARITY_TOL, "oracle_grid": grid_source,
            "oracle_seconds": time.perf_counter() - t0}


def run_reference(args):
    """Reference arm: the oracle port on all host cores, same config/metric."""
    import numpy as np

    from cryojax_b200 import synthetic

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    vol = synthetic.gaussian_sum_volume(args.box, args.gaussians, args.seed, sigma_range=(1.0, 3.0))
    n = int(args.box * args.pad_scale)
    from oracle import cryojax_oracle as O

    grid, _ = O.fourier_voxel_grid_from_real_voxel_grid(vol, pad_scale=args.pad_scale)
    batch = synthetic.image_batch(args.images, args.seed + 1)
    workers = max(1, len(os.sched_getaffinity(0)))
    sample = max(workers, args.cpu_sample)
    vals = []
    t_all = time.perf_counter()
    for _ in range(max(1, args.steps)):
        v, done, _ = cpu_oracle_throughput(grid, batch, sample, args.image, 2.0, 300.0, workers)
        vals.append(v)
    wall = time.perf_counter() - t_all
    value = statistics.median(vals)
    cfg = config_dict(args, 1)
    for key in ("volume_layout", "processing_order", "l2_flush"):  # device-side choices; the port has none
        cfg.pop(key, None)
    cfg["images_per_step"] = sample
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "images_per_step": sample,
        # one step is the bounded sample of `sample` images of the workload, not all args.images of it
        "ms_per_step": 1000.0 * sample / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": cfg,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": workers, "kind": "port",
                         "sample": f"{sample} images per step of the same workload (N={n}, {args.image}^2), float64 NumPy "
                                   f"oracle of the reference path, {workers} spawn workers; JAX is not installed so "
                                   f"the reference itself cannot run"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": wall,
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def algorithmic_bytes_per_image(kernel, n, py, px, gather_voxels=None):
    """Bytes one image moves through a kernel at the algorithmic level.

    k_gather_colifft_fused: 8 B per distinct voxel the slice touches (read
      once; `gather_voxels` per image, counted on the host) plus the
      Py x (N/2+1) complex window written to T1 (the sampled plane itself
      never leaves the SM); without `gather_voxels`, the 8 corner loads per
      sample at the L2 level.
    k_gather_colifft: 8 corner loads of 8 B per slice sample over the
      N x (N/2+1) half-plane, plus the Py x (N/2+1) complex window written.
    k_gather_slice:  8 B per distinct voxel the slice touches (read once) plus
      one 8 B store per slice sample (`gather_voxels` = distinct voxels per
      image, counted on the host); the L2-level figure (8 corner loads + one
      store = 72 B per sample) is reported separately against the L2 probe.
    k_colifft_window: read the N x (N/2+1) slice, write the Py x (N/2+1) window.
    k_rows_c2r_r2c:  read Py x (N/2+1), write Py x (Px/2+1) complex.
    k_colfft_epilogue: read Py x (Px/2+1), write Py x (Px/2+1) complex.
    k_slice_direct:  8 corner loads + one store per output pixel.
    """
    nxh, pxh = n // 2 + 1, px // 2 + 1
    if kernel == "k_gather_colifft_fused":
        if gather_voxels is not None:
            return 8 * gather_voxels + 8 * py * nxh
        return 64 * n * nxh + 8 * py * nxh
    if kernel == "k_gather_colifft":
        return 64 * n * nxh + 8 * py * nxh
    if kernel == "k_gather_slice":
        if gather_voxels is not None:
            return 8 * gather_voxels + 8 * n * nxh
        return 72 * n * nxh
    if kernel == "k_colifft_window":
        return 8 * n * nxh + 8 * py * nxh
    if kernel == "k_rows_c2r_r2c":
        return 8 * py * nxh + 8 * py * pxh
    if kernel == "k_colfft_epilogue":
        return 16 * py * pxh
    if kernel == "k_slice_direct":
        return 72 * n * nxh
    return None


def unique_voxels_per_image(n, rotations, max_images=4):
    """Mean number of distinct grid voxels the half-plane slice of an image
    interpolates from (its 8 trilinear corners per sample, the reference's
    out-of-bounds rule), over the first `max_images` rotations."""
    import numpy as np

    h = n // 2
    nxh = n // 2 + 1
    u = np.arange(nxh)
    u = np.where(u < n - h, u, u - n).astype(np.float64)
    v = np.arange(n)
    v = np.where(v < n - h, v, v - n).astype(np.float64)
    U, V = np.meshgrid(u, v)
    counts = []
    for R in rotations[:max_images]:
        pts = np.stack([U.ravel(), V.ravel()], 1) @ R[:, :2].T  # (x, y, z) offsets
        lo = np.floor(pts).astype(np.int64) + h
        keys = []
        for dz in (0, 1):
            for dy in (0, 1):
                for dx in (0, 1):
                    iz, iy, ix = lo[:, 2] + dz, lo[:, 1] + dy, lo[:, 0] + dx
                    iz = np.where(iz < 0, iz + n, iz)
                    iy = np.where(iy < 0, iy + n, iy)
                    ix = np.where(ix < 0, ix + n, ix)
                    ok = (iz >= 0) & (iz < n) & (iy >= 0) & (iy < n) & (ix >= 0) & (ix < n)
                    keys.append(((iz * n + iy) * n + ix)[ok])
        counts.append(np.unique(np.concatenate(keys)).size)
    return float(np.mean(counts))


def measure_batched_uneven(dev, steps, warmup, seed):
    """Mixed volumes and image sizes in one CUDA-graph launch.

    Four Gaussian-sum volumes of 96^3, 128^3, 192^3 and 256^3 voxels
    (150 / 400 / 1500 / 5000 Gaussians, sigma 1-3 voxels, pad 2), 4096 images
    each at their box size with their own pose, +-20 A offsets and CTF
    (defocus U(5000, 25000), astigmatism U(0, 500), angle U(0, 180)).
    All 16384 images run through one cjx_slice_ctf_forward_multi call with
    autotuned per-group kernel choices, captured in one CUDA graph.
    """
    import torch

    from cryojax_b200 import simulator as S
    from cryojax_b200 import synthetic
    from cryojax_b200.batched import BatchedSimulator

    specs = [(96, 150), (128, 400), (192, 1500), (256, 5000)]
    models = []
    for i, (box, ng) in enumerate(specs):
        vol_np = synthetic.gaussian_sum_volume(box, ng, seed + 10 + i, sigma_range=(1.0, 3.0))
        vol = S.FourierVoxelGridVolume.from_real_voxel_grid(vol_np, pad_scale=2.0, device=str(dev))
        b = synthetic.image_batch(4096, seed + 20 + i)
        pose = S.QuaternionPose(b.offsets[:, 0], b.offsets[:, 1], wxyz=b.wxyz)
        tt = S.ContrastTransferTheory(S.AstigmaticCTF(b.defocus, b.astigmatism, b.astigmatism_angle))
        cfg = S.BasicImageConfig((box, box), 2.0, 300.0)
        models.append(S.make_image_model(vol, cfg, pose, tt))
    sim = BatchedSimulator(models, tuning="auto", autotune_kw=dict(n_sample=512, repeats=2))
    sim.capture()
    for _ in range(warmup):
        sim.replay()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        sim.replay()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    tun = []
    for m in models:
        from cryojax_b200.batched import autotune

        tun.append(autotune(m))
    # the timed replay's own first images of each group, for the oracle check after all timed regions
    parity = [{"box": box, "gaussians": ng, "volume_seed": seed + 10 + i, "batch_seed": seed + 20 + i,
               "got": sim.outputs[i][:PARITY_IMAGES].cpu().numpy()} for i, (box, ng) in enumerate(specs)]
    return {"_parity": parity,
            "metric": "mixed-size slice+CTF images/s (96^3..256^3 volumes, images at box size)",
            "value": sim.n_images / (ms / 1000.0), "unit": "images/s", "ms_per_step": ms,
            "images_per_step": sim.n_images, "groups": [f"N={2 * b} -> {b}x{b} x 4096" for b, _ in specs],
            "launch": "one CUDA graph replay per step (cjx_slice_ctf_forward_multi captured once)",
            "autotuned": tun}


def measure_gradient(dev, steps, warmup, seed):
    """Squared residual + gradients w.r.t. pose, offsets, defocus and the grid.

    A 192^3 Gaussian-sum volume (2000 Gaussians, pad 2 -> N = 384) and 1024
    observed 192 x 192 images simulated at seeded true poses plus white noise
    at SNR 0.1 (the noise model's recipe); loss and gradients evaluated at
    poses perturbed by <= 3 deg, +-2 A offsets and +-300 A defocus.  One step =
    one cjx_slice_ctf_loss_grad call over the 1024 images (forward, adjoint
    passes, grid scatter-add).
    """
    import numpy as np
    import torch

    from cryojax_b200 import _native as nat
    from cryojax_b200 import rotations as rot
    from cryojax_b200 import simulator as S
    from cryojax_b200 import synthetic
    from cryojax_b200.gradients import observed_to_fourier, squared_residual_and_grad
    from cryojax_b200.noise import GaussianWhiteNoiseModel, noise_variance_for_snr

    n_img = 1024
    vol_np = synthetic.gaussian_sum_volume(192, 2000, seed + 30, sigma_range=(1.0, 3.0))
    vol = S.FourierVoxelGridVolume.from_real_voxel_grid(vol_np, pad_scale=2.0, device=str(dev))
    rng = np.random.default_rng(seed + 31)
    b = synthetic.image_batch(n_img, seed + 32, max_offset=10.0, defocus_range=(8000.0, 20000.0))
    cfg = S.BasicImageConfig((192, 192), 2.0, 300.0)
    true_model = S.make_image_model(vol, cfg, S.QuaternionPose(b.offsets[:, 0], b.offsets[:, 1], wxyz=b.wxyz),
                                    S.ContrastTransferTheory(S.AstigmaticCTF(b.defocus, b.astigmatism,
                                                                             b.astigmatism_angle)))
    signal = true_model.simulate()
    var = noise_variance_for_snr(signal, 0.1)
    gen = torch.Generator(device=dev).manual_seed(seed + 33)
    obs = signal + GaussianWhiteNoiseModel(true_model, variance=var).compute_noise(gen)
    axis = rng.standard_normal((n_img, 3))
    axis /= np.linalg.norm(axis, axis=1, keepdims=True)
    dq = rot.so3_exp(np.deg2rad(rng.uniform(0, 3.0, n_img))[:, None] * axis)
    q = rot.quat_compose(dq, b.wxyz)
    off = b.offsets + rng.uniform(-2, 2, (n_img, 2))
    df = b.defocus + rng.uniform(-300, 300, n_img)
    model = S.make_image_model(vol, cfg, S.QuaternionPose(off[:, 0], off[:, 1], wxyz=q),
                               S.ContrastTransferTheory(S.AstigmaticCTF(df, b.astigmatism, b.astigmatism_angle)))
    obs_f = observed_to_fourier(obs)
    # full public call once (host chain to quaternion gradients included)
    res = squared_residual_and_grad(model, obs_f, observed_is_fourier=True, grid_grad=True)
    # device-timed loop of the library call
    integ = model.volume_integrator
    grid_b, layout = vol.bricked_grid(), nat.CJX_GRID_BRICKED  # the layout squared_residual_and_grad takes
    flags = model._flags() | layout
    desc = nat.make_desc(vol.shape[0], 192, 192, flags)
    pd = torch.as_tensor(model.image_params(), device=dev)
    order = torch.as_tensor(S.orientation_order(model.image_params()[:, 0:9].reshape(-1, 3, 3)), device=dev)
    grads = torch.empty((n_img, nat.GRAD_DOUBLES), dtype=torch.float64, device=dev)
    gg = torch.zeros(vol.shape, dtype=torch.complex64, device=dev)
    ws = torch.empty(nat.loss_workspace_size(desc, n_img), dtype=torch.uint8, device=dev)
    for _ in range(warmup):
        nat.slice_ctf_loss_grad(desc, grid_b, pd, obs_f, grads, gg, ws, order=order)
    torch.cuda.synchronize()
    nat.profile_enable(True)
    nat.slice_ctf_loss_grad(desc, grid_b, pd, obs_f, grads, gg, ws, order=order)
    torch.cuda.synchronize()
    prof = nat.profile_read()
    nat.profile_enable(False)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        nat.slice_ctf_loss_grad(desc, grid_b, pd, obs_f, grads, gg, ws, order=order)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    gnorm = float(gg.abs().pow(2).sum().sqrt())
    ewald = measure_gradient_ewald(vol, model, obs_f, grid_b, gg, steps, warmup)
    return {"metric": "loss + gradient images/s (192^3 volume, 192^2 images, pose/offset/defocus/grid)",
            "value": n_img / (ms / 1000.0), "unit": "images/s", "ms_per_step": ms, "images_per_step": n_img,
            "kernels_per_step": {k: {"launches": c, "ms": t} for k, (c, t) in prof.items()},
            "layout": "x-pair bricked grid" if layout == nat.CJX_GRID_BRICKED_PAIRS else "bricked grid",
            "scatter_mode": nat.tuning_get(nat.CJX_TUNE_SCATTER_VEC),
            "mean_loss": float(np.mean(res["loss"])), "grid_grad_norm": gnorm, "ewald_sphere": ewald}


def measure_gradient_ewald(vol, model, obs_f, grid_b, gg, steps, warmup):
    """The same loss + gradients through EwaldSphereExtraction (300 kV contrast), same volume, poses, CTFs
    and observed images; one step = one cjx_slice_ctf_loss_grad call over the 1024 images."""
    import torch

    from cryojax_b200 import _native as nat
    from cryojax_b200 import simulator as S

    try:
        n_img = obs_f.shape[0]
        integ = S.EwaldSphereExtraction()
        em = S.make_image_model(vol, model.image_config, model.pose, model.transfer_theory, volume_integrator=integ)
        params = em.image_params()
        desc = nat.make_desc(vol.shape[0], 192, 192, em._flags() | integ._base_flags() | nat.CJX_GRID_BRICKED)
        dev = obs_f.device
        pd = torch.as_tensor(params, device=dev)
        order = torch.as_tensor(S.orientation_order(params[:, 0:9].reshape(-1, 3, 3)), device=dev)
        grads = torch.empty((n_img, nat.GRAD_DOUBLES), dtype=torch.float64, device=dev)
        ws = torch.empty(nat.loss_workspace_size(desc, n_img), dtype=torch.uint8, device=dev)
        gg.zero_()
        for _ in range(warmup):
            nat.slice_ctf_loss_grad(desc, grid_b, pd, obs_f, grads, gg, ws, order=order)
        torch.cuda.synchronize()
        nat.profile_enable(True)
        nat.slice_ctf_loss_grad(desc, grid_b, pd, obs_f, grads, gg, ws, order=order)
        torch.cuda.synchronize()
        prof = nat.profile_read()
        nat.profile_enable(False)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            nat.slice_ctf_loss_grad(desc, grid_b, pd, obs_f, grads, gg, ws, order=order)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        return {"value": n_img / (ms / 1000.0), "unit": "images/s", "ms_per_step": ms,
                "kernels_per_step": {k: {"launches": c, "ms": t} for k, (c, t) in prof.items()},
                "mean_loss": float(grads[:, nat.G_LOSS].mean())}
    except Exception as exc:  # reported in the line; the slice figures above stand
        nat.profile_enable(False)
        return {"error": f"{type(exc).__name__}: {exc}"}


def measure_pose_search(dev, seed, n_obs):
    """Pose search on a 128^3 volume (800 Gaussians, pad 2 -> N = 256), 128^2 images at SNR 0.05.

    Observed images: true poses uniform on SO(3), defocus U(8000, 20000) A,
    white noise at SNR 0.05.  Grid: 768 HEALPix directions (nside 8) x 48
    in-plane angles = 36,864 orientations.  Plain: every orientation
    simulated with the image's own CTF and scored by NCC (the reference's
    grid search).  Learned: the pose-proposal network (trained here on 200k
    simulator images) proposes the top-16 directions, their 16 x 48
    orientations are rescored by the same scorer, and images whose best
    score falls below a threshold calibrated on 1024 separate images go to
    the exhaustive search.  Both are timed on the device end to end (network
    included; training reported separately).
    """
    import numpy as np
    import torch

    from cryojax_b200 import _native as nat
    from cryojax_b200 import pose_training as PT
    from cryojax_b200 import rotations as rot
    from cryojax_b200 import simulator as S
    from cryojax_b200 import synthetic
    from cryojax_b200.healpix import OrientationGrid
    from cryojax_b200.pose_net import PoseProposalNet
    from cryojax_b200.search import LearnedPoseSearch, PoseSearch, TemplateSharingSearch

    vol_np = synthetic.gaussian_sum_volume(128, 800, seed + 40, sigma_range=(1.0, 3.0))
    V = S.FourierVoxelGridVolume.from_real_voxel_grid(vol_np, pad_scale=2.0, device=str(dev))
    cfg = S.BasicImageConfig((128, 128), 2.0, 300.0)
    grid = OrientationGrid(8, 48)
    search = PoseSearch(grid.rotation_matrices())

    def batch(n, s, snr=0.05):
        rng = np.random.default_rng(s)
        q = rot.sample_uniform_quaternions(rng, n)
        df = rng.uniform(8000.0, 20000.0, n)
        clean = PT.simulate_clean_images(V, cfg, q, df)
        g = torch.Generator(device=dev).manual_seed(s)
        noisy = clean + torch.randn(clean.shape, generator=g, device=dev) * torch.sqrt(
            clean.var(dim=(1, 2), keepdim=True) / snr)
        ctf = S.AstigmaticCTF(defocus_in_angstroms=df, astigmatism_in_angstroms=np.zeros(n),
                              astigmatism_angle=np.zeros(n))
        model = S.make_image_model(V, cfg, S.QuaternionPose(np.zeros(n), np.zeros(n), wxyz=q),
                                   S.ContrastTransferTheory(ctf, amplitude_contrast_ratio=0.1))
        return model, noisy, q

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = fn()
        e1.record()
        torch.cuda.synchronize()
        return out, e0.elapsed_time(e1) / 1000.0

    data, t_data = timed(lambda: PT.TrainingSet(V, cfg, 200000, seed=seed + 41))
    net = PoseProposalNet(128, grid.n_dir, max_batch=256, seed=seed + 42)
    hist = PT.train_pose_net(net, data, epochs=12, lr=1e-3, snr=0.05, snr_start=2.0, snr_ramp=0.6, seed=seed + 43)
    n_train_steps = hist["steps"]
    del data
    torch.cuda.empty_cache()
    # fallback threshold: calibrated on 1024 separate images whose exhaustive optimum comes from the
    # template-sharing exhaustive search with FP32 re-ranking of its 8 best candidates per image
    cal_model, cal_obs, _ = batch(1024, seed + 44)
    cal_ex = TemplateSharingSearch(grid.rotation_matrices()).run(cal_model, cal_obs, rerank_top=8)
    learned = LearnedPoseSearch(net, grid, top_k=16, search=search)
    thr = learned.calibrate_threshold(cal_model, cal_obs, cal_ex.best_orientation, target_agreement=0.995)
    model, obs, q = batch(n_obs, seed + 45)
    df_obs = np.asarray(model.transfer_theory.ctf.defocus_in_angstroms)
    true_dir = grid.direction_of(rot.quat_to_matrix(q))

    def first(k):  # the image model of the first k observed images
        return S.make_image_model(V, cfg, S.QuaternionPose(np.zeros(k), np.zeros(k), wxyz=q[:k]),
                                  S.ContrastTransferTheory(S.AstigmaticCTF(
                                      defocus_in_angstroms=df_obs[:k], astigmatism_in_angstroms=np.zeros(k),
                                      astigmatism_angle=np.zeros(k)), amplitude_contrast_ratio=0.1))

    # the plain exhaustive arm (one simulation per image and orientation) runs on the first n_plain images and
    # the simulate-every-candidate learned arm on the first n_sim; every other arm on all n_obs images
    n_plain, n_sim = min(n_obs, 256), min(n_obs, 1024)
    plain_model, sim_model = first(n_plain), first(n_sim)
    learned.run(first(64), obs[:64], fallback=False)  # warm-up
    ex, t_ex = timed(lambda: search.run(plain_model, obs[:n_plain]))
    res, t_l = timed(lambda: learned.run(sim_model, obs[:n_sim]))
    nat.profile_enable(True)  # one extra, profiled run of the learned arm (not part of its value)
    learned.run(sim_model, obs[:n_sim])
    torch.cuda.synchronize()
    learned_kernels = {k: {"launches": c, "ms": t} for k, (c, t) in nat.profile_read().items()}
    nat.profile_enable(False)
    _, t_net = timed(lambda: net.propose(obs, k=16, n_inplane=grid.n_inplane))
    shared = TemplateSharingSearch(grid.rotation_matrices())
    shared.build_templates(model)  # warm-up: buffer allocation; the timed build below recomputes every template
    shared._key = None
    _, t_tmpl = timed(lambda: shared.build_templates(model))
    sh, t_sh = timed(lambda: shared.run(model, obs))
    shr, t_shr = timed(lambda: shared.run(model, obs, rerank_top=8))  # re-ranked from the FP32 template bank
    shared.rerank = "simulate"  # the same 8 candidates simulated again by the plain scorer (bit-exact scores)
    shs, t_shs = timed(lambda: shared.run(model, obs, rerank_top=8))
    shared.rerank = "bank"
    # learned proposals scored from the shared template rows, FP32 re-ranking of the 8 best, template-sharing
    # exhaustive fallback; threshold calibrated the same way on the same calibration images
    learned_t = LearnedPoseSearch(net, grid, top_k=16, search=search, templates=shared, rerank_top=8)
    thr_t = learned_t.calibrate_threshold(cal_model, cal_obs, cal_ex.best_orientation, target_agreement=0.995)
    del cal_obs
    learned_t.run(first(64), obs[:64])  # warm-up
    rt, t_lt = timed(lambda: learned_t.run(model, obs))
    nat.profile_enable(True)
    learned_t.run(model, obs)
    torch.cuda.synchronize()
    learned_t_kernels = {k: {"launches": c, "ms": t} for k, (c, t) in nat.profile_read().items()}
    nat.profile_enable(False)
    R_ex, R_true = grid.rotation_matrices(ex.best_orientation), rot.quat_to_matrix(q[:n_plain])
    ang = np.degrees(np.arccos(np.clip((np.einsum("nij,nij->n", R_ex, R_true) - 1) / 2, -1, 1)))
    return {
        "metric": "pose-search images/s, learned vs exhaustive (128^2 images, N=256, 36,864 orientations)",
        "unit": "images/s", "n_images": n_obs,
        "plain_exhaustive": {"value": n_plain / t_ex, "seconds": t_ex, "n_images": n_plain,
                             "candidates_per_image": grid.size, "candidates_per_s": n_plain * grid.size / t_ex},
        "learned": {"value": n_sim / t_l, "seconds": t_l, "n_images": n_sim,
                    "candidates_per_image": 16 * grid.n_inplane,
                    "scoring": "every candidate simulated with the image's CTF and scored in FP32",
                    "network_seconds_all_images": t_net, "fallback_fraction": float(res.fallback.mean()),
                    "threshold": thr, "kernels_per_run": learned_kernels},
        "learned_template_rows": {
            "value": n_obs / t_lt, "seconds": t_lt, "n_images": n_obs,
            "scoring": "candidates scored from the shared FP16 template rows (cjx_ncc_directions), the 8 best "
                       "re-ranked in FP32 from the FP32 template bank, template-sharing exhaustive fallback "
                       "(templates prebuilt, as for the template-sharing arm's search time)",
            "fallback_fraction": float(rt.fallback.mean()), "threshold": thr_t,
            # with the template bank's build counted, as the template-sharing arm's value counts it
            "value_with_template_bank": n_obs / (t_tmpl + t_lt),
            "agreement_with_plain_exhaustive": float(np.mean(rt.best_orientation[:n_plain] == ex.best_orientation)),
            "agreement_with_template_exhaustive_reranked": float(np.mean(rt.best_orientation == shr.best_orientation)),
            "speedup_vs_template_exhaustive_reranked_search": t_shr / t_lt,
            "speedup_vs_plain_exhaustive": (n_obs / t_lt) / (n_plain / t_ex),
            "kernels_per_run": learned_t_kernels},
        "template_sharing_exhaustive": {
            "value": n_obs / (t_tmpl + t_sh), "seconds": t_tmpl + t_sh, "template_seconds": t_tmpl,
            "gemm_search_seconds": t_sh,
            "agreement_with_plain_exhaustive": float(np.mean(sh.best_orientation[:n_plain] == ex.best_orientation)),
            "with_fp32_rerank_of_top8": {
                "value": n_obs / (t_tmpl + t_shr), "seconds": t_tmpl + t_shr, "search_seconds": t_shr,
                "rerank": "FP32 NCC of the 8 best from the FP32 template bank",
                "agreement_with_plain_exhaustive": float(np.mean(shr.best_orientation[:n_plain]
                                                                 == ex.best_orientation)),
                "score_max_rel_diff_vs_plain": float(np.max(np.abs(shr.best_score[:n_plain] - ex.best_score)
                                                            / np.maximum(np.abs(ex.best_score), 1e-30)))},
            "with_simulated_rerank_of_top8": {
                "value": n_obs / (t_tmpl + t_shs), "seconds": t_tmpl + t_shs, "search_seconds": t_shs,
                "rerank": "the 8 best simulated again and scored by the plain scorer",
                "agreement_with_plain_exhaustive": float(np.mean(shs.best_orientation[:n_plain]
                                                                 == ex.best_orientation)),
                "score_identical_fraction": float(np.mean(shs.best_score[:n_plain] == ex.best_score))},
            "gemm_tflop": 2.0 * n_obs * grid.size * 3 * 128 * 65 / 1e12,
            "note": "CTF moved onto the observed image; NCC numerator/denominator as two FP16 tcgen05 GEMMs"},
        "speedup_learned_vs_plain": (n_sim / t_l) / (n_plain / t_ex),
        "agreement_with_exhaustive": float(np.mean(res.best_orientation[:n_plain] == ex.best_orientation)),
        "true_direction_in_top16": float(np.mean(np.any(rt.proposed_directions.cpu().numpy() == true_dir[:, None],
                                                       axis=1))),
        "exhaustive_within_10deg_of_truth": float(np.mean(ang < 10.0)),
        "training": {"images": 200000, "data_seconds": t_data, "train_seconds": hist["seconds"],
                     "steps": n_train_steps, "batch": 256, "final_loss": hist["loss"][-1],
                     "images_per_s": n_train_steps * 256 / hist["seconds"]},
        "device_status": nat.device_status(),
    }


def measure_search_and_refine(dev, seed, n_learned, n_exhaustive):
    """Learned pose search + 20 refinement steps vs exhaustive search + the same refinement.

    A 256^3 volume (6000 Gaussians, pad 2 -> N = 512), 320 x 320 images at
    SNR 0.05, defocus U(5000, 25000) A, poses uniform on SO(3).  The network
    (trained here on 200k simulator images area-downsampled to 128^2) sees
    each observed image downsampled the same way; its top-16 directions x 48
    in-plane angles are rescored at full size against the N = 512 volume,
    with exhaustive fallback below a threshold calibrated on 512 separate
    images (their exhaustive optimum from the template-sharing search).  Both arms then refine rotation and defocus for 20 steps of
    normalised gradient descent through the adjoint kernels
    (cryojax_b200.refine).  The exhaustive arm runs on the first
    `n_exhaustive` images (its cost per image does not depend on the count),
    and the comparison is made on those images.
    """
    import numpy as np
    import torch

    from cryojax_b200 import _native as nat
    from cryojax_b200 import pose_training as PT
    from cryojax_b200 import rotations as rot
    from cryojax_b200 import simulator as S
    from cryojax_b200 import synthetic
    from cryojax_b200.healpix import OrientationGrid
    from cryojax_b200.pose_net import PoseProposalNet
    from cryojax_b200.gradients import observed_to_fourier
    from cryojax_b200.refine import refine_poses, rotation_angle_deg, with_rotations_and_defocus
    from cryojax_b200.search import LearnedPoseSearch, PoseSearch, TemplateSharingSearch

    vol_np = synthetic.gaussian_sum_volume(256, 6000, seed + 50, sigma_range=(1.0, 3.0))
    V = S.FourierVoxelGridVolume.from_real_voxel_grid(vol_np, pad_scale=2.0, device=str(dev))
    cfg = S.BasicImageConfig((320, 320), 2.0, 300.0)
    grid = OrientationGrid(8, 48)
    search = PoseSearch(grid.rotation_matrices())
    df_range = (5000.0, 25000.0)

    def batch(n, s, snr=0.05):
        rng = np.random.default_rng(s)
        q = rot.sample_uniform_quaternions(rng, n)
        df = rng.uniform(*df_range, n)
        clean = PT.simulate_clean_images(V, cfg, q, df)
        g = torch.Generator(device=dev).manual_seed(s)
        noisy = clean + torch.randn(clean.shape, generator=g, device=dev) * torch.sqrt(
            clean.var(dim=(1, 2), keepdim=True) / snr)
        del clean
        ctf = S.AstigmaticCTF(defocus_in_angstroms=df, astigmatism_in_angstroms=np.zeros(n),
                              astigmatism_angle=np.zeros(n))
        model = S.make_image_model(V, cfg, S.QuaternionPose(np.zeros(n), np.zeros(n), wxyz=q),
                                   S.ContrastTransferTheory(ctf, amplitude_contrast_ratio=0.1))
        return model, noisy, q, df

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = fn()
        e1.record()
        torch.cuda.synchronize()
        return out, e0.elapsed_time(e1) / 1000.0

    data, t_data = timed(lambda: PT.TrainingSet(V, cfg, 200000, seed=seed + 51, defocus_range=df_range,
                                                out_size=128))
    net = PoseProposalNet(128, grid.n_dir, max_batch=256, seed=seed + 52)
    hist = PT.train_pose_net(net, data, epochs=12, lr=1e-3, snr=0.05, snr_start=2.0, snr_ramp=0.6, seed=seed + 53)
    del data
    torch.cuda.empty_cache()
    tss = TemplateSharingSearch(grid.rotation_matrices())
    # candidates simulated at full size; the fallback images take the template-sharing exhaustive search
    learned = LearnedPoseSearch(net, grid, top_k=16, search=search, fallback_search=tss)
    cal_model, cal_obs, _, _ = batch(512, seed + 54)
    cal_ex = tss.run(cal_model, cal_obs, rerank_top=8)
    thr = learned.calibrate_threshold(cal_model, cal_obs, cal_ex.best_orientation, target_agreement=0.995)
    # the same proposals scored from the template-sharing search's CTF-free rows (no simulation), the 8 best
    # re-ranked in FP32, the same fallback; threshold calibrated on the same images
    learned_t = LearnedPoseSearch(net, grid, top_k=16, search=search, templates=tss, rerank_top=8,
                                  fallback_search=tss)
    thr_t = learned_t.calibrate_threshold(cal_model, cal_obs, cal_ex.best_orientation, target_agreement=0.995)
    del cal_obs
    torch.cuda.empty_cache()
    model, obs, q, df = batch(n_learned, seed + 55)
    obs_f = observed_to_fourier(obs)

    # starting defocus: the truth + U(-300, 300) A (a CTF-estimation error for the refinement to remove)
    df_start = df + np.random.default_rng(seed + 56).uniform(-300.0, 300.0, n_learned)

    def learned_arm(m, o, of, searcher=learned):
        res = searcher.run(m, o)
        init = with_rotations_and_defocus(m, grid.rotation_matrices(res.best_orientation),
                                          df_start[:len(o)])
        ref = refine_poses(init, of, steps=20, observed_is_fourier=True)
        return res, ref

    def exhaustive_arm(m, o, of):
        # exhaustive over all 36,864 orientations: the template-sharing search with its 8 best per image
        # re-ranked in FP32 (the plain search's answer whenever that is among them; the plain search itself
        # is timed on a smaller sample below); search and refinement timed separately
        res, t_s = timed(lambda: tss.run(m, of, observed_is_fourier=True, rerank_top=8))
        init = with_rotations_and_defocus(m, grid.rotation_matrices(res.best_orientation),
                                          df_start[:len(o)])
        ref, t_r = timed(lambda: refine_poses(init, of, steps=20, observed_is_fourier=True))
        exhaustive_times.update(search=t_s, refine=t_r)
        return res, ref

    exhaustive_times = {}

    def sub_model(k):
        ctf = S.AstigmaticCTF(defocus_in_angstroms=df[:k], astigmatism_in_angstroms=np.zeros(k),
                              astigmatism_angle=np.zeros(k))
        return S.make_image_model(V, cfg, S.QuaternionPose(np.zeros(k), np.zeros(k), wxyz=q[:k]),
                                  S.ContrastTransferTheory(ctf, amplitude_contrast_ratio=0.1))

    tss.build_templates(sub_model(64))  # the fallback's template bank, built before either arm is timed
    learned_arm(sub_model(64), obs[:64].contiguous(), obs_f[:64].contiguous())  # warm-up
    (lres, lref), t_l = timed(lambda: learned_arm(model, obs, obs_f))
    learned_arm(sub_model(64), obs[:64].contiguous(), obs_f[:64].contiguous(), learned_t)  # warm-up
    (ltres, ltref), t_lt = timed(lambda: learned_arm(model, obs, obs_f, learned_t))
    sub = sub_model(n_exhaustive)
    tss._key = None  # the template bank (CTF-free slices of every orientation), timed separately
    _, t_tmpl = timed(lambda: tss.build_templates(sub))
    (eres, eref), t_e = timed(lambda: exhaustive_arm(sub, obs[:n_exhaustive], obs_f[:n_exhaustive].contiguous()))
    n_pl = min(n_exhaustive, 32)  # the plain search (one simulation per orientation) on a small sample
    pl, t_pl = timed(lambda: search.run(sub_model(n_pl), obs_f[:n_pl].contiguous(), observed_is_fourier=True))
    ang = rotation_angle_deg(lref.rotations[:n_exhaustive], eref.rotations)
    ang_t = rotation_angle_deg(ltref.rotations[:n_exhaustive], eref.rotations)
    R_true = rot.quat_to_matrix(q)
    per_image_plain_plus_refine = 1.0 / (n_pl / t_pl) + exhaustive_times["refine"] / n_exhaustive
    return {
        "metric": "pose search + 20 refinement steps, images/s (320^2 images, N=512, 36,864 orientations)",
        "unit": "images/s",
        "learned_plus_refine": {"value": n_learned / t_l, "seconds": t_l, "n_images": n_learned,
                                "fallback_fraction": float(lres.fallback.mean()), "threshold": thr,
                                "refine_accepted_steps_mean": float(lref.accepted.mean())},
        "exhaustive_plus_refine": {"value": n_exhaustive / t_e, "seconds": t_e, "n_images": n_exhaustive,
                                   "search": "template-sharing exhaustive, 8 best per image re-ranked in FP32 from the FP32 template bank",
                                   "template_bank_seconds": t_tmpl,
                                   "plain_exhaustive_search": {
                                       "value": n_pl / t_pl, "n_images": n_pl,
                                       "agreement_with_template_search": float(np.mean(
                                           pl.best_orientation == eres.best_orientation[:n_pl]))}},
        "speedup": (n_learned / t_l) / (n_exhaustive / t_e),
        "speedup_vs_plain_exhaustive_plus_refine": (n_learned / t_l) * per_image_plain_plus_refine,
        "learned_template_rows_plus_refine": {
            "value": n_learned / t_lt, "seconds": t_lt, "n_images": n_learned,
            "scoring": "the network's 16 x 48 candidates scored from the template-sharing search's FP16 rows "
                       "(cjx_ncc_directions), the 8 best re-ranked in FP32 from the FP32 template bank (template "
                       "banks prebuilt, as for the exhaustive arm)",
            "fallback_fraction": float(ltres.fallback.mean()), "threshold": thr_t,
            "speedup_vs_exhaustive_plus_refine": (n_learned / t_lt) / (n_exhaustive / t_e),
            "speedup_vs_plain_exhaustive_plus_refine": (n_learned / t_lt) * per_image_plain_plus_refine,
            "fraction_within_2deg_of_exhaustive": float(np.mean(ang_t < 2.0)),
            "search_agreement_with_exhaustive": float(np.mean(ltres.best_orientation[:n_exhaustive]
                                                              == eres.best_orientation))},
        "refine_seconds_per_image": exhaustive_times["refine"] / n_exhaustive,
        "fraction_within_2deg_of_exhaustive": float(np.mean(ang < 2.0)),
        "search_agreement_with_exhaustive": float(np.mean(lres.best_orientation[:n_exhaustive]
                                                          == eres.best_orientation)),
        "median_error_to_truth_deg": {
            "learned_refined": float(np.median(rotation_angle_deg(lref.rotations, R_true))),
            "exhaustive_refined": float(np.median(rotation_angle_deg(eref.rotations, R_true[:n_exhaustive])))},
        "median_defocus_error_A": {"start": float(np.median(np.abs(df_start - df))),
                                   "learned_refined": float(np.median(np.abs(lref.defocus - df)))},
        "training": {"images": 200000, "input": "320^2 area-downsampled to 128^2", "data_seconds": t_data,
                     "train_seconds": hist["seconds"], "final_loss": hist["loss"][-1]},
        "device_status": nat.device_status(),
    }


def measure_spline(dev, grid, batch, cfg, steps, warmup, n_images, cpu_images):
    """FourierVoxelSplineVolume at the headline shape: coefficients of the headline grid solved on the
    device, then `n_images` of the headline images through the cubic-spline gather (x-pair coefficients)."""
    import numpy as np
    import torch

    from cryojax_b200 import _native as nat
    from cryojax_b200 import simulator as S

    n = grid.shape[0]
    ws = torch.empty(nat.spline_coefficients_workspace_size(n), dtype=torch.uint8, device=dev)
    coef = torch.empty((n + 2,) * 3, dtype=torch.complex64, device=dev)
    nat.spline_coefficients(grid, coef, ws)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    nat.spline_coefficients(grid, coef, ws)
    e1.record()
    torch.cuda.synchronize()
    coef_ms = e0.elapsed_time(e1)
    del ws
    vol = S.FourierVoxelSplineVolume(coef)
    sl = slice(0, n_images)
    pose = S.QuaternionPose(batch.offsets[sl, 0], batch.offsets[sl, 1], wxyz=batch.wxyz[sl])
    tt = S.ContrastTransferTheory(S.AstigmaticCTF(batch.defocus[sl], batch.astigmatism[sl],
                                                  batch.astigmatism_angle[sl]))
    model = S.make_image_model(vol, cfg, pose, tt)
    integ = model.volume_integrator
    flags = model._flags()
    py, px = cfg.padded_shape
    pd = torch.as_tensor(model.image_params(), device=dev)
    order = torch.as_tensor(S.orientation_order(pose.rotation_matrices()), device=dev)
    out = torch.empty((n_images, py, px // 2 + 1), dtype=torch.complex64, device=dev)
    desc = nat.make_desc(n, py, px, flags | integ.device_grid(vol)[1])
    wsf = torch.empty(max(nat.workspace_size(desc, n_images), 1), dtype=torch.uint8, device=dev)

    def step():
        integ.run(vol, cfg, None, flags, params_device=pd, out=out, workspace=wsf, order=order)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    nat.profile_enable(True)
    step()
    torch.cuda.synchronize()
    prof = nat.profile_read()
    nat.profile_enable(False)
    res = {"value": n_images / (ms / 1000.0), "unit": UNIT, "images": n_images, "ms_per_step": ms,
           "layout": "x-pair bricked coefficients, side N + 2 = %d" % (n + 2),
           "coefficients_ms": coef_ms,
           "gather_us_per_image": prof["k_gather_slice"][1] * 1000.0 / n_images,
           "kernels_per_step": {k: {"launches": c, "ms": t} for k, (c, t) in prof.items()},
           "bound": "L1 data-stage wavefronts (ncu: 83 % of peak; DRAM 27 %)"}
    got = out[:PARITY_IMAGES].cpu().numpy()
    del out, wsf, pd
    if cpu_images:
        from oracle import cryojax_oracle as O

        coef_h = coef.cpu().numpy().astype(np.complex128)
        res["parity"] = oracle_parity(coef_h, got, oracle_specs(batch, range(len(got)), cfg.shape), n=n,
                                      grid_source="the device-solved coefficients in float64 (the solve itself is "
                                                  "checked against the oracle's banded solve in the tests)",
                                      spline=True)
        fs = O.make_frequency_slice((n, n), outputs_rfftfreqs=False)
        t0 = time.perf_counter()
        for b in range(cpu_images):
            spec = O.ImageSpec(shape=cfg.shape, pixel_size=2.0, voltage_in_kilovolts=300.0, wxyz=batch.wxyz[b],
                               offset_in_angstroms=batch.offsets[b], defocus_in_angstroms=batch.defocus[b],
                               astigmatism_in_angstroms=batch.astigmatism[b],
                               astigmatism_angle=batch.astigmatism_angle[b])
            O.compute_fourier_image(coef_h, fs, spec, spline=True)
        wall = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": cpu_images / wall, "unit": UNIT, "cores": 1, "kind": "port",
                               "sample": f"{cpu_images} images through the float64 NumPy oracle's 64-tap "
                                         f"spline restatement, 1 process ({wall:.1f} s)"}
        del coef_h
    del vol, coef
    return res


def measure_ewald(dev, volume, batch, cfg, steps, warmup, n_images, cpu_images):
    """EwaldSphereExtraction + ContrastTransferTheory (non-projection contrast) on the headline volume and
    images: `n_images` of them, x-pair bricked trilinear grid."""
    import numpy as np
    import torch

    from cryojax_b200 import _native as nat
    from cryojax_b200 import simulator as S

    sl = slice(0, n_images)
    pose = S.QuaternionPose(batch.offsets[sl, 0], batch.offsets[sl, 1], wxyz=batch.wxyz[sl])
    tt = S.ContrastTransferTheory(S.AstigmaticCTF(batch.defocus[sl], batch.astigmatism[sl],
                                                  batch.astigmatism_angle[sl]))
    integ = S.EwaldSphereExtraction(outputs_integral=False)
    model = S.make_image_model(volume, cfg, pose, tt, volume_integrator=integ)
    flags = model._flags()
    n = volume.shape[0]
    py, px = cfg.padded_shape
    pd = torch.as_tensor(model.image_params(), device=dev)
    order = torch.as_tensor(S.orientation_order(pose.rotation_matrices()), device=dev)
    out = torch.empty((n_images, py, px // 2 + 1), dtype=torch.complex64, device=dev)
    desc = nat.make_desc(n, py, px, flags | integ._base_flags() | integ.device_grid(volume)[1])
    ws = torch.empty(max(nat.workspace_size(desc, n_images), 1), dtype=torch.uint8, device=dev)

    def step():
        integ.run(volume, cfg, None, flags, params_device=pd, out=out, workspace=ws, order=order)

    for _ in range(warmup):
        step()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    nat.profile_enable(True)
    step()
    torch.cuda.synchronize()
    prof = nat.profile_read()
    nat.profile_enable(False)
    res = {"value": n_images / (ms / 1000.0), "unit": UNIT, "images": n_images, "ms_per_step": ms,
           "layout": "x-pair bricked grid, trilinear",
           "kernels_per_step": {k: {"launches": c, "ms": t} for k, (c, t) in prof.items()},
           "_parity": out[:PARITY_IMAGES].cpu().numpy()}
    del out, ws, pd
    if cpu_images:
        from oracle import cryojax_oracle as O

        grid_h = volume.fourier_voxel_grid.cpu().numpy().astype(np.complex128)
        fs = O.make_frequency_slice((n, n), outputs_rfftfreqs=False)
        t0 = time.perf_counter()
        for b in range(cpu_images):
            spec = O.ImageSpec(shape=cfg.shape, pixel_size=2.0, voltage_in_kilovolts=300.0, wxyz=batch.wxyz[b],
                               offset_in_angstroms=batch.offsets[b], defocus_in_angstroms=batch.defocus[b],
                               astigmatism_in_angstroms=batch.astigmatism[b],
                               astigmatism_angle=batch.astigmatism_angle[b])
            O.compute_fourier_image(grid_h, fs, spec, ewald=True)
        wall = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": cpu_images / wall, "unit": UNIT, "cores": 1, "kind": "port",
                               "sample": f"{cpu_images} images through the float64 NumPy oracle's Ewald-sphere "
                                         f"restatement, 1 process ({wall:.1f} s)"}
        del grid_h
    return res


def measure_relion_stack(dev, volume, cfg, n_particles, seed):
    """simulate_particle_stack end to end: a RELION STAR file of `n_particles` (random Euler poses, CTFs and
    origins) is read, simulated in batches of 1024 through the device launch and written as MRC stacks of 1024
    images.  Host wall clock; the split into device and I/O time is measured inside."""
    import pathlib
    import shutil
    import tempfile

    import numpy as np
    import torch

    from cryojax_b200 import relion
    from cryojax_b200 import simulator as S

    rng = np.random.default_rng(seed)
    n = n_particles
    ox, oy = rng.uniform(-20, 20, n), rng.uniform(-20, 20, n)
    rot, psi = rng.uniform(-180, 180, n), rng.uniform(-180, 180, n)
    tilt = np.rad2deg(np.arccos(rng.uniform(-1, 1, n)))
    df, astig, ang = rng.uniform(5000, 25000, n), rng.uniform(0, 500, n), rng.uniform(0, 180, n)
    root = pathlib.Path(tempfile.mkdtemp(prefix="relion_bench_"))

    def write_star(path, k):
        pf = relion.RelionParticleParameterFile(path, mode="w")
        pf.append({"image_config": S.BasicImageConfig(cfg.shape, 2.0, 300.0),
                   "pose": S.EulerAnglePose(ox[:k], oy[:k], rot[:k], tilt[:k], psi[:k]),
                   "transfer_theory": S.ContrastTransferTheory(S.AstigmaticCTF(df[:k], astig[:k], ang[:k], 2.7))})
        pf.save()

    device_s = [0.0]

    def compute(parameters, vol, _):
        torch.cuda.synchronize()
        t = time.perf_counter()
        model = S.make_image_model(vol, parameters["image_config"], parameters["pose"], parameters["transfer_theory"])
        dimg = model.simulate()
        img = torch.empty(dimg.shape, dtype=dimg.dtype, pin_memory=True)
        img.copy_(dimg)
        device_s[0] += time.perf_counter() - t
        return img

    def run(star_in, project, batch):
        pf = relion.RelionParticleParameterFile(star_in)
        pf.path_to_starfile = project / "sim.star"
        ds = relion.RelionParticleStackDataset(pf, project, mode="w")
        relion.simulate_particle_stack(ds, compute, constant_args=volume, batch_size=batch, images_per_file=batch)

    try:
        write_star(root / "warm.star", 64)
        write_star(root / "in.star", n)
        run(root / "warm.star", root / "warm", 64)
        device_s[0] = 0.0
        t0 = time.perf_counter()
        run(root / "in.star", root / "out", 1024)
        wall = time.perf_counter() - t0
        written = sum(f.stat().st_size for f in (root / "out").iterdir())
    finally:
        shutil.rmtree(root, ignore_errors=True)
    return {"value": n / wall, "unit": UNIT, "particles": n, "wall_s": wall,
            "device_simulate_and_d2h_s": device_s[0], "host_io_and_parsing_s": wall - device_s[0],
            "bytes_written": written,
            "path": "STAR read -> RelionParticleParameterFile[batch] -> make_image_model(...).simulate() on the "
                    "device (batches of 1024) -> D2H -> MRC stacks of 1024 images + STAR write"}


def measure_render(dev, seed, n_atoms=50000, shape=(256, 256, 256), voxel=1.0, cpu_sample=True):
    """GaussianMixtureRenderFn: `n_atoms` atoms x 5 Gaussians (variances 0.2-2.0 A^2, the range of tabulated
    atomic scattering factors plus B-factors) spread over a 200 A box, rendered into a 256^3 grid at 1 A."""
    import numpy as np
    import torch

    from cryojax_b200 import _native as nat

    rng = np.random.default_rng(seed)
    pos = torch.as_tensor(rng.uniform(-100, 100, (n_atoms, 3)), dtype=torch.float32, device=dev)
    amp = torch.as_tensor(rng.uniform(0.1, 1.0, (n_atoms, 5)), dtype=torch.float32, device=dev)
    var = torch.as_tensor(rng.uniform(0.2, 2.0, (n_atoms, 5)), dtype=torch.float32, device=dev)
    out = torch.empty(shape, dtype=torch.float32, device=dev)
    for _ in range(2):
        nat.render_gaussians(shape, voxel, pos, amp, var, out=out)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    reps = 5
    for _ in range(reps):
        nat.render_gaussians(shape, voxel, pos, amp, var, out=out)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    # window voxels actually updated (the 7-sigma boxes clipped to the grid), for the update rate
    sig = np.sqrt(var.max(dim=1).values.cpu().numpy())
    reach = 7.0 * sig + voxel
    p = pos.cpu().numpy()
    upd = 1.0
    for a, d in enumerate((shape[2], shape[1], shape[0])):
        lo = np.clip(np.floor((p[:, a] - reach) / voxel + d // 2), 0, d)
        hi = np.clip(np.ceil((p[:, a] + reach) / voxel + d // 2), -1, d - 1)
        upd = upd * np.maximum(hi - lo + 1, 0)
    res = {"value": n_atoms / (ms / 1000.0), "unit": "atoms/s", "ms": ms, "atoms": n_atoms, "gaussians_per_atom": 5,
           "grid": list(shape), "voxel_A": voxel, "voxel_updates_per_s": float(upd.sum()) / (ms / 1000.0)}
    if cpu_sample:
        from oracle import cryojax_oracle as O

        k = 100
        t0 = time.perf_counter()
        O.render_gaussian_mixture((64, 64, 64), voxel, p[:k] * 0.25, amp[:k].cpu().numpy(), var[:k].cpu().numpy())
        wall = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": k / wall, "unit": "atoms/s", "cores": 1, "kind": "port",
                               "sample": f"{k} atoms into a 64^3 grid through the float64 NumPy oracle's dense "
                                         f"restatement (every voxel against every Gaussian, as the reference), "
                                         f"1 process ({wall:.2f} s)"}
    return res


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel):
    """DRAM bytes per image of `kernel` from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(path):
        return None
    try:
        d = json.load(open(path))
        return d.get(kernel, {}).get("dram_bytes_per_image")
    except Exception:
        return None


def ncu_limiter(kernel):
    """The unit that bounds `kernel` and its fraction of peak, from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(path):
        return None
    try:
        return json.load(open(path)).get(kernel, {}).get("limiter")
    except Exception:
        return None


def run_probe(kind, seed):
    """Small fixed workloads for ncu captures: few launches before the one of interest."""
    import numpy as np
    import torch

    from cryojax_b200 import _native as nat

    dev = torch.device("cuda", 0)
    out = {"probe": kind}

    def ev_time(fn, reps=1):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    if kind == "gemm":
        g = torch.Generator(device=dev).manual_seed(seed)
        for name, (m, n, k, dt, flags) in {
            "bf16_8192^3": (8192, 8192, 8192, torch.bfloat16, 0),
            "fp16_template_ncc_1024x36864x16640": (1024, 36864, 16640, torch.float16, nat.CJX_GEMM_F16),
        }.items():
            a = torch.randn((m, k), generator=g, device=dev).to(dt)
            b = torch.randn((n, k), generator=g, device=dev).to(dt)
            c = torch.empty((m, n), device=dev)
            for _ in range(2):
                nat.gemm(a, b, c, flags=flags)
            ms = ev_time(lambda: nat.gemm(a, b, c, flags=flags))
            out[name] = {"ms": ms, "tflops": 2.0 * m * n * k / ms / 1e9}
            del a, b, c
    elif kind == "search":
        from cryojax_b200 import simulator as S
        from cryojax_b200 import synthetic
        from cryojax_b200.healpix import OrientationGrid
        from cryojax_b200.search import PoseSearch

        vol = S.FourierVoxelGridVolume.from_real_voxel_grid(synthetic.gaussian_sum_volume(128, 800, seed),
                                                            pad_scale=2.0, device=str(dev))
        b = synthetic.image_batch(8, seed + 1, max_offset=0.0, defocus_range=(8000.0, 20000.0))
        cfg = S.BasicImageConfig((128, 128), 2.0, 300.0)
        model = S.make_image_model(vol, cfg, S.QuaternionPose(b.offsets[:, 0], b.offsets[:, 1], wxyz=b.wxyz),
                                   S.ContrastTransferTheory(S.AstigmaticCTF(b.defocus, b.astigmatism,
                                                                            b.astigmatism_angle)))
        obs = model.simulate()
        grid = OrientationGrid(8, 48)
        ps = PoseSearch(grid.rotation_matrices())
        ms = ev_time(lambda: ps.run(model, obs))
        out["plain_exhaustive_8_images"] = {"ms": ms, "candidates_per_s": 8 * grid.size / (ms / 1000.0)}
    elif kind == "ncc":
        # the learned search's candidate sums (cjx_ncc_directions) and FP32 bank re-ranking (cjx_ncc_rerank32) at
        # the pose-search sizes: 4096 images 128^2 (kp = 128 x 65), 16 proposed directions of 768 x 48 in-plane
        # templates, 8 re-ranked candidates per image; random FP16 / FP32 rows (two warm-up runs, one timed)
        g = torch.Generator(device=dev).manual_seed(seed)
        n, kd, n_dir, ni, py, px = 4096, 16, 768, 48, 128, 128
        kp = py * (px // 2 + 1)
        T = n_dir * ni
        y16 = torch.randn((n, 2 * kp), generator=g, device=dev).half()
        z16 = torch.rand((n, kp), generator=g, device=dev).half()
        s16 = torch.randn((T, 2 * kp), generator=g, device=dev).half()
        p16 = torch.rand((T, kp), generator=g, device=dev).half()
        dirs = torch.randint(0, n_dir, (n, kd), generator=g, device=dev, dtype=torch.int32)
        num = torch.empty((n, kd * ni), device=dev)
        den = torch.empty_like(num)
        ws = torch.empty(nat.ncc_directions_workspace_size(n, kd, n_dir), dtype=torch.uint8, device=dev)
        run = lambda: nat.ncc_directions(y16, z16, s16, p16, kp, dirs, n_dir, ni, num, den, ws)
        for _ in range(2):
            run()
        ms = ev_time(run)
        flop = 2.0 * n * kd * ni * 3 * kp
        out["ncc_directions"] = {"ms": ms, "tflops": flop / ms / 1e9}
        del s16, p16
        bank = torch.randn((T, py, px // 2 + 1), generator=g, device=dev, dtype=torch.complex64)
        y32 = torch.randn((n, py, px // 2 + 1), generator=g, device=dev, dtype=torch.complex64)
        z32 = torch.rand((n, py, px // 2 + 1), generator=g, device=dev)
        oo = torch.rand(n, generator=g, device=dev) + 1.0
        cand = torch.randint(0, T, (n, 8), generator=g, device=dev, dtype=torch.int32)
        bs = torch.empty(n, device=dev)
        bo = torch.empty(n, dtype=torch.int32, device=dev)
        run = lambda: nat.ncc_rerank32(bank, py, px, y32, z32, oo, cand, bs, bo)
        for _ in range(2):
            run()
        ms = ev_time(run)
        out["ncc_rerank32"] = {"ms": ms, "bank_bytes_read_per_run": n * 8 * kp * 8,
                               "gbs": n * 8 * kp * 8 / ms / 1e6}
    elif kind == "render":
        # GaussianMixtureRenderFn: 50k atoms x 5 Gaussians into 256^3 at 1 A (two warm-up launches, one timed)
        rng = np.random.default_rng(seed)
        pos = torch.as_tensor(rng.uniform(-100, 100, (50000, 3)), dtype=torch.float32, device=dev)
        amp = torch.as_tensor(rng.uniform(0.1, 1.0, (50000, 5)), dtype=torch.float32, device=dev)
        var = torch.as_tensor(rng.uniform(0.2, 2.0, (50000, 5)), dtype=torch.float32, device=dev)
        grid = torch.empty((256, 256, 256), dtype=torch.float32, device=dev)
        for _ in range(2):
            nat.render_gaussians(grid.shape, 1.0, pos, amp, var, out=grid)
        ms = ev_time(lambda: nat.render_gaussians(grid.shape, 1.0, pos, amp, var, out=grid))
        out["render_50k_atoms_256^3"] = {"ms": ms, "atoms_per_s": 50000 / (ms / 1000.0)}
    elif kind == "ewald":
        from cryojax_b200 import simulator as S
        from cryojax_b200 import synthetic

        # EwaldSphereExtraction + CTF at the benchmark shape (N = 512 -> 320^2), 64 images
        vol = S.FourierVoxelGridVolume.from_real_voxel_grid(synthetic.gaussian_sum_volume(256, 6000, seed),
                                                            pad_scale=2.0, device=str(dev))
        b = synthetic.image_batch(64, seed + 1)
        cfg = S.BasicImageConfig((320, 320), 2.0, 300.0)
        integ = S.EwaldSphereExtraction(outputs_integral=False)
        model = S.make_image_model(vol, cfg, S.QuaternionPose(b.offsets[:, 0], b.offsets[:, 1], wxyz=b.wxyz),
                                   S.ContrastTransferTheory(S.AstigmaticCTF(b.defocus, b.astigmatism,
                                                                            b.astigmatism_angle)),
                                   volume_integrator=integ)
        pd = torch.as_tensor(model.image_params(), device=dev)
        o = torch.empty((64, 320, 161), dtype=torch.complex64, device=dev)

        def fwd():
            integ.run(vol, cfg, None, model._flags(), params_device=pd, out=o)

        for _ in range(3):
            fwd()
        ms = ev_time(fwd)
        out["ewald_forward_64_images"] = {"ms": ms, "images_per_s": 64 / (ms / 1000.0)}
    elif kind == "spline":
        from cryojax_b200 import simulator as S
        from cryojax_b200 import synthetic

        # FourierVoxelSplineVolume at the benchmark shape (N = 512 -> 320^2), 64 images, x-pair coefficients
        grid = S.FourierVoxelGridVolume.from_real_voxel_grid(synthetic.gaussian_sum_volume(256, 6000, seed),
                                                             pad_scale=2.0, device=str(dev)).fourier_voxel_grid
        n = grid.shape[0]
        ws = torch.empty(nat.spline_coefficients_workspace_size(n), dtype=torch.uint8, device=dev)
        coef = torch.empty((n + 2,) * 3, dtype=torch.complex64, device=dev)
        nat.spline_coefficients(grid, coef, ws)
        out["coefficients_ms_N512"] = ev_time(lambda: nat.spline_coefficients(grid, coef, ws))
        del grid, ws
        torch.cuda.empty_cache()
        vol = S.FourierVoxelSplineVolume(coef)
        b = synthetic.image_batch(64, seed + 1)
        cfg = S.BasicImageConfig((320, 320), 2.0, 300.0)
        model = S.make_image_model(vol, cfg, S.QuaternionPose(b.offsets[:, 0], b.offsets[:, 1], wxyz=b.wxyz),
                                   S.ContrastTransferTheory(S.AstigmaticCTF(b.defocus, b.astigmatism,
                                                                            b.astigmatism_angle)))
        integ = model.volume_integrator
        pd = torch.as_tensor(model.image_params(), device=dev)
        o = torch.empty((64, 320, 161), dtype=torch.complex64, device=dev)

        def fwd():
            integ.run(vol, cfg, None, model._flags(), params_device=pd, out=o)

        for _ in range(3):
            fwd()
        ms = ev_time(fwd)
        out["spline_forward_64_images"] = {"ms": ms, "images_per_s": 64 / (ms / 1000.0)}
    else:
        from cryojax_b200.pose_net import PoseProposalNet

        net = PoseProposalNet(128, 768, max_batch=256, seed=seed)
        g = torch.Generator(device=dev).manual_seed(seed)
        imgs = torch.randn((256, 128, 128), generator=g, device=dev)
        labels = torch.randint(0, 768, (256,), generator=g, device=dev, dtype=torch.int32)

        def step():
            nat.cnn_noisy_normalize(imgs, net.x0, snr=0.05, seed=1)
            net.forward(B=256)
            net.backward(labels, B=256)
            net.adam_step(1e-3)

        for _ in range(2):
            step()
        ms = ev_time(step)
        out["train_step_batch256"] = {"ms": ms, "images_per_s": 256 / (ms / 1000.0)}
        # proposals (inference): first layer without im2col, the others as implicit GEMMs on mma.sync tiles
        x = torch.randn((2048, 128, 128), generator=g, device=dev)

        def prop():
            net.propose(x, k=16, n_inplane=48)

        for _ in range(2):
            prop()
        ms = ev_time(prop)
        out["proposals_batch2048"] = {"ms": ms, "images_per_s": 2048 / (ms / 1000.0)}
    out["device_status"] = nat.device_status()
    print(json.dumps(out))
    return 0


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.probe:
        return run_probe(args.probe, args.seed)

    import numpy as np
    import torch

    from cryojax_b200 import _native as nat
    from cryojax_b200 import simulator as S
    from cryojax_b200 import synthetic
    from cryojax_b200.pipeline import HostStreamingSimulator

    from cryojax_b200 import replicas

    info = replicas.rank_info()
    rank, world, local = info.rank, info.world, info.local_rank
    replicas.init("nccl", info)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    nat.load_library()

    # ---- inputs (seeded; one volume replica per rank, own images per rank)
    vol_np = synthetic.gaussian_sum_volume(args.box, args.gaussians, args.seed, sigma_range=(1.0, 3.0))
    volume = S.FourierVoxelGridVolume.from_real_voxel_grid(vol_np, pad_scale=args.pad_scale, device=str(dev))
    n = volume.shape[0]
    batch = synthetic.image_batch(args.images, replicas.image_seed(args.seed, rank))
    pose = S.QuaternionPose(batch.offsets[:, 0], batch.offsets[:, 1], wxyz=batch.wxyz)
    tt = S.ContrastTransferTheory(S.AstigmaticCTF(batch.defocus, batch.astigmatism, batch.astigmatism_angle))
    cfg = S.BasicImageConfig((args.image, args.image), 2.0, 300.0)
    model = S.make_image_model(volume, cfg, pose, tt)
    params_h = model.image_params()
    params_d = torch.as_tensor(params_h, device=dev)
    if args.ilp:
        nat.tuning_set(nat.CJX_TUNE_GATHER_ILP, args.ilp)
    for key, val in ((nat.CJX_TUNE_GATHER_MODE, args.gather_mode), (nat.CJX_TUNE_SCATTER_VEC, args.scatter_mode)):
        if val >= 0:
            nat.tuning_set(key, val)
    order_d = None
    if args.order == "orientation":
        order_d = torch.as_tensor(S.orientation_order(pose.rotation_matrices()), device=dev)
    flags = model._flags()
    integ = model.volume_integrator
    integ.use_bricked_layout = args.layout != "linear"
    integ.pair_layout = args.layout == "pairs"
    py, px = cfg.padded_shape
    out = torch.empty((args.images, py, px // 2 + 1), dtype=torch.complex64, device=dev)
    desc = nat.make_desc(n, py, px, flags, integ.fill_value, args.chunk)
    ws_bytes = nat.workspace_size(desc, args.images)
    ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()

    def step():
        integ.run(volume, cfg, None, flags, params_device=params_d, out=out, workspace=ws, stream=stream,
                  images_per_chunk=args.chunk, order=order_d)

    def barrier():
        replicas.barrier(info)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    # ---- device-timed region
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks.mark()
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    t_ms = replicas.max_over_ranks(ev0.elapsed_time(ev1), info, dev)
    value = replicas.job_rate(args.images, info, args.steps, t_ms)

    # ---- per-kernel timing (one extra profiled step, not part of `value`)
    nat.profile_enable(True)
    step()
    torch.cuda.synchronize()
    prof = nat.profile_read()
    nat.profile_enable(False)
    headline_got = out[:PARITY_IMAGES].cpu().numpy()  # the timed steps' images 0..7 (every step writes the same)
    launches_per_step = sum(c for c, _ in prof.values())
    top = max(prof.items(), key=lambda kv: kv[1][1])
    top_name, (top_count, top_ms) = top
    images_per_launch = args.images / top_count
    gather_voxels = unique_voxels_per_image(n, pose.rotation_matrices())
    alg = algorithmic_bytes_per_image(top_name, n, py, px, gather_voxels)
    achieved = alg * images_per_launch / (top_ms / top_count / 1000.0) / 1e9
    hbm_peak, peak_kind = measured_peaks()
    trf = ncu_traffic(top_name)

    # ---- L2 read bandwidth probe (roofline denominator for the gather)
    l2 = None
    try:
        buf = torch.empty(48 << 20, dtype=torch.uint8, device=dev)
        sink = torch.zeros(4, dtype=torch.float32, device=dev)
        nat.probe_read_bandwidth(buf, 2, sink)
        torch.cuda.synchronize()
        nat.profile_enable(True)
        nat.probe_read_bandwidth(buf, 50, sink)
        torch.cuda.synchronize()
        pr = nat.profile_read()
        nat.profile_enable(False)
        l2_gbs = buf.numel() * 50 / (pr["k_read_probe"][1] / 1000.0) / 1e9
        gname = next(k for k in ("k_gather_colifft_fused", "k_gather_slice", "k_gather_colifft", "k_slice_direct")
                     if k in prof)
        gather = prof[gname]
        g_alg = (72 * n * (n // 2 + 1) if gname in ("k_gather_slice", "k_slice_direct") else
                 algorithmic_bytes_per_image(gname, n, py, px)) * args.images / (gather[1] / 1000.0) / 1e9
        l2 = {"kernel": gname, "bytes_per_sample": 72 if gname in ("k_gather_slice", "k_slice_direct") else
              "64 per sample (8 corner loads) + the T1 window store",
              "achieved": g_alg, "peak": l2_gbs, "unit": "GB/s",
              "frac": g_alg / l2_gbs,
              "peak_source": "k_read_probe, 48 MB buffer x 50 passes (measured in this run)"}
        del buf
    except Exception as e:  # measurement helper only
        l2 = {"error": str(e)}

    # ---- end to end through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        sim = HostStreamingSimulator(volume, cfg, integ, flags, sub_batch=2048, images_per_chunk=args.chunk)
        ph = sim.pinned_params(params_h)
        oh = sim.pinned_output(args.images)
        for _ in range(2):
            sim.run(ph, oh)
        torch.cuda.synchronize()
        barrier()
        e_steps = max(2, min(args.steps, 5))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(e_steps):
            sim.run(ph, oh)
        e1.record(stream)
        torch.cuda.synchronize()
        et_ms = replicas.max_over_ranks(e0.elapsed_time(e1), info, dev)
        e2e = {"value": replicas.job_rate(args.images, info, e_steps, et_ms), "unit": UNIT,
               "h2d_bytes_per_step": int(ph.numel() * ph.element_size()),
               "d2h_bytes_per_step": int(oh.numel() * oh.element_size()),
               "path": "HostStreamingSimulator: pinned host params -> H2D -> cjx_slice_ctf_forward -> D2H "
                       "into pinned host images, 2 streams, 2048-image sub-batches after a 256/512/1024 ramp"}
        del oh, ph, sim
        try:  # the host link's own device-to-host rate: the e2e roof when the images dominate the traffic
            nbytes = 1 << 30
            src = torch.empty(nbytes, dtype=torch.uint8, device=dev)
            dst = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
            for _ in range(2):
                dst.copy_(src, non_blocking=True)
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(4):
                dst.copy_(src, non_blocking=True)
            e1.record(stream)
            torch.cuda.synchronize()
            link_gbs = 4 * nbytes / (e0.elapsed_time(e1) * 1e6)
            d2h_gbs = e2e["d2h_bytes_per_step"] * e_steps / (et_ms * 1e6)
            e2e["host_link"] = {"d2h_probe_gbs": link_gbs, "d2h_achieved_gbs": d2h_gbs,
                                "frac": d2h_gbs / link_gbs,
                                "probe": "4 x 1 GiB device -> pinned host copies, CUDA events"}
            del src, dst
        except Exception as e:  # measurement helper only
            e2e["host_link"] = {"error": str(e)}

    # ---- mixed-size batch (configuration with four volume sizes)
    batched = None
    if not args.no_batched:
        try:
            del out, ws
            torch.cuda.empty_cache()
            batched = measure_batched_uneven(dev, max(3, min(args.steps, 10)), 3, args.seed)
        except Exception as e:
            batched = {"error": repr(e)}

    # ---- loss + gradient (differentiation configuration)
    gradient = None
    if not args.no_grad:
        try:
            torch.cuda.empty_cache()
            gradient = measure_gradient(dev, max(3, min(args.steps, 10)), 2, args.seed)
        except Exception as e:
            gradient = {"error": repr(e)}

    # ---- pose search, learned vs plain exhaustive
    pose_search = None
    if not args.no_search and world == 1:
        try:
            torch.cuda.empty_cache()
            pose_search = measure_pose_search(dev, args.seed, args.search_images)
        except Exception as e:
            pose_search = {"error": repr(e)}

    # ---- pose search + refinement at 320^2 from N = 512
    search_refine = None
    if not args.no_refine and world == 1:
        try:
            torch.cuda.empty_cache()
            search_refine = measure_search_and_refine(dev, args.seed, args.refine_images,
                                                      args.refine_exhaustive_images)
        except Exception as e:
            search_refine = {"error": repr(e)}

    # ---- spline volume (cubic-spline extraction) at the headline shape
    spline = None
    if not args.no_spline and world == 1:
        try:
            torch.cuda.empty_cache()
            spline = measure_spline(dev, volume.fourier_voxel_grid, batch, cfg, max(3, min(args.steps, 10)), 3,
                                    min(4096, args.images), 0 if args.no_cpu_baseline else 2)
        except Exception as e:
            spline = {"error": repr(e)}

    # ---- Ewald-sphere extraction at the headline shape
    ewald = None
    if not args.no_ewald and world == 1:
        try:
            torch.cuda.empty_cache()
            ewald = measure_ewald(dev, volume, batch, cfg, max(3, min(args.steps, 10)), 3, min(4096, args.images),
                                  0 if args.no_cpu_baseline else 2)
        except Exception as e:
            ewald = {"error": repr(e)}

    # ---- RELION particle stack: STAR in, MRC stacks out
    relion_stack = None
    if not args.no_relion and world == 1:
        try:
            torch.cuda.empty_cache()
            relion_stack = measure_relion_stack(dev, volume, cfg, 4096, args.seed + 60)
        except Exception as e:
            relion_stack = {"error": repr(e)}

    # ---- Gaussian-mixture rendering (volume preparation on the device)
    render = None
    if not args.no_render and world == 1:
        try:
            torch.cuda.empty_cache()
            render = measure_render(dev, args.seed + 70, cpu_sample=not args.no_cpu_baseline)
        except Exception as e:
            render = {"error": repr(e)}

    # ---- CPU legs (rank 0, N=1 only): the oracle as CPU baseline and as the parity check of the timed images
    cpu = None
    parity = None
    batched_parity = batched.pop("_parity", None) if isinstance(batched, dict) else None
    ewald_parity = ewald.pop("_parity", None) if isinstance(ewald, dict) else None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import cryojax_oracle as O

        grid_f64 = None
        try:
            grid_f64, _ = O.fourier_voxel_grid_from_real_voxel_grid(vol_np, pad_scale=args.pad_scale)
            v, done, wall = cpu_oracle_throughput(grid_f64, batch, args.cpu_sample, args.image, 2.0, 300.0, 1)
            cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
                   "sample": f"{done} images of this workload through the float64 NumPy oracle of the reference "
                             f"path, 1 process ({wall:.1f} s)"}
        except Exception as e:
            cpu = {"error": str(e)}
        parity = {}
        try:
            parity["headline"] = oracle_parity(grid_f64, headline_got,
                                               oracle_specs(batch, range(len(headline_got)), cfg.shape))
        except Exception as e:
            parity["headline"] = {"error": repr(e)}
        if ewald_parity is not None:
            try:
                ewald["parity"] = oracle_parity(grid_f64, ewald_parity,
                                                oracle_specs(batch, range(len(ewald_parity)), cfg.shape), ewald=True)
            except Exception as e:
                ewald["parity"] = {"error": repr(e)}
        del grid_f64
        if batched_parity is not None:
            groups = []
            for grp in batched_parity:
                try:
                    v_np = synthetic.gaussian_sum_volume(grp["box"], grp["gaussians"], grp["volume_seed"],
                                                         sigma_range=(1.0, 3.0))
                    g64, _ = O.fourier_voxel_grid_from_real_voxel_grid(v_np, pad_scale=2.0)
                    b = synthetic.image_batch(4096, grp["batch_seed"])
                    r = oracle_parity(g64, grp["got"], oracle_specs(b, range(len(grp["got"])), (grp["box"],) * 2))
                    r["group"] = f"N={2 * grp['box']} -> {grp['box']}^2"
                    groups.append(r)
                    del g64
                except Exception as e:
                    groups.append({"error": repr(e)})
            batched["parity"] = {"groups": groups,
                                 "max_rel_l2": max((g.get("max_rel_l2", float("inf")) for g in groups),
                                                   default=None)}
        parity["max_rel_l2_per_leg"] = {
            "headline": parity["headline"].get("max_rel_l2"),
            "batched_uneven": (batched or {}).get("parity", {}).get("max_rel_l2"),
            "spline": ((spline or {}).get("parity") or {}).get("max_rel_l2"),
            "ewald": ((ewald or {}).get("parity") or {}).get("max_rel_l2")}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Gaussian-sum volume and poses)",
            "config": config_dict(args, world),
            "roofline": {"bound": "hbm", "kernel": top_name, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak, "traffic": (trf * images_per_launch if trf else None),
                         "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": alg * images_per_launch,
                         "gather_distinct_voxels_per_image": gather_voxels,
                         "avg_launch_ms": top_ms / top_count, "launches_per_step": top_count,
                         # DRAM bytes the kernel actually moves (ncu, scaled per launch) over its live launch
                         # time: how close it runs to the HBM bandwidth it is bound by
                         "traffic_gbs": ((trf * images_per_launch) / (top_ms / top_count) / 1e6 if trf else None),
                         "traffic_frac": ((trf * images_per_launch) / (top_ms / top_count) / 1e6 / hbm_peak
                                          if trf else None),
                         # the unit ncu finds closest to its peak for this kernel (not HBM for the fused pass)
                         "limiter": ncu_limiter(top_name)},
            "l2": l2,
            "kernels_per_step": {k: {"launches": c, "ms": ms} for k, (c, ms) in prof.items()},
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clk,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "parity": parity,
            "batched_uneven": batched,
            "gradient": gradient,
            "pose_search": pose_search,
            "search_refine": search_refine,
            "spline": spline,
            "ewald": ewald,
            "relion_stack": relion_stack,
            "render": render,
        }
        print(json.dumps(line))
    replicas.shutdown(info)
    return 0


if __name__ == "__main__":
    sys.exit(main())
