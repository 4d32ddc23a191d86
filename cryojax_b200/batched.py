"""Batches that mix volumes and image shapes, an autotuner, CUDA graphs.

``BatchedSimulator`` takes several image models.  Each model is one group:
its own volume, image shape and batched poses / CTFs.  All groups run
through one ``cjx_slice_ctf_forward_multi`` call, and that call can be
captured once into a CUDA graph and replayed as a single launch.  In the
reference each distinct volume size or image shape is a separate
``eqx.filter_vmap`` trace (cryojax/simulator/_image_model/base_image_model.py:68-105
under ``eqx.filter_jit``).

``autotune`` picks the gather kernel's choices (ILP, lane tile) and the
workspace chunk size for one (volume side, image shape, flags) by timing
the candidates on a sample of the caller's images.  Each candidate carries
its choices in its own call (a group record and the descriptor), so tuning
never changes process-wide state and other threads can simulate meanwhile.
The result is cached in a JSON file keyed by GPU name and shape.
"""

from __future__ import annotations

import json
import os
import threading

import numpy as np

from . import _native as nat

_CACHE_LOCK = threading.Lock()
DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "cryojax_b200", "autotune.json")


def _cache_path():
    return os.environ.get("CRYOJAX_B200_AUTOTUNE_CACHE", DEFAULT_CACHE)


def _load_cache(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store_cache(path, cache):
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # a read-only home is not an error: the tuning just is not kept


def _key(n, py, px, flags):
    import torch

    name = torch.cuda.get_device_name().replace(" ", "_")
    return f"{name}|N{n}|P{py}x{px}|f{flags}"


CANDIDATES = [
    {"ilp": ilp, "tile": tile, "chunk_mb": chunk}
    for ilp in (1, 2, 4)
    for tile in (0, 1, 2)
    for chunk in (512, 1024)
]


def autotune(model, *, n_sample=1024, repeats=2, candidates=None, use_cache=True, cache_path=None):
    """Best {"ilp", "tile", "chunk_mb"} for this model's volume side and image shape."""
    import torch

    vol = model.volume_parametrization
    cfg = model.image_config
    integ = model.volume_integrator
    grid, layout = integ.device_grid(vol)
    flags = model._flags() | integ._base_flags() | layout
    n = vol.shape[0]
    py, px = cfg.padded_shape
    key = _key(n, py, px, flags)
    path = cache_path or _cache_path()
    if use_cache:
        with _CACHE_LOCK:
            hit = _load_cache(path).get(key)
        if hit:
            return hit
    params = model.image_params()
    m = min(n_sample, params.shape[0])
    pd = torch.as_tensor(params[:m], device=vol.device)
    out = torch.empty((m, py, px // 2 + 1), dtype=torch.complex64, device=pd.device)
    per_image = nat.workspace_size(nat.make_desc(n, py, px, flags, integ.fill_value, 1), 1)
    best, best_ms = None, float("inf")
    # each candidate runs through the multi-group entry point with its kernel choices in the group record
    # and its chunk in the descriptor: the process-wide knobs are never touched, so forward calls on other
    # threads meanwhile keep their own settings
    for c in candidates or CANDIDATES:
        chunk = max(1, min(m, (c["chunk_mb"] << 20) // max(per_image, 1)))
        desc = nat.make_desc(n, py, px, flags, integ.fill_value, chunk)
        groups = nat.make_groups([{"desc": desc, "grid": grid, "params": pd, "order": None, "out": out,
                                   "n_images": m, "tuning": {"ilp": c["ilp"], "tile": c["tile"]}}])
        ws = nat.multi_workspace_size(groups)
        wsb = torch.empty(max(ws, 1), dtype=torch.uint8, device=pd.device)
        nat.slice_ctf_forward_multi(groups, wsb)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(repeats):
            nat.slice_ctf_forward_multi(groups, wsb)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / repeats
        if ms < best_ms:
            best, best_ms = dict(c), ms
        del wsb
    best["ms_per_image"] = best_ms / m
    if use_cache:
        with _CACHE_LOCK:
            cache = _load_cache(path)
            cache[key] = best
            _store_cache(path, cache)
    return best


class BatchedSimulator:
    """Fourier images for several image-model groups in one library call.

    Parameters and processing orders are uploaded once.  Outputs
    (``outputs[i]``: complex64 [n_i, Py_i, Px_i//2+1]) and the shared
    workspace are allocated once.  ``run()`` launches everything on the
    current stream; ``capture()`` records that call into a CUDA graph that
    ``replay()`` launches as one unit.
    """

    def __init__(self, models, *, sort_orientations=True, tuning="auto", autotune_kw=None):
        import torch

        from .simulator import orientation_order

        self.torch = torch
        self.models = list(models)
        self.outputs = []
        self._keep = []
        groups = []
        for model in self.models:
            vol = model.volume_parametrization
            cfg = model.image_config
            integ = model.volume_integrator
            grid, layout = integ.device_grid(vol)
            flags = model._flags() | integ._base_flags() | layout
            params = model.image_params()
            dev = grid.device
            pd = torch.as_tensor(params, device=dev)
            order = None
            if sort_orientations:
                order = torch.as_tensor(orientation_order(params[:, 0:9].reshape(-1, 3, 3)), device=dev)
            py, px = cfg.padded_shape
            out = torch.empty((params.shape[0], py, px // 2 + 1), dtype=torch.complex64, device=dev)
            tun = None
            chunk = 0
            if tuning == "auto":
                t = autotune(model, **(autotune_kw or {}))
                tun = {"ilp": t["ilp"], "tile": t["tile"]}
                per = nat.workspace_size(nat.make_desc(vol.shape[0], py, px, flags, integ.fill_value, 1), 1)
                chunk = max(1, (t["chunk_mb"] << 20) // max(per, 1))
            elif isinstance(tuning, dict):
                tun = tuning
            desc = nat.make_desc(vol.shape[0], py, px, flags, integ.fill_value, chunk)
            groups.append({"desc": desc, "grid": grid, "params": pd, "order": order, "out": out,
                           "n_images": params.shape[0], "tuning": tun})
            self.outputs.append(out)
            self._keep += [grid, pd, order]
        self._groups = nat.make_groups(groups)
        ws = nat.multi_workspace_size(self._groups)
        self.workspace = torch.empty(max(ws, 1), dtype=torch.uint8, device=self.outputs[0].device)
        self.graph = None

    @property
    def n_images(self):
        return sum(int(o.shape[0]) for o in self.outputs)

    def run(self, stream=None):
        nat.slice_ctf_forward_multi(self._groups, self.workspace, stream)
        return self.outputs

    def capture(self):
        torch = self.torch
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            self.run()  # warm-up outside the graph (sets kernel attributes)
        torch.cuda.current_stream().wait_stream(side)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.run()
        self.graph = g
        return g

    def replay(self):
        if self.graph is None:
            self.capture()
        self.graph.replay()
        return self.outputs
