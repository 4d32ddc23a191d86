"""Orientation search on the device: simulate every candidate pose with the
image's own CTF and keep the best normalised cross-correlation.

In the reference a pose search is ``run_grid_search(fn, MinimumSearchMethod,
grid, args)``: fn simulates the image at one grid point and returns a cost,
and the method keeps an elementwise running argmin with the earliest index
winning ties (cryojax/jax_util/_grid_search/search_loop.py:24-158,
search_method.py:149-310).  Here fn is fixed to "simulate with this image's
CTF and shifts, score by NCC against the observed image" and the whole
(image x orientation) sweep is one C-ABI call (cjx_search): candidate
simulation through the same gather / resize kernels as the forward, and a
scoring pass that replaces the final column FFT's store by the two NCC sums.

The score is Pearson's r between the simulated and observed real-space
images -- the mean of normalize_image(sim) * normalize_image(obs)
(cryojax/ndimage/_normalize.py:11-28) -- computed in Fourier space by
Parseval with the DC term left out.  It needs padded_shape == shape, so that
the real-space image is the whole padded image.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _native as nat
from .gradients import observed_to_fourier


def _torch():
    import torch

    return torch


@dataclass
class SearchResult:
    best_orientation: np.ndarray   # (n,) int64, index into the rotation table
    best_score: np.ndarray         # (n,) float32, NCC of the best orientation
    scores: object = None          # (n, K) float32 CUDA tensor when requested
    candidates: object = None      # (n, K) int32 CUDA tensor of the orientations scored


class PoseSearch:
    """Exhaustive or candidate-list orientation search over a fixed rotation table.

    ``rotations``: (T, 3, 3) rotation matrices (the grid's orientations, e.g.
    ``healpix.OrientationGrid(8, 48).rotation_matrices()``), uploaded once.
    ``image_model``: a batched LinearImageModel / ContrastImageModel over the
    observed images; its CTF, scale and in-plane offsets are used per image,
    its pose rotation is replaced by every candidate's.
    """

    def __init__(self, rotations, *, device="cuda"):
        torch = _torch()
        r = np.ascontiguousarray(np.asarray(rotations, np.float64).reshape(-1, 9))
        self.n_orientations = r.shape[0]
        self.rotations = torch.as_tensor(r, device=device)
        self._ws = None

    def _desc(self, image_model, n, k):
        cfg = image_model.image_config
        if tuple(cfg.padded_shape) != tuple(cfg.shape):
            raise NotImplementedError("the NCC search needs padded_shape == shape")
        integ = image_model.volume_integrator
        vol = image_model.volume_parametrization.get_representation()
        grid, layout = integ.device_grid(vol)
        flags = image_model._flags() | integ._base_flags() | layout
        py, px = cfg.padded_shape
        sdesc = nat.SearchDesc()
        sdesc.slice = nat.make_desc(vol.shape[0], py, px, flags, integ.fill_value)
        sdesc.n_images = n
        sdesc.n_orientations = self.n_orientations
        sdesc.candidates_per_image = k
        return sdesc, grid

    def run(self, image_model, observed, *, candidates=None, return_scores=False, observed_is_fourier=False,
            image_params_device=None, stream=None) -> SearchResult:
        """Best orientation per observed image.

        observed: real-space images (n, P, P) in cryoJAX's centred convention,
        or their rfftn (complex64 (n, P, P//2+1) on the device) when
        ``observed_is_fourier``.  candidates: optional (n, K) orientation
        indices to score per image (each in [0, T)); default every
        orientation.
        """
        torch = _torch()
        dev = self.rotations.device
        params = image_model.image_params() if image_params_device is None else None
        n = image_params_device.shape[0] if image_params_device is not None else params.shape[0]
        obs_f = observed if observed_is_fourier else observed_to_fourier(observed)
        py, px = image_model.image_config.padded_shape
        if tuple(obs_f.shape) != (n, py, px // 2 + 1):
            raise ValueError(f"observed has shape {tuple(obs_f.shape)}, expected {(n, py, px // 2 + 1)} "
                             "in Fourier space")
        cand = None
        k = 0
        if candidates is not None:
            cand = candidates if isinstance(candidates, torch.Tensor) else torch.as_tensor(
                np.asarray(candidates, np.int32))
            cand = cand.to(device=dev, dtype=torch.int32).reshape(n, -1).contiguous()
            k = cand.shape[1]
            if k == 0:
                raise ValueError("candidates must list at least one orientation per image")
            lo, hi = int(cand.min()), int(cand.max())
            if lo < 0 or hi >= self.n_orientations:
                raise ValueError(f"candidate orientation indices must lie in [0, {self.n_orientations})")
        sdesc, grid = self._desc(image_model, n, k)
        pd = image_params_device if image_params_device is not None else torch.as_tensor(params, device=dev)
        ws_bytes = nat.search_workspace_size(sdesc)
        if self._ws is None or self._ws.numel() < ws_bytes:
            self._ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=dev)
        kk = k if k else self.n_orientations
        scores = torch.empty((n, kk), dtype=torch.float32, device=dev) if return_scores else None
        best_score = torch.empty(n, dtype=torch.float32, device=dev)
        best_orient = torch.empty(n, dtype=torch.int32, device=dev)
        nat.search(sdesc, grid, pd, self.rotations, obs_f, best_score, best_orient, self._ws,
                   candidates=cand, scores=scores, stream=stream)
        return SearchResult(best_orient.cpu().numpy().astype(np.int64), best_score.cpu().numpy(), scores, cand)


def search_orientations(image_model, observed, rotations, **kw) -> SearchResult:
    """One-shot exhaustive / candidate search (see PoseSearch.run)."""
    return PoseSearch(rotations).run(image_model, observed, **kw)


@dataclass
class LearnedSearchResult:
    best_orientation: np.ndarray   # (n,) int64
    best_score: np.ndarray         # (n,) float32
    fallback: np.ndarray           # (n,) bool: the exhaustive grid search decided this image
    proposed_directions: object    # (n, k) int32 CUDA tensor, the network's top-k directions


class LearnedPoseSearch:
    """Network-proposed candidates rescored by the grid search's scorer, exhaustive fallback.

    For each observed image the pose-proposal network ranks the grid's
    HEALPix directions; the top ``top_k`` directions x every in-plane angle
    are simulated and scored exactly as in the exhaustive search
    (PoseSearch with a candidate list), and images whose best score falls
    below ``threshold`` are searched exhaustively.  The exhaustive grid
    search therefore stays both the fallback and the scorer of every result.
    """

    def __init__(self, net, grid, *, top_k=16, threshold=float("-inf"), search: PoseSearch | None = None,
                 templates: "TemplateSharingSearch | None" = None, rerank_top=8,
                 fallback_search: "TemplateSharingSearch | None" = None):
        if net.n_classes != grid.n_dir:
            raise ValueError("the network's classes must be the grid's directions")
        self.net = net
        self.grid = grid
        self.top_k = top_k
        self.threshold = threshold
        self.search = search if search is not None else PoseSearch(grid.rotation_matrices())
        # with `templates` (a TemplateSharingSearch over the same grid) the proposed candidates are scored
        # from its CTF-free template rows and only the `rerank_top` best per image are simulated (FP32);
        # the fallback is then its exhaustive search with the same re-ranking
        self.templates = templates
        self.rerank_top = rerank_top
        # the exhaustive search of the fallback images: the template-sharing search (with the same FP32
        # re-ranking) when given or when the candidates are scored from templates, else PoseSearch
        self.fallback_search = fallback_search if fallback_search is not None else templates

    def run(self, image_model, observed, *, batch=None, fallback=True) -> LearnedSearchResult:
        """observed: real-space float32 CUDA images (n, P, P)."""
        torch = _torch()
        obs = observed if isinstance(observed, torch.Tensor) else torch.as_tensor(np.asarray(observed, np.float32))
        obs = obs.to(device=self.search.rotations.device, dtype=torch.float32).contiguous()
        obs_f = observed_to_fourier(obs)
        pd = torch.as_tensor(image_model.image_params(), device=obs.device)
        x = obs
        if obs.shape[-1] != self.net.image_size or obs.shape[-2] != self.net.image_size:
            x = torch.empty((obs.shape[0], self.net.image_size, self.net.image_size), dtype=torch.float32,
                            device=obs.device)
            nat.area_downsample(obs, x)  # the network's input size
        dirs, cand = self.net.propose(x, k=self.top_k, n_inplane=self.grid.n_inplane, batch=batch)
        if self.templates is not None:
            res = self.templates.run_directions(image_model, obs_f, dirs, self.grid.n_inplane,
                                                rerank_top=self.rerank_top, observed_is_fourier=True,
                                                image_params_device=pd)
        else:
            res = self.search.run(image_model, obs_f, candidates=cand, observed_is_fourier=True,
                                  image_params_device=pd)
        best, score = res.best_orientation.copy(), res.best_score.copy()
        low = score < self.threshold
        if fallback and low.any():
            idx = torch.as_tensor(np.flatnonzero(low), device=obs.device)
            sub_obs, sub_pd = obs_f.index_select(0, idx).contiguous(), pd.index_select(0, idx).contiguous()
            if self.fallback_search is not None:
                ex = self.fallback_search.run(image_model, sub_obs, observed_is_fourier=True,
                                              image_params_device=sub_pd, rerank_top=self.rerank_top)
            else:
                ex = self.search.run(image_model, sub_obs, observed_is_fourier=True, image_params_device=sub_pd)
            best[low] = ex.best_orientation
            score[low] = ex.best_score
        return LearnedSearchResult(best, score, low if fallback else np.zeros_like(low), dirs)

    def calibrate_threshold(self, image_model, observed, exhaustive_best, *, target_agreement=0.995,
                            min_fallback_fraction=0.02):
        """Fallback threshold from calibration images whose exhaustive optimum is known.

        Runs the learned search without fallback on the calibration images.
        Images that disagree with the exhaustive optimum need the fallback,
        so the threshold is set just above the best score of the disagreeing
        images, allowing (1 - target_agreement) of the set to disagree above
        it.  The threshold is never below the ``min_fallback_fraction``
        quantile of the calibration images' best scores: when (almost) no
        calibration image disagrees, the least confident images still fall
        back, so the fallback stays live on images unlike the calibration
        set.  Sets and returns ``self.threshold`` (always finite).
        """
        res = self.run(image_model, observed, fallback=False)
        wrong = res.best_orientation != np.asarray(exhaustive_best)
        allowed = int(np.floor((1.0 - target_agreement) * len(wrong)))
        s = np.sort(res.best_score[wrong])[::-1]
        floor = float(np.quantile(res.best_score, min_fallback_fraction)) if min_fallback_fraction > 0 else -np.inf
        thr = float(np.nextafter(np.float32(s[allowed]), np.float32(np.inf))) if len(s) > allowed else -np.inf
        self.threshold = max(thr, floor)
        if not np.isfinite(self.threshold):  # min_fallback_fraction = 0 and nothing disagreed
            self.threshold = float(np.min(res.best_score))
        return self.threshold


class TemplateSharingSearch:
    """Exhaustive NCC search through CTF-free templates shared by all images.

    Each orientation's central slice is simulated once without CTF; every
    image's CTF (and shifts, envelope, scale) moves onto its observed image,
    and the numerator and denominator of all (image, orientation) NCCs are
    two FP16 tensor-core GEMMs (see cjx_pack_templates / cjx_pack_observed /
    cjx_ncc_argmax).  Exact in real arithmetic; FP16 operands make the scores
    approximate (about 1e-3 relative), so near-ties may resolve differently
    from PoseSearch.  Needs padded_shape == shape and Py a multiple of 8.

    ``rerank`` chooses how the ``rerank_top`` best FP16 candidates of each
    image are rescored in FP32: ``"bank"`` (default) from the templates' own
    FP32 simulations, kept as a bank beside the FP16 rows (T Py (Px/2+1)
    complex64, 2.4 GB at 128^2 for 36,864 orientations), the same NCC as
    PoseSearch's up to FP32 rounding; ``"simulate"`` by PoseSearch with
    candidate lists, which simulates each candidate again and returns its
    scores bit for bit.
    """

    def __init__(self, rotations, *, device="cuda", template_chunk=4096, image_chunk=4096, rerank="bank"):
        torch = _torch()
        if rerank not in ("bank", "simulate"):
            raise ValueError("rerank must be 'bank' or 'simulate'")
        self.rot = np.ascontiguousarray(np.asarray(rotations, np.float64).reshape(-1, 9))
        self.n_orientations = self.rot.shape[0]
        self.device = torch.device(device)
        self.template_chunk = template_chunk
        self.image_chunk = image_chunk
        self.rerank = rerank
        self.s16 = self.p16 = self.t32 = None
        self._key = None

    def build_templates(self, image_model):
        """Simulate and pack the CTF-free templates of every orientation (cached per volume and shape)."""
        torch = _torch()
        from .constants import wavelength_from_kilovolts

        cfg = image_model.image_config
        if tuple(cfg.padded_shape) != tuple(cfg.shape):
            raise NotImplementedError("the NCC search needs padded_shape == shape")
        vol = image_model.volume_parametrization.get_representation()
        py, px = cfg.padded_shape
        if py % 8:
            raise NotImplementedError("TemplateSharingSearch needs Py to be a multiple of 8")
        integ = image_model.volume_integrator
        if not integ.is_projection_approximation:
            # the Ewald contrast pairs +q with -q, so the CTF cannot be moved onto the observed image
            raise NotImplementedError("TemplateSharingSearch needs a projection integrator; use PoseSearch")
        key = (id(integ.device_grid(vol)[0]), py, px, float(np.ravel(cfg.pixel_size)[0]))
        if key == self._key and self.s16 is not None:
            return
        kp = py * (px // 2 + 1)
        T = self.n_orientations
        if self.s16 is None or tuple(self.s16.shape) != (T, 2 * kp):  # a rebuild reuses the buffers
            self.s16 = self.p16 = None
            self.s16 = torch.empty((T, 2 * kp), dtype=torch.float16, device=self.device)
            self.p16 = torch.empty((T, kp), dtype=torch.float16, device=self.device)
        integ = image_model.volume_integrator
        p = nat.empty_params(T)
        p[:, 0:9] = self.rot
        p[:, nat.P_PIXEL_SIZE] = float(np.ravel(cfg.pixel_size)[0])
        p[:, nat.P_WAVELENGTH] = wavelength_from_kilovolts(float(np.ravel(cfg.voltage_in_kilovolts)[0]))
        p[:, nat.P_SCALE] = 1.0
        pd = torch.as_tensor(p, device=self.device)
        tc = min(self.template_chunk, T)
        if self.rerank == "bank":  # the simulations themselves are the FP32 bank
            if self.t32 is None or tuple(self.t32.shape) != (T, py, px // 2 + 1):
                self.t32 = None
                self.t32 = torch.empty((T, py, px // 2 + 1), dtype=torch.complex64, device=self.device)
            buf = None
        else:
            buf = torch.empty((tc, py, px // 2 + 1), dtype=torch.complex64, device=self.device)
        ws = None
        for s in range(0, T, tc):
            e = min(T, s + tc)
            out = self.t32[s:e] if buf is None else buf[:e - s]
            integ.run(vol, cfg, None, 0, params_device=pd[s:e], out=out, workspace=ws, n=e - s)
            nat.pack_templates(out, py, px, self.s16[s:e], self.p16[s:e])
        self._key = key

    def _pack_observed(self, image_model, obs_f, pd):
        torch = _torch()
        cfg = image_model.image_config
        py, px = cfg.padded_shape
        kp = py * (px // 2 + 1)
        n = obs_f.shape[0]
        dev = self.device
        y16 = torch.empty((n, 2 * kp), dtype=torch.float16, device=dev)
        z16 = torch.empty((n, kp), dtype=torch.float16, device=dev)
        oo, yinv, zinv = (torch.empty(n, dtype=torch.float32, device=dev) for _ in range(3))
        nat.pack_observed(obs_f, pd, py, px, image_model._flags(), y16, z16, oo, yinv, zinv)
        return y16, z16, oo, yinv, zinv

    def _rerank(self, image_model, obs_f, pd, top):
        """FP32 best of the (n, m) template indices `top` per image: from the FP32 bank, or by PoseSearch with
        candidate lists."""
        if self.rerank == "bank" and self.t32 is not None:
            torch = _torch()
            cfg = image_model.image_config
            py, px = cfg.padded_shape
            n = obs_f.shape[0]
            dev = self.device
            best_score = torch.empty(n, dtype=torch.float32, device=dev)
            best = torch.empty(n, dtype=torch.int32, device=dev)
            mc = min(self.image_chunk, n)
            y32 = torch.empty((mc, py, px // 2 + 1), dtype=torch.complex64, device=dev)
            z32 = torch.empty((mc, py, px // 2 + 1), dtype=torch.float32, device=dev)
            oo = torch.empty(mc, dtype=torch.float32, device=dev)
            for s in range(0, n, mc):
                e = min(n, s + mc)
                nat.pack_observed32(obs_f[s:e], pd[s:e], py, px, image_model._flags(), y32, z32, oo)
                nat.ncc_rerank32(self.t32, py, px, y32, z32, oo, top[s:e], best_score[s:e], best[s:e])
            return SearchResult(best.cpu().numpy().astype(np.int64), best_score.cpu().numpy(), None, top)
        if getattr(self, "_plain", None) is None:
            self._plain = PoseSearch(self.rot, device=self.device)
        return self._plain.run(image_model, obs_f, candidates=top, observed_is_fourier=True, image_params_device=pd)

    def run_directions(self, image_model, observed, dirs, n_inplane, *, rerank_top=8, observed_is_fourier=False,
                       image_params_device=None) -> SearchResult:
        """Best orientation per image among its proposed directions' templates, with no simulation.

        ``dirs`` (n, kd) int32 CUDA: each image's proposed directions; template t = dir * n_inplane + a
        (the orientation grid's order).  Every candidate is scored from the FP16 template rows
        (cjx_ncc_directions), the ``rerank_top`` best of each image are rescored by the FP32 scorer
        (PoseSearch with candidate lists) and the best of those is returned: the candidate set's FP32
        optimum whenever it is among them.
        """
        torch = _torch()
        if not 1 <= rerank_top <= 16:
            raise ValueError("rerank_top must be in [1, 16]")
        self.build_templates(image_model)
        cfg = image_model.image_config
        py, px = cfg.padded_shape
        kp = py * (px // 2 + 1)
        obs_f = observed if observed_is_fourier else observed_to_fourier(observed)
        n = obs_f.shape[0]
        pd = image_params_device if image_params_device is not None else torch.as_tensor(
            image_model.image_params(), device=self.device)
        dirs = dirs.to(device=self.device, dtype=torch.int32).contiguous()
        kd = dirs.shape[1]
        K = kd * n_inplane
        if self.n_orientations % n_inplane:
            raise ValueError("the template count must be a multiple of n_inplane")
        n_dir = self.n_orientations // n_inplane
        y16, z16, oo, yinv, zinv = self._pack_observed(image_model, obs_f, pd)
        num = torch.empty((n, K), dtype=torch.float32, device=self.device)
        den = torch.empty((n, K), dtype=torch.float32, device=self.device)
        ws = torch.empty(nat.ncc_directions_workspace_size(n, kd, n_dir), dtype=torch.uint8, device=self.device)
        nat.ncc_directions(y16, z16, self.s16, self.p16, kp, dirs, n_dir, n_inplane, num, den, ws)
        m = min(rerank_top, K)
        pos = torch.empty((n, m), dtype=torch.int32, device=self.device)
        nat.ncc_topk(num, den, n, K, oo, yinv, zinv, m, pos)
        # position k n_inplane + a -> template dirs[b][k] n_inplane + a
        pos64 = pos.long()
        top = (dirs.long().gather(1, pos64 // n_inplane) * n_inplane + pos64 % n_inplane).to(torch.int32)
        exact = self._rerank(image_model, obs_f, pd, top.contiguous())
        return SearchResult(exact.best_orientation, exact.best_score, None, top)

    def run(self, image_model, observed, *, observed_is_fourier=False, image_params_device=None,
            return_scores=False, rerank_top=0) -> SearchResult:
        """Best orientation per image; with ``rerank_top`` = k (<= 16) the k best FP16 candidates of
        each image are rescored by the FP32 scorer (PoseSearch with candidate lists) and the best of
        those is returned, which is the exhaustive FP32 answer whenever it is among them."""
        torch = _torch()
        if rerank_top < 0 or rerank_top > 16:
            raise ValueError("rerank_top must be in [0, 16]")
        self.build_templates(image_model)
        cfg = image_model.image_config
        py, px = cfg.padded_shape
        kp = py * (px // 2 + 1)
        obs_f = observed if observed_is_fourier else observed_to_fourier(observed)
        n = obs_f.shape[0]
        pd = image_params_device if image_params_device is not None else torch.as_tensor(
            image_model.image_params(), device=self.device)
        T = self.n_orientations
        dev = self.device
        y16, z16, oo, yinv, zinv = self._pack_observed(image_model, obs_f, pd)
        best_score = torch.empty(n, dtype=torch.float32, device=dev)
        best = torch.empty(n, dtype=torch.int32, device=dev)
        scores = torch.empty((n, T), dtype=torch.float32, device=dev) if return_scores else None
        top = torch.empty((n, rerank_top), dtype=torch.int32, device=dev) if rerank_top else None
        mc = min(self.image_chunk, n)
        num = torch.empty((mc, T), dtype=torch.float32, device=dev)
        den = torch.empty((mc, T), dtype=torch.float32, device=dev)
        for s in range(0, n, mc):
            e = min(n, s + mc)
            m = e - s
            nat.gemm(y16[s:e], self.s16, num, m=m, n=T, k=2 * kp, flags=nat.CJX_GEMM_F16)
            nat.gemm(z16[s:e], self.p16, den, m=m, n=T, k=kp, flags=nat.CJX_GEMM_F16)
            nat.ncc_argmax(num, den, m, T, oo[s:e], yinv[s:e], zinv[s:e], best_score[s:e], best[s:e],
                           scores=None if scores is None else scores[s:e])
            if top is not None:
                nat.ncc_topk(num, den, m, T, oo[s:e], yinv[s:e], zinv[s:e], rerank_top, top[s:e])
        if top is None:
            return SearchResult(best.cpu().numpy().astype(np.int64), best_score.cpu().numpy(), scores, None)
        exact = self._rerank(image_model, obs_f, pd, top)
        return SearchResult(exact.best_orientation, exact.best_score, scores, top)
