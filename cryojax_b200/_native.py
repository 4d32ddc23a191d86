"""ctypes binding of libcryojax_b200.so (the C-ABI in include/cryojax_b200.h).

The library is the product: there is no CPU fallback.  Loading fails loudly
when the shared library is missing; calls fail loudly when a tensor is not
on a CUDA device.
"""

from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

from .build import LIB_PATH

# ---- constants mirrored from include/cryojax_b200.h ----------------------
CJX_OK = 0
CJX_ERR_INVALID_ARGUMENT = 1
CJX_ERR_UNSUPPORTED = 2
CJX_ERR_CUDA = 3
CJX_ERR_WORKSPACE = 4

CJX_APPLY_CTF = 1 << 0
CJX_APPLY_TRANSLATION = 1 << 1
CJX_APPLY_ENVELOPE = 1 << 2
CJX_ZERO_FILL_NEGATIVE = 1 << 3
CJX_GRID_BRICKED = 1 << 4
CJX_GRID_BRICKED_PAIRS = 1 << 5
CJX_GRID_SPLINE = 1 << 6
CJX_EWALD_SPHERE = 1 << 7

CJX_MAX_SIDE = 1024
CJX_TUNE_GATHER_ILP = 1
CJX_TUNE_CHUNK_BYTES = 2
CJX_TUNE_GATHER_MODE = 3
CJX_TUNE_FFT_MODE = 4
CJX_TUNE_GATHER_TILE = 5
CJX_TUNE_SCATTER_VEC = 6
CJX_TUNE_SPLINE_ILP = 7
CJX_TUNE_MULTI_WAVES = 9
PARAMS_DOUBLES = 32  # sizeof(cjx_image_params) / 8

# field offsets (in doubles) of cjx_image_params
P_ROT = 0
P_SHIFT_X = 9
P_SHIFT_Y = 10
P_DEFOCUS = 11
P_ASTIG = 12
P_ASTIG_ANGLE = 13
P_CS = 14
P_WAVELENGTH = 15
P_PHASE_TOTAL = 16
P_PIXEL_SIZE = 17
P_SCALE = 18
P_ENV_AMP = 19
P_ENV_B = 20
P_AC = 21
P_PHASE_SHIFT = 22


CJX_RENDER_ACCUMULATE = 1
CJX_RENDER_MAX_GAUSSIANS = 8


class RenderDesc(ctypes.Structure):
    _fields_ = [
        ("nz", ctypes.c_int32),
        ("ny", ctypes.c_int32),
        ("nx", ctypes.c_int32),
        ("n_gaussians", ctypes.c_int32),
        ("voxel_size", ctypes.c_float),
        ("cutoff_sigmas", ctypes.c_float),
        ("flags", ctypes.c_uint32),
        ("reserved", ctypes.c_int32),
    ]


class SliceDesc(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int32),
        ("py", ctypes.c_int32),
        ("px", ctypes.c_int32),
        ("flags", ctypes.c_uint32),
        ("fill_re", ctypes.c_float),
        ("fill_im", ctypes.c_float),
        ("images_per_chunk", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class SliceGroup(ctypes.Structure):
    _fields_ = [
        ("desc", SliceDesc),
        ("grid", ctypes.c_void_p),
        ("params", ctypes.c_void_p),
        ("order", ctypes.c_void_p),
        ("out", ctypes.c_void_p),
        ("n_images", ctypes.c_int64),
        ("tuning_valid", ctypes.c_int32),
        ("gather_ilp", ctypes.c_int32),
        ("gather_tile", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class SearchDesc(ctypes.Structure):
    _fields_ = [
        ("slice", SliceDesc),
        ("n_images", ctypes.c_int64),
        ("n_orientations", ctypes.c_int64),
        ("candidates_per_image", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class CryojaxB200Error(RuntimeError):
    """Raised when a C-ABI entry point returns a nonzero status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"cryojax_b200 error {code}: {message}")
        self.code = code


# Every exported symbol of include/cryojax_b200.h with (restype, argtypes).
_SIGNATURES = {
    "cjx_get_version": (ctypes.c_int, []),
    "cjx_spline_coefficients_workspace_size": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]),
    "cjx_render_gaussians": (
        ctypes.c_int,
        [ctypes.POINTER(RenderDesc), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
         ctypes.c_void_p, ctypes.c_void_p],
    ),
    "cjx_spline_coefficients": (
        ctypes.c_int,
        [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p],
    ),
    "cjx_get_last_error": (ctypes.c_char_p, []),
    "cjx_slice_ctf_workspace_size": (
        ctypes.c_int,
        [ctypes.POINTER(SliceDesc), ctypes.c_int64, ctypes.POINTER(ctypes.c_size_t)],
    ),
    "cjx_slice_ctf_forward": (
        ctypes.c_int,
        [
            ctypes.POINTER(SliceDesc),
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_int64,
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_size_t,
            ctypes.c_void_p,
        ],
    ),
    "cjx_slice_ctf_forward_filtered": (
        ctypes.c_int,
        [
            ctypes.POINTER(SliceDesc),
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_int64,
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_size_t,
            ctypes.c_void_p,
        ],
    ),
    "cjx_slice_ctf_loss_workspace_size": (
        ctypes.c_int,
        [ctypes.POINTER(SliceDesc), ctypes.c_int64, ctypes.POINTER(ctypes.c_size_t)],
    ),
    "cjx_slice_ctf_loss_grad": (
        ctypes.c_int,
        [
            ctypes.POINTER(SliceDesc),
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_int64,
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_size_t,
            ctypes.c_void_p,
        ],
    ),
    "cjx_search_workspace_size": (ctypes.c_int, [ctypes.POINTER(SearchDesc), ctypes.POINTER(ctypes.c_size_t)]),
    "cjx_search": (
        ctypes.c_int,
        [ctypes.POINTER(SearchDesc)] + [ctypes.c_void_p] * 9 + [ctypes.c_size_t, ctypes.c_void_p],
    ),
    "cjx_slice_ctf_multi_workspace_size": (
        ctypes.c_int,
        [ctypes.POINTER(SliceGroup), ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)],
    ),
    "cjx_slice_ctf_forward_multi": (
        ctypes.c_int,
        [ctypes.POINTER(SliceGroup), ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p],
    ),
    "cjx_slice_ctf_forward_noalloc": (
        ctypes.c_int,
        [
            ctypes.POINTER(SliceDesc),
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_void_p,
            ctypes.c_int64,
            ctypes.c_void_p,
            ctypes.c_void_p,
        ],
    ),
    "cjx_bricked_volume_size": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]),
    "cjx_brick_volume": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "cjx_fft_c2c": (
        ctypes.c_int,
        [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p],
    ),
    "cjx_postprocess_workspace_size": (
        ctypes.c_int, [ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]),
    "cjx_postprocess_real": (
        ctypes.c_int,
        [ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint32, ctypes.c_void_p,
         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p],
    ),
    "cjx_rfft2": (
        ctypes.c_int, [ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "cjx_tuning_set": (ctypes.c_int, [ctypes.c_int, ctypes.c_int64]),
    "cjx_tuning_get": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_int64)]),
    "cjx_brick_volume_pairs": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "cjx_gemm": (
        ctypes.c_int,
        [ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
         ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
         ctypes.c_void_p],
    ),
    "cjx_device_status": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_void_p]),
    "cjx_selftest_bounded_wait": (ctypes.c_int, [ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p]),
    "cjx_cnn_noisy_normalize": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_float,
         ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p],
    ),
    "cjx_area_downsample": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
         ctypes.c_void_p],
    ),
    "cjx_cnn_conv_s2": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int64,
         ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    ),
    "cjx_cnn_conv0": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int,
         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    ),
    "cjx_cnn_im2col": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int64,
         ctypes.c_void_p],
    ),
    "cjx_cnn_col2im": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
         ctypes.c_void_p, ctypes.c_void_p],
    ),
    "cjx_transpose_to_bf16": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p,
         ctypes.c_int64, ctypes.c_void_p],
    ),
    "cjx_relu_mask": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                     ctypes.c_void_p]),
    "cjx_colsum": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p,
         ctypes.c_void_p],
    ),
    "cjx_softmax_xent": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
         ctypes.c_float, ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    ),
    "cjx_adamw": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
         ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
         ctypes.c_int64, ctypes.c_void_p],
    ),
    "cjx_topk_candidates": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
         ctypes.c_void_p, ctypes.c_void_p],
    ),
    "cjx_pack_templates": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
         ctypes.c_void_p],
    ),
    "cjx_pack_observed": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    ),
    "cjx_ncc_argmax": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p,
         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
         ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p],
    ),
    "cjx_ncc_topk": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p,
         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p],
    ),
    "cjx_pack_observed32": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    ),
    "cjx_ncc_rerank32": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
         ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
         ctypes.c_void_p, ctypes.c_void_p],
    ),
    "cjx_ncc_directions_workspace_size": (
        ctypes.c_int, [ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]),
    "cjx_ncc_directions": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
         ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
         ctypes.c_size_t, ctypes.c_void_p],
    ),
    "cjx_probe_read_bandwidth": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p],
    ),
    "cjx_profile_enable": (ctypes.c_int, [ctypes.c_int]),
    "cjx_profile_read": (
        ctypes.c_int,
        [
            ctypes.c_char_p,
            ctypes.POINTER(ctypes.c_int64),
            ctypes.POINTER(ctypes.c_double),
            ctypes.c_int,
            ctypes.POINTER(ctypes.c_int),
        ],
    ),
}

_lib = None
_lock = threading.Lock()


def library_path() -> str:
    return os.environ.get("CRYOJAX_B200_LIB", LIB_PATH)


def load_library() -> ctypes.CDLL:
    """Load the shared library (once).  Raises if it has not been built."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = library_path()
        if not os.path.exists(path):
            raise ImportError(
                f"libcryojax_b200.so not found at {path}; build it with "
                "`python -m cryojax_b200.build` (there is no CPU fallback)"
            )
        lib = ctypes.CDLL(path)
        for name, (restype, argtypes) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = lib
        return lib


def exported_symbols() -> list[str]:
    return list(_SIGNATURES)


def _check(code: int) -> None:
    if code != CJX_OK:
        msg = load_library().cjx_get_last_error().decode(errors="replace")
        raise CryojaxB200Error(code, msg)


def make_desc(n, py, px, flags, fill_value=0j, images_per_chunk=0) -> SliceDesc:
    fill = complex(fill_value)
    return SliceDesc(int(n), int(py), int(px), int(flags), fill.real, fill.imag, int(images_per_chunk), 0)


def workspace_size(desc: SliceDesc, n_images: int) -> int:
    out = ctypes.c_size_t(0)
    _check(load_library().cjx_slice_ctf_workspace_size(ctypes.byref(desc), int(n_images), ctypes.byref(out)))
    return int(out.value)


def _cuda_ptr(t, what):
    if not t.is_cuda:
        raise ValueError(f"{what} must be a CUDA tensor (no CPU fallback)")
    if not t.is_contiguous():
        raise ValueError(f"{what} must be contiguous")
    return ctypes.c_void_p(t.data_ptr())


def _stream_ptr(stream):
    import torch

    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


def _order_ptr(order, n_images):
    import torch

    if order is None:
        return ctypes.c_void_p(0)
    if order.dtype != torch.int32 or order.numel() != n_images:
        raise ValueError("order must be an int32 permutation of length n_images")
    return _cuda_ptr(order, "order")


def slice_ctf_forward(desc: SliceDesc, grid, params, out, workspace=None, stream=None, order=None,
                      filter=None) -> None:
    """Launch cjx_slice_ctf_forward on torch CUDA tensors (stream-ordered).

    ``filter``: an optional float32 CUDA array with one image's output shape, multiplied into every
    output image inside the epilogue (cjx_slice_ctf_forward_filtered).
    """
    import torch

    n_images = params.shape[0]
    if params.dtype != torch.float64 or params.shape[-1] != PARAMS_DOUBLES:
        raise ValueError("params must be float64 [n_images, 32]")
    if grid.dtype != torch.complex64:
        raise ValueError("grid must be complex64")
    if out.dtype != torch.complex64:
        raise ValueError("out must be complex64")
    ws_ptr = ctypes.c_void_p(0)
    ws_bytes = 0
    if workspace is not None:
        ws_ptr = _cuda_ptr(workspace, "workspace")
        ws_bytes = workspace.numel() * workspace.element_size()
    if filter is not None:
        if filter.dtype != torch.float32 or tuple(filter.shape) != tuple(out.shape[-2:]):
            raise ValueError(f"filter must be float32 {tuple(out.shape[-2:])} (one output image's shape)")
        _check(
            load_library().cjx_slice_ctf_forward_filtered(
                ctypes.byref(desc), _cuda_ptr(grid, "grid"), _cuda_ptr(params, "params"),
                _order_ptr(order, n_images), int(n_images), _cuda_ptr(filter, "filter"), _cuda_ptr(out, "out"),
                ws_ptr, ws_bytes, _stream_ptr(stream)))
        return
    _check(
        load_library().cjx_slice_ctf_forward(
            ctypes.byref(desc),
            _cuda_ptr(grid, "grid"),
            _cuda_ptr(params, "params"),
            _order_ptr(order, n_images),
            int(n_images),
            _cuda_ptr(out, "out"),
            ws_ptr,
            ws_bytes,
            _stream_ptr(stream),
        )
    )


GRAD_DOUBLES = 16  # sizeof(cjx_image_grads) / 8
G_LOSS, G_TX, G_TY, G_DF, G_ROT = 0, 1, 2, 3, 4


def loss_workspace_size(desc: SliceDesc, n_images: int) -> int:
    out = ctypes.c_size_t(0)
    _check(load_library().cjx_slice_ctf_loss_workspace_size(ctypes.byref(desc), int(n_images), ctypes.byref(out)))
    return int(out.value)


def slice_ctf_loss_grad(desc: SliceDesc, grid, params, observed, image_grads, grid_grad=None, workspace=None,
                        stream=None, order=None) -> None:
    """cjx_slice_ctf_loss_grad on torch CUDA tensors."""
    import torch

    n = params.shape[0]
    if image_grads.dtype != torch.float64 or tuple(image_grads.shape) != (n, GRAD_DOUBLES):
        raise ValueError("image_grads must be float64 [n_images, 16]")
    if observed.dtype != torch.complex64:
        raise ValueError("observed must be complex64")
    gg = ctypes.c_void_p(0) if grid_grad is None else _cuda_ptr(grid_grad, "grid_grad")
    ws_ptr = _cuda_ptr(workspace, "workspace") if workspace is not None else ctypes.c_void_p(0)
    ws_bytes = workspace.numel() * workspace.element_size() if workspace is not None else 0
    _check(
        load_library().cjx_slice_ctf_loss_grad(
            ctypes.byref(desc), _cuda_ptr(grid, "grid"), _cuda_ptr(params, "params"), _order_ptr(order, n), int(n),
            _cuda_ptr(observed, "observed"), _cuda_ptr(image_grads, "image_grads"), gg, ws_ptr, ws_bytes,
            _stream_ptr(stream)))


def search_workspace_size(sdesc: SearchDesc) -> int:
    out = ctypes.c_size_t(0)
    _check(load_library().cjx_search_workspace_size(ctypes.byref(sdesc), ctypes.byref(out)))
    return int(out.value)


def search(sdesc: SearchDesc, grid, image_params, rotations, observed, best_score, best_orientation, workspace,
           candidates=None, scores=None, stream=None) -> None:
    """cjx_search on torch CUDA tensors."""
    def ptr(t, what):
        return ctypes.c_void_p(0) if t is None else _cuda_ptr(t, what)

    _check(load_library().cjx_search(
        ctypes.byref(sdesc), ptr(grid, "grid"), ptr(image_params, "image_params"), ptr(rotations, "rotations"),
        ptr(candidates, "candidates"), ptr(observed, "observed"), ptr(scores, "scores"),
        ptr(best_score, "best_score"), ptr(best_orientation, "best_orientation"), ptr(workspace, "workspace"),
        workspace.numel() * workspace.element_size(), _stream_ptr(stream)))


def make_groups(groups):
    """ctypes array of SliceGroup from dicts with desc, grid, params, order, out, tuning."""
    arr = (SliceGroup * len(groups))()
    for i, g in enumerate(groups):
        arr[i].desc = g["desc"]
        arr[i].grid = g["grid"].data_ptr() if g.get("grid") is not None else 0
        arr[i].params = g["params"].data_ptr() if g.get("params") is not None else 0
        arr[i].order = g["order"].data_ptr() if g.get("order") is not None else 0
        arr[i].out = g["out"].data_ptr() if g.get("out") is not None else 0
        arr[i].n_images = int(g["n_images"])
        tun = g.get("tuning")
        if tun:
            arr[i].tuning_valid = 1
            arr[i].gather_ilp = int(tun["ilp"])
            arr[i].gather_tile = int(tun["tile"])
    return arr


def multi_workspace_size(groups_arr) -> int:
    out = ctypes.c_size_t(0)
    _check(load_library().cjx_slice_ctf_multi_workspace_size(groups_arr, len(groups_arr), ctypes.byref(out)))
    return int(out.value)


def slice_ctf_forward_multi(groups_arr, workspace=None, stream=None) -> None:
    ws_ptr = ctypes.c_void_p(0)
    ws_bytes = 0
    if workspace is not None:
        ws_ptr = _cuda_ptr(workspace, "workspace")
        ws_bytes = workspace.numel() * workspace.element_size()
    _check(load_library().cjx_slice_ctf_forward_multi(groups_arr, len(groups_arr), ws_ptr, ws_bytes,
                                                      _stream_ptr(stream)))


NOALLOC_SCRATCH_BYTES = 32 << 20  # CJX_NOALLOC_SCRATCH_BYTES


def slice_ctf_forward_noalloc(desc: SliceDesc, grid, params, out, stream=None, order=None) -> None:
    """Launch cjx_slice_ctf_forward_noalloc (scratch inside the library, no allocation)."""
    import torch

    if params.dtype != torch.float64 or params.shape[-1] != PARAMS_DOUBLES:
        raise ValueError("params must be float64 [n_images, 32]")
    if grid.dtype != torch.complex64 or out.dtype != torch.complex64:
        raise ValueError("grid and out must be complex64")
    _check(
        load_library().cjx_slice_ctf_forward_noalloc(
            ctypes.byref(desc),
            _cuda_ptr(grid, "grid"),
            _cuda_ptr(params, "params"),
            _order_ptr(order, params.shape[0]),
            int(params.shape[0]),
            _cuda_ptr(out, "out"),
            _stream_ptr(stream),
        )
    )


CJX_GEMM_OUT_BF16 = 1
CJX_GEMM_BIAS = 2
CJX_GEMM_RELU = 4
CJX_GEMM_ACCUMULATE = 8
CJX_GEMM_F16 = 16


def gemm(a, b, c, *, bias=None, flags=0, split_k=1, m=None, n=None, k=None, stream=None) -> None:
    """cjx_gemm: c[:m, :n] (op)= a[:m, :k] @ b[:n, :k].T on torch CUDA tensors (row-major 2-D)."""
    for t, what in ((a, "a"), (b, "b"), (c, "c")):
        if t.dim() != 2:
            raise ValueError(f"gemm operand {what} must be a 2-D tensor (row pitch = stride(0))")
    m = a.shape[0] if m is None else m
    n = b.shape[0] if n is None else n
    k = a.shape[1] if k is None else k
    if bias is not None:
        flags |= CJX_GEMM_BIAS
    _check(load_library().cjx_gemm(
        int(m), int(n), int(k), _cuda_ptr(a, "a"), int(a.stride(0)), _cuda_ptr(b, "b"), int(b.stride(0)),
        _cuda_ptr(c, "c"), int(c.stride(0)), ctypes.c_void_p(0) if bias is None else _cuda_ptr(bias, "bias"),
        int(flags), int(split_k), _stream_ptr(stream)))


class ParamSegment(ctypes.Structure):
    _fields_ = [
        ("offset", ctypes.c_int64),
        ("count", ctypes.c_int64),
        ("cols", ctypes.c_int64),
        ("ldk", ctypes.c_int64),
        ("w_bf16", ctypes.c_void_p),
        ("wt_bf16", ctypes.c_void_p),
        ("weight_decay", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


def _opt_ptr(t, what):
    return ctypes.c_void_p(0) if t is None else _cuda_ptr(t, what)


def cnn_noisy_normalize(images, out, *, index=None, snr=0.0, seed=0, n=None, stream=None) -> None:
    n = out.shape[0] if n is None else n
    h, w = images.shape[-2], images.shape[-1]
    _check(load_library().cjx_cnn_noisy_normalize(
        _cuda_ptr(images, "images"), _opt_ptr(index, "index"), int(n), int(h), int(w), float(snr),
        ctypes.c_uint64(int(seed) & 0xFFFFFFFFFFFFFFFF), _cuda_ptr(out, "out"), _stream_ptr(stream)))


def area_downsample(src, dst, stream=None) -> None:
    """dst (n, h, w) FP32 = area-weighted downsample of src (n, H, W) FP32 (CUDA tensors)."""
    n, H, W = src.shape
    h, w = dst.shape[-2], dst.shape[-1]
    _check(load_library().cjx_area_downsample(_cuda_ptr(src, "src"), int(n), int(H), int(W), _cuda_ptr(dst, "dst"),
                                              int(h), int(w), _stream_ptr(stream)))


def cnn_im2col(x, B, H, W, C, col, ldk, stream=None) -> None:
    _check(load_library().cjx_cnn_im2col(_cuda_ptr(x, "x"), int(B), int(H), int(W), int(C), _cuda_ptr(col, "col"),
                                         int(ldk), _stream_ptr(stream)))


def cnn_conv0(x, B, H, W, w, ldk, cout, bias, y, stream=None) -> None:
    """cjx_cnn_conv0: first 3x3 stride-2 layer (one input channel) + bias + ReLU without im2col."""
    _check(load_library().cjx_cnn_conv0(_cuda_ptr(x, "x"), int(B), int(H), int(W), _cuda_ptr(w, "w"), int(ldk),
                                        int(cout), _opt_ptr(bias, "bias"), _cuda_ptr(y, "y"), _stream_ptr(stream)))


def cnn_conv_s2(x, B, H, W, C, w, ldk, cout, bias, y, stream=None) -> None:
    """cjx_cnn_conv_s2: a 3x3 stride-2 layer + bias + ReLU as an implicit GEMM on the tensor cores."""
    _check(load_library().cjx_cnn_conv_s2(_cuda_ptr(x, "x"), int(B), int(H), int(W), int(C), _cuda_ptr(w, "w"),
                                          int(ldk), int(cout), _opt_ptr(bias, "bias"), _cuda_ptr(y, "y"),
                                          _stream_ptr(stream)))


def cnn_col2im(dcol, ldk, act, B, H, W, C, dx, stream=None) -> None:
    _check(load_library().cjx_cnn_col2im(_cuda_ptr(dcol, "dcol"), int(ldk), _opt_ptr(act, "act"), int(B), int(H),
                                         int(W), int(C), _cuda_ptr(dx, "dx"), _stream_ptr(stream)))


def transpose_to_bf16(inp, rows, cols, ld_in, out, ld_out, stream=None) -> None:
    import torch

    _check(load_library().cjx_transpose_to_bf16(
        _cuda_ptr(inp, "in"), 1 if inp.dtype == torch.bfloat16 else 0, int(rows), int(cols), int(ld_in),
        _cuda_ptr(out, "out"), int(ld_out), _stream_ptr(stream)))


def relu_mask(grad, act, n, out, stream=None) -> None:
    _check(load_library().cjx_relu_mask(_cuda_ptr(grad, "grad"), _opt_ptr(act, "act"), int(n), _cuda_ptr(out, "out"),
                                        _stream_ptr(stream)))


def colsum(x, rows, cols, ld, out, stream=None) -> None:
    import torch

    _check(load_library().cjx_colsum(_cuda_ptr(x, "x"), 1 if x.dtype == torch.bfloat16 else 0, int(rows), int(cols),
                                     int(ld), _cuda_ptr(out, "out"), _stream_ptr(stream)))


def softmax_xent(logits, labels, *, neighbours=None, smoothing=0.0, grad_scale=1.0, loss=None, dlogits=None,
                 B=None, stream=None) -> None:
    B = logits.shape[0] if B is None else B
    n_nb = 0 if neighbours is None else neighbours.shape[1]
    _check(load_library().cjx_softmax_xent(
        _cuda_ptr(logits, "logits"), int(B), int(logits.shape[1]), _cuda_ptr(labels, "labels"),
        _opt_ptr(neighbours, "neighbours"), int(n_nb), float(smoothing), float(grad_scale), _opt_ptr(loss, "loss"),
        _opt_ptr(dlogits, "dlogits"), _stream_ptr(stream)))


def adamw(params, grads, m, v, segments, *, lr, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0, step,
          stream=None) -> None:
    _check(load_library().cjx_adamw(
        _cuda_ptr(params, "params"), _cuda_ptr(grads, "grads"), _cuda_ptr(m, "m"), _cuda_ptr(v, "v"),
        int(params.numel()), ctypes.cast(segments, ctypes.c_void_p), len(segments), float(lr), float(beta1),
        float(beta2), float(eps), float(weight_decay), int(step), _stream_ptr(stream)))


def topk_candidates(logits, k, n_inplane, *, dirs=None, candidates=None, B=None, stream=None) -> None:
    B = logits.shape[0] if B is None else B
    _check(load_library().cjx_topk_candidates(
        _cuda_ptr(logits, "logits"), int(B), int(logits.shape[1]), int(k), int(n_inplane), _opt_ptr(dirs, "dirs"),
        _opt_ptr(candidates, "candidates"), _stream_ptr(stream)))


def pack_templates(images, py, px, s16, p16, n=None, stream=None) -> None:
    n = images.shape[0] if n is None else n
    _check(load_library().cjx_pack_templates(_cuda_ptr(images, "images"), int(n), int(py), int(px),
                                             _cuda_ptr(s16, "s16"), _cuda_ptr(p16, "p16"), _stream_ptr(stream)))


def pack_observed(observed, params, py, px, flags, y16, z16, oo, yinv, zinv, stream=None) -> None:
    _check(load_library().cjx_pack_observed(
        _cuda_ptr(observed, "observed"), _cuda_ptr(params, "params"), int(observed.shape[0]), int(py), int(px),
        int(flags), _cuda_ptr(y16, "y16"), _cuda_ptr(z16, "z16"), _cuda_ptr(oo, "oo"), _cuda_ptr(yinv, "yinv"),
        _cuda_ptr(zinv, "zinv"), _stream_ptr(stream)))


def ncc_argmax(num, den, n, T, oo, yinv, zinv, best_score, best_orientation, *, t0=0, scores=None,
               accumulate_best=False, stream=None) -> None:
    _check(load_library().cjx_ncc_argmax(
        _cuda_ptr(num, "num"), _cuda_ptr(den, "den"), int(num.stride(0)), int(n), int(T), _cuda_ptr(oo, "oo"),
        _cuda_ptr(yinv, "yinv"), _cuda_ptr(zinv, "zinv"), int(t0), _opt_ptr(scores, "scores"),
        int(scores.stride(0)) if scores is not None else 0, _cuda_ptr(best_score, "best_score"),
        _cuda_ptr(best_orientation, "best_orientation"), 1 if accumulate_best else 0, _stream_ptr(stream)))


def ncc_topk(num, den, n, T, oo, yinv, zinv, k, indices, stream=None) -> None:
    _check(load_library().cjx_ncc_topk(
        _cuda_ptr(num, "num"), _cuda_ptr(den, "den"), int(num.stride(0)), int(n), int(T), _cuda_ptr(oo, "oo"),
        _cuda_ptr(yinv, "yinv"), _cuda_ptr(zinv, "zinv"), int(k), _cuda_ptr(indices, "indices"), _stream_ptr(stream)))


def pack_observed32(observed, params, py, px, flags, y32, z32, oo, stream=None) -> None:
    """cjx_pack_observed32: unscaled FP32 NCC terms of each observed image (complex64 y32, float z32, oo)."""
    _check(load_library().cjx_pack_observed32(
        _cuda_ptr(observed, "observed"), _cuda_ptr(params, "params"), int(observed.shape[0]), int(py), int(px),
        int(flags), _cuda_ptr(y32, "y32"), _cuda_ptr(z32, "z32"), _cuda_ptr(oo, "oo"), _stream_ptr(stream)))


def ncc_rerank32(bank, py, px, y32, z32, oo, candidates, best_score, best_orientation, *, scores=None,
                 stream=None) -> None:
    """cjx_ncc_rerank32: FP32 NCC of each image against its candidates [n, m] from the FP32 template bank."""
    n, m = int(candidates.shape[0]), int(candidates.shape[1])
    _check(load_library().cjx_ncc_rerank32(
        _cuda_ptr(bank, "bank"), int(py), int(px), int(bank.shape[0]), _cuda_ptr(y32, "y32"), _cuda_ptr(z32, "z32"),
        _cuda_ptr(oo, "oo"), n, _cuda_ptr(candidates, "candidates"), m, _opt_ptr(scores, "scores"),
        _cuda_ptr(best_score, "best_score"), _cuda_ptr(best_orientation, "best_orientation"), _stream_ptr(stream)))


def ncc_directions_workspace_size(n: int, kd: int, n_dir: int) -> int:
    v = ctypes.c_size_t(0)
    _check(load_library().cjx_ncc_directions_workspace_size(int(n), int(kd), int(n_dir), ctypes.byref(v)))
    return int(v.value)


def ncc_directions(y16, z16, s16, p16, kp, dirs, n_dir, n_inplane, num, den, workspace, stream=None) -> None:
    """cjx_ncc_directions: num / den [n, kd * n_inplane] of each image against its proposed directions'
    templates (rows from pack_observed / pack_templates)."""
    n, kd = int(dirs.shape[0]), int(dirs.shape[1])
    _check(load_library().cjx_ncc_directions(
        _cuda_ptr(y16, "y16"), _cuda_ptr(z16, "z16"), _cuda_ptr(s16, "s16"), _cuda_ptr(p16, "p16"), n, int(kp),
        _cuda_ptr(dirs, "dirs"), kd, int(n_dir), int(n_inplane), _cuda_ptr(num, "num"), _cuda_ptr(den, "den"),
        _cuda_ptr(workspace, "workspace"), int(workspace.numel() * workspace.element_size()), _stream_ptr(stream)))


def selftest_bounded_wait(limit_ns: int, status, stream=None) -> None:
    """Launch the bounded-wait self-test; `status` is a zeroed int32 CUDA tensor of one element."""
    _check(load_library().cjx_selftest_bounded_wait(ctypes.c_uint64(int(limit_ns)), _cuda_ptr(status, "status"),
                                                    _stream_ptr(stream)))


def device_status(reset: bool = True, stream=None) -> int:
    """First error code a device-side wait recorded (0 = none); synchronises the stream."""
    v = ctypes.c_int(0)
    _check(load_library().cjx_device_status(ctypes.byref(v), 1 if reset else 0, _stream_ptr(stream)))
    return int(v.value)


def probe_read_bandwidth(buf, passes, sink, stream=None) -> None:
    _check(
        load_library().cjx_probe_read_bandwidth(
            _cuda_ptr(buf, "buf"),
            buf.numel() * buf.element_size(),
            int(passes),
            _cuda_ptr(sink, "sink"),
            _stream_ptr(stream),
        )
    )


def brick_volume_pairs(n: int, grid, pairs, stream=None) -> None:
    """x-pair bricked copy (CJX_GRID_BRICKED_PAIRS) of a complex64 N^3 grid into `pairs`."""
    _check(load_library().cjx_brick_volume_pairs(int(n), _cuda_ptr(grid, "grid"), _cuda_ptr(pairs, "pairs"),
                                                 _stream_ptr(stream)))


def bricked_volume_size(n: int) -> int:
    out = ctypes.c_size_t(0)
    _check(load_library().cjx_bricked_volume_size(int(n), ctypes.byref(out)))
    return int(out.value)


def brick_volume(grid, stream=None):
    """Bricked copy (complex64, 1-D) of a complex64 [N, N, N] CUDA grid."""
    import torch

    n = grid.shape[0]
    if grid.dtype != torch.complex64 or tuple(grid.shape) != (n, n, n):
        raise ValueError("grid must be complex64 [N, N, N]")
    out = torch.empty(bricked_volume_size(n) // 8, dtype=torch.complex64, device=grid.device)
    _check(load_library().cjx_brick_volume(int(n), _cuda_ptr(grid, "grid"), _cuda_ptr(out, "bricked"),
                                           _stream_ptr(stream)))
    return out


def brick_volume_pairs_new(grid, stream=None):
    """x-pair bricked copy (CJX_GRID_BRICKED_PAIRS; 16 bytes per entry) of a complex64 [N, N, N] grid."""
    import torch

    n = grid.shape[0]
    if grid.dtype != torch.complex64 or tuple(grid.shape) != (n, n, n):
        raise ValueError("grid must be complex64 [N, N, N]")
    out = torch.empty(2 * bricked_volume_size(n) // 8, dtype=torch.complex64, device=grid.device)
    brick_volume_pairs(n, grid.contiguous(), out, stream)
    return out


def spline_coefficients_workspace_size(n: int) -> int:
    out = ctypes.c_size_t(0)
    _check(load_library().cjx_spline_coefficients_workspace_size(int(n), ctypes.byref(out)))
    return int(out.value)


def spline_coefficients(grid, out=None, workspace=None, stream=None):
    """Cubic-spline coefficients ((N+2)^3 complex64) of a centred complex64 [N, N, N] CUDA grid.

    cryojax/ndimage/_map_coordinates.py:71-82 (compute_spline_coefficients).
    """
    import torch

    n = grid.shape[0]
    if grid.dtype != torch.complex64 or tuple(grid.shape) != (n, n, n):
        raise ValueError("grid must be complex64 [N, N, N]")
    grid = grid.contiguous()
    m = n + 2
    if out is None:
        out = torch.empty((m, m, m), dtype=torch.complex64, device=grid.device)
    elif out.dtype != torch.complex64 or tuple(out.shape) != (m, m, m) or not out.is_contiguous():
        raise ValueError("out must be contiguous complex64 [N+2, N+2, N+2]")
    need = spline_coefficients_workspace_size(n)
    if workspace is None or workspace.numel() * workspace.element_size() < need:
        workspace = torch.empty(need, dtype=torch.uint8, device=grid.device)
    _check(load_library().cjx_spline_coefficients(int(n), _cuda_ptr(grid, "grid"), _cuda_ptr(out, "coefficients"),
                                                  _cuda_ptr(workspace, "workspace"),
                                                  workspace.numel() * workspace.element_size(), _stream_ptr(stream)))
    return out


def render_gaussians(shape, voxel_size, positions, amplitudes, variances, out=None, accumulate=False,
                     cutoff_sigmas=0.0, stream=None):
    """Voxel-averaged Gaussian mixture on a float32 [nz, ny, nx] CUDA grid (cjx_render_gaussians)."""
    import torch

    nz, ny, nx = (int(v) for v in shape)
    dev = positions.device
    pos = positions.to(torch.float32).contiguous()
    amp = amplitudes.to(torch.float32).contiguous()
    var = variances.to(torch.float32).contiguous()
    n = pos.shape[0]
    if pos.shape != (n, 3) or amp.dim() != 2 or amp.shape[0] != n or var.shape != amp.shape:
        raise ValueError("positions [n, 3], amplitudes and variances [n, n_gaussians]")
    if out is None:
        out = torch.empty((nz, ny, nx), dtype=torch.float32, device=dev)
    elif out.dtype != torch.float32 or tuple(out.shape) != (nz, ny, nx) or not out.is_contiguous():
        raise ValueError("out must be contiguous float32 [nz, ny, nx]")
    d = RenderDesc(nz, ny, nx, int(amp.shape[1]), float(voxel_size), float(cutoff_sigmas),
                   CJX_RENDER_ACCUMULATE if accumulate else 0, 0)
    null = ctypes.c_void_p(0)
    _check(load_library().cjx_render_gaussians(
        ctypes.byref(d), _cuda_ptr(pos, "positions") if n else null, _cuda_ptr(amp, "amplitudes") if n else null,
        _cuda_ptr(var, "variances") if n else null, n, _cuda_ptr(out, "grid"), _stream_ptr(stream)))
    return out


def fft_c2c(x, direction: int, out=None, stream=None):
    """Row-wise complex64 FFT of a CUDA tensor [..., n] with the library's warp FFTs."""
    import torch

    if x.dtype != torch.complex64:
        raise ValueError("x must be complex64")
    x = x.contiguous()
    if out is None:
        out = torch.empty_like(x)
    n = x.shape[-1]
    _check(load_library().cjx_fft_c2c(int(n), int(direction), _cuda_ptr(x, "x"), _cuda_ptr(out, "out"),
                                      int(x.numel() // n), _stream_ptr(stream)))
    return out


CJX_PP_NORMALIZE = 1


def postprocess_workspace_size(n_images: int, py: int, px: int) -> int:
    v = ctypes.c_size_t(0)
    _check(load_library().cjx_postprocess_workspace_size(int(n_images), int(py), int(px), ctypes.byref(v)))
    return int(v.value)


def postprocess_real(fourier, padded_shape, shape, *, normalize=False, mask=None, out=None, workspace=None,
                     stream=None):
    """cjx_postprocess_real: complex64 CUDA [..., Py, Px//2+1] -> float32 [..., H, W] real-space images
    (irfftn -> centre crop -> optional normalisation -> optional float32 [H, W] mask)."""
    import torch

    if fourier.dtype != torch.complex64:
        raise ValueError("fourier must be complex64")
    py, px = (int(v) for v in padded_shape)
    h, w = (int(v) for v in shape)
    if tuple(fourier.shape[-2:]) != (py, px // 2 + 1):
        raise ValueError(f"fourier images must be [..., {py}, {px // 2 + 1}], got {tuple(fourier.shape)}")
    f = fourier.contiguous()
    lead = tuple(f.shape[:-2])
    n = int(np.prod(lead)) if lead else 1
    if out is None:
        out = torch.empty(lead + (h, w), dtype=torch.float32, device=f.device)
    if n == 0:
        return out
    if mask is not None:
        mask = torch.as_tensor(mask, dtype=torch.float32, device=f.device).contiguous()
        if tuple(mask.shape) != (h, w):
            raise ValueError(f"mask must be [{h}, {w}], got {tuple(mask.shape)}")
    if workspace is None or workspace.numel() * workspace.element_size() < postprocess_workspace_size(1, py, px):
        # up to 2048 images per pass: larger batches take several passes over the same workspace
        workspace = torch.empty(postprocess_workspace_size(min(n, 2048), py, px), dtype=torch.uint8, device=f.device)
    wsb = workspace.numel() * workspace.element_size()
    _check(load_library().cjx_postprocess_real(
        n, py, px, h, w, CJX_PP_NORMALIZE if normalize else 0, _cuda_ptr(f, "fourier"),
        _cuda_ptr(mask, "mask") if mask is not None else None, _cuda_ptr(out, "out"),
        _cuda_ptr(workspace, "workspace"), int(wsb), _stream_ptr(stream)))
    return out


def rfft2(image, out=None, stream=None):
    """cjx_rfft2: float32 CUDA [..., Py, Px] -> complex64 [..., Py, Px//2+1], rfft2 of ifftshift(image)."""
    import torch

    x = image.to(torch.float32).contiguous()
    py, px = int(x.shape[-2]), int(x.shape[-1])
    lead = tuple(x.shape[:-2])
    n = int(np.prod(lead)) if lead else 1
    if out is None:
        out = torch.empty(lead + (py, px // 2 + 1), dtype=torch.complex64, device=x.device)
    if n == 0:
        return out
    _check(load_library().cjx_rfft2(n, py, px, _cuda_ptr(x, "image"), _cuda_ptr(out, "out"), _stream_ptr(stream)))
    return out


def tuning_set(key: int, value: int) -> None:
    _check(load_library().cjx_tuning_set(int(key), int(value)))


def tuning_get(key: int) -> int:
    v = ctypes.c_int64(0)
    _check(load_library().cjx_tuning_get(int(key), ctypes.byref(v)))
    return int(v.value)


def profile_enable(on: bool) -> None:
    _check(load_library().cjx_profile_enable(1 if on else 0))


def profile_read(max_kernels: int = 32) -> dict:
    """{kernel name: (launches, total ms)} recorded since the last read."""
    names = ctypes.create_string_buffer(32 * max_kernels)
    counts = (ctypes.c_int64 * max_kernels)()
    ms = (ctypes.c_double * max_kernels)()
    n = ctypes.c_int(0)
    _check(load_library().cjx_profile_read(names, counts, ms, max_kernels, ctypes.byref(n)))
    out = {}
    for i in range(n.value):
        name = names.raw[32 * i: 32 * (i + 1)].split(b"\0", 1)[0].decode()
        out[name] = (int(counts[i]), float(ms[i]))
    return out


def empty_params(n_images: int) -> np.ndarray:
    p = np.zeros((n_images, PARAMS_DOUBLES), np.float64)
    p[:, P_SCALE] = 1.0
    p[:, P_ENV_AMP] = 1.0
    return p
