"""The C-ABI library loads and exports every symbol include/cryojax_b200.h declares.

No compute calls here (no GPU needed): argument validation paths only.
"""

import ctypes
import os
import re

import pytest

from cryojax_b200 import _native as nat

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "cryojax_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"CJX_API\s+[\w\s\*]+?\b(cjx_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "cjx_slice_ctf_forward" in syms and "cjx_get_version" in syms


def test_library_exports_every_declared_symbol():
    lib = nat.load_library()
    for name in declared_symbols():
        assert hasattr(lib, name), name
    assert set(declared_symbols()) == set(nat.exported_symbols())


def test_version():
    assert nat.load_library().cjx_get_version() == 1


def test_struct_sizes_match_header():
    assert ctypes.sizeof(nat.SliceDesc) == 32
    assert nat.PARAMS_DOUBLES * 8 == 256


def test_workspace_size_and_validation():
    d = nat.make_desc(64, 32, 32, nat.CJX_APPLY_CTF | nat.CJX_APPLY_TRANSLATION)
    ws = nat.workspace_size(d, 10)
    # per image: Py * round8(N/2+1) + Py * round8(Px/2+1) + (N/2+1) * round8(N) complex64
    assert ws == 10 * 8 * (32 * 40 + 32 * 24 + 33 * 64)
    assert nat.workspace_size(nat.make_desc(64, 64, 64, 0), 10) == 0  # no resize stage
    assert nat.workspace_size(d, 0) == 0  # no images, no scratch
    assert nat.loss_workspace_size(d, 0) == 0
    with pytest.raises(nat.CryojaxB200Error) as e:
        nat.workspace_size(nat.make_desc(1, 32, 32, 0), 1)
    assert e.value.code == nat.CJX_ERR_INVALID_ARGUMENT
    with pytest.raises(nat.CryojaxB200Error) as e:
        nat.workspace_size(nat.make_desc(2048, 32, 32, 0), 1)
    assert e.value.code == nat.CJX_ERR_UNSUPPORTED
    with pytest.raises(nat.CryojaxB200Error) as e:
        nat.workspace_size(nat.make_desc(64, 32, 32, 1 << 20), 1)
    assert "flag" in str(e.value)


def test_forward_rejects_null_pointers_without_touching_the_gpu():
    lib = nat.load_library()
    d = nat.make_desc(64, 32, 32, 0)
    rc = lib.cjx_slice_ctf_forward(ctypes.byref(d), None, None, None, 4, None, None, 0, None)
    assert rc == nat.CJX_ERR_INVALID_ARGUMENT
    assert b"non-NULL" in lib.cjx_get_last_error()
    # zero images is a no-op
    assert lib.cjx_slice_ctf_forward(ctypes.byref(d), None, None, None, 0, None, None, 0, None) == nat.CJX_OK


def test_tuning_knobs():
    assert nat.tuning_get(nat.CJX_TUNE_GATHER_ILP) in (1, 2, 4)
    old = nat.tuning_get(nat.CJX_TUNE_GATHER_ILP)
    nat.tuning_set(nat.CJX_TUNE_GATHER_ILP, 4)
    assert nat.tuning_get(nat.CJX_TUNE_GATHER_ILP) == 4
    nat.tuning_set(nat.CJX_TUNE_GATHER_ILP, old)
    with pytest.raises(nat.CryojaxB200Error):
        nat.tuning_set(nat.CJX_TUNE_GATHER_ILP, 3)
    with pytest.raises(nat.CryojaxB200Error):
        nat.tuning_set(99, 1)
    assert nat.tuning_get(nat.CJX_TUNE_FFT_MODE) == 3  # transpose FFT for the 512-point column and row transforms
    assert nat.tuning_get(nat.CJX_TUNE_SCATTER_VEC) == 1
    assert nat.tuning_get(nat.CJX_TUNE_SPLINE_ILP) == 4
    with pytest.raises(nat.CryojaxB200Error):
        nat.tuning_set(nat.CJX_TUNE_SPLINE_ILP, 3)
    with pytest.raises(nat.CryojaxB200Error):
        nat.tuning_set(nat.CJX_TUNE_FFT_MODE, 4)
    with pytest.raises(nat.CryojaxB200Error):
        nat.tuning_set(nat.CJX_TUNE_SCATTER_VEC, 3)
    with pytest.raises(nat.CryojaxB200Error):
        nat.tuning_set(nat.CJX_TUNE_GATHER_MODE, 3)
    with pytest.raises(nat.CryojaxB200Error):
        nat.tuning_set(nat.CJX_TUNE_GATHER_TILE, 4)


def _search_desc(n, py, px, n_img, n_orient, k):
    s = nat.SearchDesc()
    s.slice = nat.make_desc(n, py, px, nat.CJX_APPLY_CTF)
    s.n_images, s.n_orientations, s.candidates_per_image = n_img, n_orient, k
    return s


def test_search_workspace_plan():
    assert ctypes.sizeof(nat.SearchDesc) == 32 + 24
    small = nat.search_workspace_size(_search_desc(64, 32, 32, 2, 96, 5))
    big = nat.search_workspace_size(_search_desc(64, 32, 32, 2, 96, 0))
    assert 0 < small < big  # exhaustive: 96 candidates per image, candidate lists: 5
    with pytest.raises(nat.CryojaxB200Error) as e:  # the score needs the resize stage
        nat.search_workspace_size(_search_desc(64, 64, 64, 2, 96, 0))
    assert e.value.code == nat.CJX_ERR_UNSUPPORTED
    with pytest.raises(nat.CryojaxB200Error) as e:
        nat.search_workspace_size(_search_desc(64, 32, 32, 2, 0, 0))
    assert e.value.code == nat.CJX_ERR_INVALID_ARGUMENT


def test_empty_groups_need_no_workspace():
    d = nat.make_desc(64, 32, 32, nat.CJX_APPLY_CTF)
    empty = nat.make_groups([{"desc": d, "n_images": 0}])
    assert nat.multi_workspace_size(empty) == 0
    one = nat.make_groups([{"desc": d, "n_images": 0}, {"desc": d, "n_images": 3}])
    assert nat.multi_workspace_size(one) == nat.workspace_size(d, 3)


def test_spline_flag_validation():
    d = nat.make_desc(64, 32, 32, nat.CJX_GRID_SPLINE | nat.CJX_GRID_BRICKED)
    assert nat.workspace_size(d, 2) == nat.workspace_size(nat.make_desc(64, 32, 32, 0), 2)
    assert nat.workspace_size(nat.make_desc(64, 32, 32, nat.CJX_GRID_SPLINE | nat.CJX_GRID_BRICKED_PAIRS), 1) > 0
    # spline volumes and the Ewald sphere's contrast have loss gradients; the Ewald sphere's bare spectrum
    # (no contrast transfer) has none
    assert nat.loss_workspace_size(nat.make_desc(64, 32, 32, nat.CJX_GRID_SPLINE), 1) > 0
    assert nat.loss_workspace_size(nat.make_desc(64, 32, 32, nat.CJX_EWALD_SPHERE | nat.CJX_APPLY_CTF), 1) > 0
    with pytest.raises(nat.CryojaxB200Error) as e:
        nat.loss_workspace_size(nat.make_desc(64, 32, 32, nat.CJX_EWALD_SPHERE), 1)
    assert e.value.code == nat.CJX_ERR_UNSUPPORTED
    # coefficient solve: N in [4, CJX_MAX_SIDE], scratch N (N + 2)^2 complex64
    assert nat.spline_coefficients_workspace_size(64) == 8 * 64 * 66 * 66
    for bad in (3, nat.CJX_MAX_SIDE + 1):
        with pytest.raises(nat.CryojaxB200Error) as e:
            nat.spline_coefficients_workspace_size(bad)
        assert e.value.code == nat.CJX_ERR_UNSUPPORTED
    lib = nat.load_library()
    assert lib.cjx_spline_coefficients(8, None, None, None, 0, None) == nat.CJX_ERR_INVALID_ARGUMENT
    # a coefficient array (side N + 2) can be bricked up to N = CJX_MAX_SIDE
    assert nat.bricked_volume_size(nat.CJX_MAX_SIDE + 2) > 0


@pytest.mark.skipif(__import__("torch").cuda.is_available(),
                    reason="hands the library placeholder addresses: argument validation only, on a machine without a GPU")
def test_misaligned_arrays_are_rejected_before_any_launch():
    """An x-pair grid that is not 16-byte aligned, a grid or an output that is not 8-byte aligned: the
    entry points return CJX_ERR_INVALID_ARGUMENT (checked on the host, before any CUDA call)."""
    lib = nat.load_library()
    vp = ctypes.c_void_p
    base = 0x10000000  # placeholder addresses; never dereferenced
    pairs = nat.make_desc(64, 32, 32, nat.CJX_APPLY_CTF | nat.CJX_GRID_BRICKED_PAIRS)
    plain = nat.make_desc(64, 32, 32, nat.CJX_APPLY_CTF)
    ws = vp(base + 0x100000)
    cases = [
        (pairs, base + 8, base + 0x2000),   # x-pair grid on an 8-byte boundary
        (plain, base + 4, base + 0x2000),   # grid on a 4-byte boundary
        (plain, base, base + 0x2004),       # output on a 4-byte boundary
    ]
    for desc, grid, out in cases:
        rc = lib.cjx_slice_ctf_forward(ctypes.byref(desc), vp(grid), vp(base + 0x1000), None, 2, vp(out), ws,
                                       1 << 30, None)
        assert rc == nat.CJX_ERR_INVALID_ARGUMENT, (grid, out)
        assert "aligned" in lib.cjx_get_last_error().decode()
        rc = lib.cjx_slice_ctf_forward_noalloc(ctypes.byref(desc), vp(grid), vp(base + 0x1000), None, 2, vp(out),
                                               None)
        assert rc == nat.CJX_ERR_INVALID_ARGUMENT, (grid, out)
    grads = vp(base + 0x3000)
    rc = lib.cjx_slice_ctf_loss_grad(ctypes.byref(pairs), vp(base + 8), vp(base + 0x1000), None, 2,
                                     vp(base + 0x2000), grads, None, ws, 1 << 30, None)
    assert rc == nat.CJX_ERR_INVALID_ARGUMENT
    rc = lib.cjx_slice_ctf_loss_grad(ctypes.byref(plain), vp(base), vp(base + 0x1000), None, 2,
                                     vp(base + 0x2000), grads, vp(base + 0x4004), ws, 1 << 30, None)
    assert rc == nat.CJX_ERR_INVALID_ARGUMENT


@pytest.mark.skipif(__import__("torch").cuda.is_available(),
                    reason="hands the library placeholder addresses: argument validation only, on a machine without a GPU")
def test_search_and_network_entry_points_validate_arguments():
    """The re-ranking, candidate-sum and convolution entry points reject bad sizes before any launch."""
    lib = nat.load_library()
    vp = ctypes.c_void_p
    base = 0x10000000  # placeholder addresses; never dereferenced
    p = [vp(base + 0x1000 * i) for i in range(8)]
    # re-ranking: m must be in [1, 16]
    assert lib.cjx_ncc_rerank32(p[0], 64, 64, 100, p[1], p[2], p[3], 4, p[4], 17, None, p[5], p[6], None) \
        == nat.CJX_ERR_INVALID_ARGUMENT
    assert lib.cjx_ncc_rerank32(p[0], 64, 64, 100, p[1], p[2], p[3], 4, p[4], 0, None, p[5], p[6], None) \
        == nat.CJX_ERR_INVALID_ARGUMENT
    # candidate sums: kp must be a positive multiple of 8
    ws = ctypes.c_size_t(0)
    assert lib.cjx_ncc_directions_workspace_size(4, 2, 10, ctypes.byref(ws)) == nat.CJX_OK
    assert ws.value == 4 * (3 * 12 + 8)
    assert lib.cjx_ncc_directions(p[0], p[1], p[2], p[3], 4, 12, p[4], 2, 10, 48, p[5], p[6], p[7], ws.value,
                                  None) == nat.CJX_ERR_INVALID_ARGUMENT
    # implicit convolution: only the network's (C, cout) pairs are compiled
    assert lib.cjx_cnn_conv_s2(p[0], 2, 16, 16, 48, p[1], 9 * 48, 64, None, p[2], None) == nat.CJX_ERR_UNSUPPORTED
    assert lib.cjx_cnn_conv_s2(p[0], 2, 15, 16, 32, p[1], 288, 64, None, p[2], None) == nat.CJX_ERR_INVALID_ARGUMENT
    assert lib.cjx_cnn_conv0(p[0], 2, 16, 16, p[1], 16, 64, None, p[2], None) == nat.CJX_ERR_INVALID_ARGUMENT
