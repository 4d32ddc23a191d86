"""cjx_slice_ctf_forward_noalloc against cjx_slice_ctf_forward, through the C-ABI.

The allocation-free entry point serves callers that cannot call cudaMalloc
themselves (a runtime that owns every device allocation, such as an XLA
custom call without a scratch allocator, or a service that forbids
allocation after start-up).  Its scratch is a fixed array inside the
library.  Two calls in a row must both match the allocating entry point:
the second one runs on scratch left over from the first.

This file is collected last on purpose (tests run in file order), so a
failure here comes after every other test has run.
"""

import numpy as np
import pytest

from tests.helpers import IMAGE_REL_L2_TOL, make_volume, random_specs, rel_l2_per_image, specs_to_model_args

pytestmark = pytest.mark.gpu


def _inputs(seed, n_images, shape):
    import torch

    from cryojax_b200 import simulator as S

    vol, grid, fs = make_volume(32, 60, seed=seed)
    specs = random_specs(n_images, seed=seed + 1, shape=shape)
    pose, tt, cfg = specs_to_model_args(specs)
    dvol = S.FourierVoxelGridVolume(torch.as_tensor(grid.astype(np.complex64)).cuda())
    model = S.make_image_model(dvol, cfg, pose, tt)
    params = torch.as_tensor(model.image_params(), device="cuda")
    return dvol.fourier_voxel_grid, params, model._flags(), cfg.padded_shape


def _allocating(grid, params, flags, padded, n=None):
    import torch

    from cryojax_b200 import _native as nat

    py, px = padded
    desc = nat.make_desc(grid.shape[0] if n is None else n, py, px, flags)
    ws = torch.empty(max(nat.workspace_size(desc, params.shape[0]), 1), dtype=torch.uint8, device="cuda")
    out = torch.empty((params.shape[0], py, px // 2 + 1), dtype=torch.complex64, device="cuda")
    nat.slice_ctf_forward(desc, grid, params, out, ws)
    return out


def _noalloc(grid, params, flags, padded, images_per_chunk=0, n=None):
    import torch

    from cryojax_b200 import _native as nat

    py, px = padded
    desc = nat.make_desc(grid.shape[0] if n is None else n, py, px, flags, images_per_chunk=images_per_chunk)
    out = torch.empty((params.shape[0], py, px // 2 + 1), dtype=torch.complex64, device="cuda")
    nat.slice_ctf_forward_noalloc(desc, grid, params, out)
    return out


def test_noalloc_matches_allocating_entry_point_twice(cuda_device):
    import torch

    # call 1 (first call on this device: looks up the scratch address)
    g1, p1, f1, s1 = _inputs(101, 9, (32, 32))
    got1 = _noalloc(g1, p1, f1, s1)
    ref1 = _allocating(g1, p1, f1, s1)
    # call 2: different volume, images and shape, on the scratch call 1 left behind
    g2, p2, f2, s2 = _inputs(202, 13, (40, 24))
    got2 = _noalloc(g2, p2, f2, s2, images_per_chunk=4)
    ref2 = _allocating(g2, p2, f2, s2)
    torch.cuda.synchronize()
    e1 = rel_l2_per_image(got1.cpu().numpy(), ref1.cpu().numpy())
    e2 = rel_l2_per_image(got2.cpu().numpy(), ref2.cpu().numpy())
    assert max(e1) <= IMAGE_REL_L2_TOL, e1
    assert max(e2) <= IMAGE_REL_L2_TOL, e2


def test_noalloc_leaves_free_device_memory_unchanged(cuda_device):
    """The property the entry point is named for: after a warm-up call (which may load kernels and look up
    the scratch address), further calls change the device's free memory (cudaMemGetInfo, which
    torch.cuda.mem_get_info wraps) by not one byte."""
    import torch

    from cryojax_b200 import _native as nat

    g, p, f, s = _inputs(505, 11, (32, 32))
    py, px = s
    desc = nat.make_desc(g.shape[0], py, px, f, images_per_chunk=3)
    out = torch.empty((p.shape[0], py, px // 2 + 1), dtype=torch.complex64, device="cuda")
    nat.slice_ctf_forward_noalloc(desc, g, p, out)
    torch.cuda.synchronize()
    first = out.clone()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        nat.slice_ctf_forward_noalloc(desc, g, p, out)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0, (free0, free1)
    assert torch.equal(out, first)


def test_noalloc_rejects_chunks_beyond_its_scratch(cuda_device):
    from cryojax_b200 import _native as nat

    g, p, f, s = _inputs(303, 2, (32, 32))
    per_image = nat.workspace_size(nat.make_desc(g.shape[0], s[0], s[1], f, images_per_chunk=1), 1)
    too_many = nat.NOALLOC_SCRATCH_BYTES // per_image + 1
    with pytest.raises(nat.CryojaxB200Error) as e:
        _noalloc(g, p, f, s, images_per_chunk=too_many)
    assert e.value.code == nat.CJX_ERR_UNSUPPORTED
    assert "CJX_NOALLOC_SCRATCH_BYTES" in str(e.value)


@pytest.mark.parametrize("variant", ["ewald", "spline"])
def test_noalloc_ewald_and_spline_match_allocating_entry_point(cuda_device, variant):
    """The Ewald sphere's contrast (CJX_EWALD_SPHERE with the CTF) and C-order spline coefficients
    (CJX_GRID_SPLINE, desc.n = coefficient side - 2) through the allocation-free entry point."""
    import torch

    from cryojax_b200 import _native as nat

    g, p, f, s = _inputs(404, 5, (32, 32))
    n = g.shape[0]
    if variant == "ewald":
        f = f | nat.CJX_EWALD_SPHERE
    else:
        coef = torch.empty((n + 2,) * 3, dtype=torch.complex64, device="cuda")
        ws = torch.empty(nat.spline_coefficients_workspace_size(n), dtype=torch.uint8, device="cuda")
        nat.spline_coefficients(g, coef, ws)
        g, f = coef, f | nat.CJX_GRID_SPLINE
    got = _noalloc(g, p, f, s, n=n)
    ref = _allocating(g, p, f, s, n=n)
    torch.cuda.synchronize()
    err = rel_l2_per_image(got.cpu().numpy(), ref.cpu().numpy())
    assert max(err) <= IMAGE_REL_L2_TOL, err
