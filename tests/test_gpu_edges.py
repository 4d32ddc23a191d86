"""GPU: edge cases — empty batches on every entry point, and the largest volume side.

Maximum size (N = CJX_MAX_SIDE = 1024, a 8.6 GB complex64 grid): a float64
oracle of the whole grid does not fit, so the grid is a plane wave
g[z, y, x] = exp(i (a x + b y + c z)) whose trilinear samples are computed
exactly here from the sample coordinates.  The coordinates are formed as
the kernels form them (float32 rotation, a float32 product then a fused
multiply-add), so corner validity near the faces is decided identically.
Tolerances: no-resize output within 2e-6 (absolute, |g| = 1) of the
analytic samples; the resize path (N = 1024 -> 512^2) within rel-L2 1e-5 of
a float64 torch restatement of irfftn -> centre crop -> rfftn applied to the
no-resize output; the x-pair and bricked layouts bit-identical, the linear
layout within 1e-6.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _params(n, seed):
    from cryojax_b200 import _native as nat
    from cryojax_b200 import rotations as rot

    p = nat.empty_params(n)
    q = rot.sample_uniform_quaternions(np.random.default_rng(seed), n)
    p[:, 0:9] = rot.quat_to_matrix(q).reshape(n, 9)
    p[:, nat.P_PIXEL_SIZE] = 2.0
    p[:, nat.P_WAVELENGTH] = 0.0197
    p[:, nat.P_SCALE] = 1.0
    return p


def test_empty_batches_are_no_ops(cuda_device):
    import torch

    from cryojax_b200 import _native as nat

    grid = torch.zeros((64, 64, 64), dtype=torch.complex64, device="cuda")
    empty = torch.zeros((0, 32), dtype=torch.float64, device="cuda")
    desc = nat.make_desc(64, 32, 32, nat.CJX_APPLY_CTF | nat.CJX_APPLY_TRANSLATION)
    assert nat.workspace_size(desc, 0) == 0
    out = torch.zeros((0, 32, 17), dtype=torch.complex64, device="cuda")
    nat.slice_ctf_forward(desc, grid, empty, out, None)
    grads = torch.zeros((0, nat.GRAD_DOUBLES), dtype=torch.float64, device="cuda")
    obs = torch.zeros((0, 32, 17), dtype=torch.complex64, device="cuda")
    gg = torch.zeros_like(grid)
    nat.slice_ctf_loss_grad(desc, grid, empty, obs, grads, gg, None)
    assert torch.count_nonzero(gg) == 0
    sdesc = nat.SearchDesc()
    sdesc.slice, sdesc.n_images, sdesc.n_orientations, sdesc.candidates_per_image = desc, 0, 4, 0
    rots = torch.eye(3, dtype=torch.float64, device="cuda").reshape(1, 9).repeat(4, 1)
    ws = torch.empty(max(nat.search_workspace_size(sdesc), 1), dtype=torch.uint8, device="cuda")
    best = torch.zeros(0, dtype=torch.float32, device="cuda")
    best_i = torch.zeros(0, dtype=torch.int32, device="cuda")
    nat.search(sdesc, grid, empty, rots, obs, best, best_i, ws)
    arr = nat.make_groups([{"desc": desc, "grid": grid, "params": empty, "out": out, "n_images": 0}])
    nat.slice_ctf_forward_multi(arr)
    torch.cuda.synchronize()


def _plane_wave_samples(R, n, a, b, c, rows, cols):
    """Exact trilinear samples of the plane wave at rfft pixels (rows, cols), the kernels' coordinates."""
    f32 = np.float32
    h = n // 2
    ux = np.where(cols < h, cols, cols - n).astype(f32)
    vy = np.where(rows < h, rows, rows - n).astype(f32)
    o = []
    for ax in range(3):
        r0, r1 = f32(R[ax, 0]), f32(R[ax, 1])
        t = (r0.astype(np.float64) * ux).astype(f32)                      # float32 product
        o.append((r1.astype(np.float64) * vy + t.astype(np.float64)).astype(f32))  # fused multiply-add
    val = np.zeros(rows.shape, np.complex128)
    k = (a, b, c)
    nodes = []
    for ax in range(3):
        f = np.floor(o[ax])
        w1 = (o[ax] - f).astype(f32).astype(np.float64)
        i0 = f.astype(np.int64) + h
        i1 = i0 + 1
        i0 = np.where(i0 < 0, i0 + n, i0)  # JAX wraps a negative index once
        i1 = np.where(i1 < 0, i1 + n, i1)
        nodes.append(((i0, (i0 >= 0) & (i0 < n), 1.0 - w1), (i1, (i1 >= 0) & (i1 < n), w1)))
    for cz in range(2):
        for cy in range(2):
            for cx in range(2):
                (ix, vx, wx), (iy, vy_, wy), (iz, vz, wz) = nodes[0][cx], nodes[1][cy], nodes[2][cz]
                ok = vx & vy_ & vz
                g = np.exp(1j * (k[0] * ix + k[1] * iy + k[2] * iz))
                val += np.where(ok, wx * wy * wz * g, 0.0)
    return val


def test_largest_volume_side_no_resize_and_resize(cuda_device):
    import torch

    from cryojax_b200 import _native as nat

    n = 1024
    a, b, c = 0.031, -0.047, 0.019
    dev = "cuda"
    idx = torch.arange(n, device=dev, dtype=torch.float64)
    phase = (c * idx)[:, None, None] + (b * idx)[None, :, None] + (a * idx)[None, None, :]
    grid = torch.polar(torch.ones((), dtype=torch.float32, device=dev).expand(n, n, n),
                       phase.to(torch.float32)).contiguous()
    del phase
    p = _params(2, 7)
    pd = torch.as_tensor(p, device=dev)
    # no resize: (Py, Px) = (N, N)
    desc = nat.make_desc(n, n, n, 0)
    out = torch.empty((2, n, n // 2 + 1), dtype=torch.complex64, device=dev)
    nat.slice_ctf_forward(desc, grid, pd, out, None)
    got = out.cpu().numpy()
    rng = np.random.default_rng(1)
    rows = np.concatenate([rng.integers(0, n, 3000), [0, n // 2, n // 2, 0, n - 1, 1]])
    cols = np.concatenate([rng.integers(0, n // 2 + 1, 3000), [0, 0, n // 2, n // 2, n // 2, n // 2]])
    for i in range(2):
        exp = _plane_wave_samples(p[i, 0:9].reshape(3, 3), n, a, b, c, rows, cols)
        for r, cc in ((n // 2, 0), (0, n // 2), (n // 2, n // 2)):  # convert_fftn_to_rfftn(mode="real")
            exp = np.where((rows == r) & (cols == cc), exp.real, exp)
        err = np.abs(got[i, rows, cols] - exp).max()
        assert err <= 2e-6, (i, err)
    # resize N = 1024 -> 512^2 in the three layouts
    dres = {}
    for name in ("pairs", "bricked", "linear"):
        if name == "pairs":
            g, fl = nat.brick_volume_pairs_new(grid), nat.CJX_GRID_BRICKED_PAIRS
        elif name == "bricked":
            g, fl = nat.brick_volume(grid), nat.CJX_GRID_BRICKED
        else:
            g, fl = grid, 0
        d = nat.make_desc(n, 512, 512, fl)
        ws = torch.empty(nat.workspace_size(d, 2), dtype=torch.uint8, device=dev)
        o = torch.empty((2, 512, 257), dtype=torch.complex64, device=dev)
        nat.slice_ctf_forward(d, g, pd, o, ws)
        dres[name] = o.cpu().numpy()
        del g, ws
        torch.cuda.empty_cache()
    np.testing.assert_array_equal(dres["pairs"], dres["bricked"])
    assert np.abs(dres["linear"] - dres["bricked"]).max() <= 1e-6 * np.abs(dres["bricked"]).max()
    # the resize itself against float64 torch: symmetrise kx = 0 and N/2, irfftn, centre crop, rfftn
    hfull = out.to(torch.complex128)
    neg = (-torch.arange(n, device=dev)) % n
    for col in (0, n // 2):
        hfull[:, :, col] = 0.5 * (hfull[:, :, col] + torch.conj(hfull[:, neg, col]))
    x = torch.fft.fftshift(torch.fft.irfftn(hfull, s=(n, n), dim=(-2, -1)), dim=(-2, -1))
    c0 = n // 2 - 256
    x = torch.fft.ifftshift(x[:, c0:c0 + 512, c0:c0 + 512], dim=(-2, -1))
    ref = torch.fft.rfftn(x, dim=(-2, -1)).cpu().numpy()
    for i in range(2):
        rel = np.linalg.norm(dres["pairs"][i] - ref[i]) / np.linalg.norm(ref[i])
        assert rel <= 1e-5, (i, rel)
