"""GPU: cjx_ncc_directions (the learned search's candidate scoring from the shared FP16 template rows)
against float64 dot products of the same FP16 rows.

Cases: template counts per direction that are not a multiple of the kernel's column tiles (12) and larger
than one pass (50), a row length whose 16-byte vectors do not fill the last K step (kp = 104), directions
outside the grid (their sums are 0) and one direction proposed by more pairs than one tile holds (37).
Tolerance: each sum within 1e-5 of |y| |s| (FP16 products, FP32 accumulation); two runs agree bitwise.
"""

import pytest
import torch

pytestmark = pytest.mark.gpu


def _case(n, kd, n_dir, ni, kp, seed):
    from cryojax_b200 import _native as nat

    g = torch.Generator(device="cuda").manual_seed(seed)
    T = n_dir * ni
    y16 = torch.randn((n, 2 * kp), generator=g, device="cuda").half()
    z16 = torch.rand((n, kp), generator=g, device="cuda").half()
    s16 = torch.randn((T, 2 * kp), generator=g, device="cuda").half()
    p16 = torch.rand((T, kp), generator=g, device="cuda").half()
    dirs = torch.randint(0, n_dir, (n, kd), generator=g, device="cuda", dtype=torch.int32)
    dirs[:, 0] = 3 % n_dir  # one direction proposed by every image: several tiles in one bin
    dirs[0, 1] = -1  # outside the grid
    dirs[1 % n, kd - 1] = n_dir
    out = []
    for _ in range(2):
        num = torch.full((n, kd * ni), float("nan"), device="cuda")
        den = torch.full_like(num, float("nan"))
        ws = torch.empty(nat.ncc_directions_workspace_size(n, kd, n_dir), dtype=torch.uint8, device="cuda")
        nat.ncc_directions(y16, z16, s16, p16, kp, dirs, n_dir, ni, num, den, ws)
        torch.cuda.synchronize()
        out.append((num, den))
    assert torch.equal(out[0][0], out[1][0]) and torch.equal(out[0][1], out[1][1])
    num, den = out[0]
    d = dirs.long()
    valid = (d >= 0) & (d < n_dir)
    t = (d.clamp(0, n_dir - 1)[:, :, None] * ni + torch.arange(ni, device="cuda")).reshape(n, -1)
    st, pt = s16[t].double(), p16[t].double()  # the candidates' rows only
    ref_n = torch.einsum("bk,bjk->bj", y16.double(), st)
    ref_d = torch.einsum("bk,bjk->bj", z16.double(), pt)
    mask = valid[:, :, None].expand(n, kd, ni).reshape(n, -1)
    ref_n = torch.where(mask, ref_n, torch.zeros_like(ref_n))
    ref_d = torch.where(mask, ref_d, torch.zeros_like(ref_d))
    scale_n = y16.double().norm(dim=1)[:, None] * st.norm(dim=2)
    scale_d = z16.double().norm(dim=1)[:, None] * pt.norm(dim=2)
    assert torch.isfinite(num).all() and torch.isfinite(den).all()
    assert ((num.double() - ref_n).abs() <= 1e-5 * scale_n).all()
    assert ((den.double() - ref_d).abs() <= 1e-5 * scale_d).all()
    assert (num[~mask] == 0).all() and (den[~mask] == 0).all()


@pytest.mark.parametrize("n,kd,n_dir,ni,kp", [(37, 5, 11, 12, 104), (20, 3, 7, 50, 8320), (16, 4, 768, 48, 8320)])
def test_ncc_directions_matches_float64(cuda_device, n, kd, n_dir, ni, kp):
    _case(n, kd, n_dir, ni, kp, seed=n + kd)
