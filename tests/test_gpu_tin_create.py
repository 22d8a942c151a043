"""TINCreate_list (SubFunctions.cpp:2768-2846) on the GPU against the
reference build's own function, triangle for triangle and in order.

The points are snapped to the level's grid, where co-circular points (every
grid square, every rectangle) are common: the triangles there are decided by
the reference's divide and conquer, and their order by its edge allocator.
The cases: the matched points of an Ortho_blunder case, full and partly
filled integer grids (ties everywhere), random subsets from 3 to a few
thousand points (both sides of the 100-point cut where the reference stops
splitting its edge list), a thin strip, and a 45 k-point grid."""
import numpy as np
import pytest

from oracle import refpy
from setsm_b200 import abi, vll
from tests import cases

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refpy.available(), reason="reference build not available")]

RES = 2.0
X0, Y0 = 1000.0, 5000.0


def grid_points(cells, rng, jitter=True):
    """Points in the given (col, row) cells, jittered inside their cells."""
    pts = np.zeros(len(cells), dtype=abi.POINT3_DTYPE)
    j = (rng.random((len(cells), 2)) - 0.5) * 0.8 * RES if jitter else np.zeros((len(cells), 2))
    pts["x"] = X0 + cells[:, 0] * RES + j[:, 0]
    pts["y"] = Y0 + cells[:, 1] * RES + j[:, 1]
    pts["z"] = rng.random(len(cells)) * 100.0
    pts["flag"] = 1
    return pts


def extent(w, h):
    return [X0, Y0, X0 + (w - 1) * RES, Y0 + (h - 1) * RES]


def check(ctx, pts, mm, res=RES):
    want = refpy.tin_create(pts, mm, res)
    got = ctx.tin_create(pts, mm, res)
    assert len(got) == len(want)
    assert got.tobytes() == want.tobytes()
    return len(got)


def test_tin_of_matched_points(gpu_ctx):
    inp, pts, _ = cases.make_tin_case()
    n = check(gpu_ctx, pts, inp.boundary, inp.grid_resolution)
    assert n > len(pts)


@pytest.mark.parametrize("w,h,frac", [(10, 10, 1.0), (17, 13, 1.0), (64, 64, 0.3), (64, 64, 0.9),
                                      (200, 150, 0.05), (41, 3, 1.0)])
def test_tin_of_grid_subsets(gpu_ctx, w, h, frac):
    rng = np.random.default_rng(w * 1000 + h)
    for _ in range(2):
        m = rng.random((h, w)) < frac
        yy, xx = np.nonzero(m)
        cells = np.stack([xx, yy], 1)
        rng.shuffle(cells)
        check(gpu_ctx, grid_points(cells, rng), extent(w, h))


@pytest.mark.parametrize("n", [3, 4, 5, 6, 7, 9, 11, 33, 99, 100, 101, 257, 3000])
def test_tin_of_random_points(gpu_ctx, n):
    rng = np.random.default_rng(n)
    w = h = 80
    idx = rng.choice(w * h, n, replace=False)
    cells = np.stack([idx % w, idx // w], 1)
    check(gpu_ctx, grid_points(cells, rng, jitter=(n % 2 == 1)), extent(w, h))


def test_tin_of_large_grid(gpu_ctx):
    rng = np.random.default_rng(300)
    m = rng.random((300, 300)) < 0.5
    yy, xx = np.nonzero(m)
    cells = np.stack([xx, yy], 1)
    rng.shuffle(cells)
    assert check(gpu_ctx, grid_points(cells, rng), extent(300, 300)) > 80000


def test_tin_device_entry_matches_host(gpu_ctx):
    import torch
    rng = np.random.default_rng(7)
    idx = rng.choice(64 * 64, 1500, replace=False)
    pts = grid_points(np.stack([idx % 64, idx // 64], 1), rng)
    mm = extent(64, 64)
    host = gpu_ctx.tin_create(pts, mm, RES)
    d_pts = torch.from_numpy(pts.view(np.uint8).copy()).cuda()
    cap = 2 * len(pts)
    d_tris = torch.zeros(cap * abi.TRI_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    n = gpu_ctx.tin_create_device(d_pts.data_ptr(), len(pts), mm, RES, d_tris.data_ptr(), cap)
    dev = d_tris.cpu().numpy().view(abi.TRI_DTYPE)[:n]
    assert dev.tobytes() == host.tobytes()
    # too small an output: the length is reported, nothing is written
    small = torch.zeros(16 * abi.TRI_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    with pytest.raises(vll.VLLError) as e:
        gpu_ctx.tin_create_device(d_pts.data_ptr(), len(pts), mm, RES, small.data_ptr(), 16)
    assert e.value.code == abi.VLL_ERR_CAPACITY


def test_tin_rejects_two_points_in_one_cell(gpu_ctx):
    rng = np.random.default_rng(3)
    cells = np.array([[0, 0], [5, 0], [0, 5], [5, 5], [5, 5]])
    pts = grid_points(cells, rng)
    with pytest.raises(vll.VLLError) as e:
        gpu_ctx.tin_create(pts, extent(8, 8), RES)
    assert e.value.code == abi.VLL_ERR_INVALID
    # fewer than three points: no triangles, as the reference
    assert len(gpu_ctx.tin_create(pts[:2], extent(8, 8), RES)) == 0
