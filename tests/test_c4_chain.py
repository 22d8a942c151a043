"""The C4 range chain's interpolation (workloads.tin_heights): heights of a
plane are reproduced exactly inside the TIN; nodes outside every triangle take
the nearest point's height."""
import numpy as np

from setsm_b200 import abi, workloads
from setsm_b200.synth import Grid


def _grid(w, h, res, x0=100.0, y0=200.0):
    cols, rows = np.meshgrid(np.arange(w), np.arange(h))
    pts = np.stack([x0 + cols.ravel() * res, y0 + rows.ravel() * res], 1).astype(np.float64)
    return Grid(boundary=np.array([x0, y0, x0 + (w - 1) * res, y0 + (h - 1) * res]),
                resolution=res, width=w, height=h, pts=pts, wgs=np.zeros_like(pts),
                truth=np.zeros(w * h))


def _points(xy, z):
    p = np.zeros(len(xy), dtype=abi.POINT3_DTYPE)
    p["x"], p["y"], p["z"], p["flag"] = xy[:, 0], xy[:, 1], z, 1
    return p


def test_plane_is_reproduced_inside_the_tin():
    g = _grid(17, 13, 4.0)
    # two triangles covering the grid's rectangle
    corners = np.array([[100.0, 200.0], [164.0, 200.0], [164.0, 248.0], [100.0, 248.0]])
    plane = lambda x, y: 3.0 + 0.25 * (x - 100.0) - 0.5 * (y - 200.0)
    pts = _points(corners, plane(corners[:, 0], corners[:, 1]))
    tris = np.zeros(2, dtype=abi.TRI_DTYPE)
    tris[0] = (0, 1, 2)
    tris[1] = (0, 2, 3)
    h, covered = workloads.tin_heights(pts, tris, g)
    assert covered.all()
    np.testing.assert_allclose(h, plane(g.pts[:, 0], g.pts[:, 1]), rtol=0, atol=1e-9)


def test_nodes_outside_take_the_nearest_point():
    g = _grid(9, 9, 2.0)
    # one small triangle in a corner
    xy = np.array([[100.0, 200.0], [104.0, 200.0], [100.0, 204.0]])
    pts = _points(xy, np.array([10.0, 20.0, 30.0]))
    tris = np.zeros(1, dtype=abi.TRI_DTYPE)
    tris[0] = (0, 1, 2)
    h, covered = workloads.tin_heights(pts, tris, g)
    assert covered.sum() == 6          # the nodes on and inside the triangle
    at = lambda x, y: h[int((y - 200.0) / 2.0) * 9 + int((x - 100.0) / 2.0)]
    assert at(116.0, 200.0) == 20.0    # nearest point (104, 200)
    assert at(100.0, 216.0) == 30.0    # nearest point (100, 204)
    assert at(102.0, 200.0) == 15.0    # on the triangle's edge: interpolated
    assert np.isfinite(h).all()
