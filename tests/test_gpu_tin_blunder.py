"""blunder_detection_TIN on the GPU (vll_tinblunder.cu) against the reference
(setsm_code.cpp:9158-9787): the fixtures made by the reference build, the
reference build itself over levels, iterations and switches, and the C++
drop-in with the reference's signature.  Point flags, the new-blunder marks,
every UGRID field, the counts and the height extent must be identical -- with
the height-difference sums formed in parallel (the threshold band, the
default), sequentially (SETSM_VLL_TIN_SUMS=exact), and with the band widened so
that the point pass is undone and re-run (SETSM_VLL_TIN_SUMS=wideband)."""
import ctypes as C

import numpy as np
import pytest

from oracle import refpy
from setsm_b200 import abi, vll
from tests import cases
from tests.golden import make_golden as mg

pytestmark = pytest.mark.gpu

DROPIN = ("_Z21blunder_detection_TINPK11ProjectInfoR12taglevelinfoiPfbtP11tagD3DPointPblP12tag"
          "UI3DPointlP10UpdateGridPlPdSD_")


def fresh_out(n):
    return np.zeros(n, np.uint8), np.zeros(2, np.int64), np.array([1e5, -1e5])


def assert_same(pts, det, gp3, counts, zext, w_pts, w_det, w_gp3, w_counts, w_zext):
    assert np.array_equal(pts["flag"], w_pts["flag"])
    assert np.array_equal(pts["z"], w_pts["z"])
    assert np.array_equal(det, w_det)
    assert cases.field_mismatch(mg.clean(gp3), mg.clean(w_gp3)) == {}
    assert np.array_equal(counts, w_counts)
    assert np.array_equal(zext, w_zext)


MODES = ["band", "exact", "wideband"]


@pytest.fixture(params=MODES)
def sums_mode(request, monkeypatch):
    if request.param != "band":
        monkeypatch.setenv("SETSM_VLL_TIN_SUMS", request.param)
    else:
        monkeypatch.delenv("SETSM_VLL_TIN_SUMS", raising=False)
    return request.param


@pytest.mark.parametrize("name", sorted(mg.GOLDEN_TINB))
def test_matches_reference_fixture(gpu_ctx, name, sums_mode):
    inp, pts, tris, oncc, z = mg.tinb_case(name)
    it, fb, cbl, hint = mg.GOLDEN_TINB[name]["call"]
    det, counts, zext = fresh_out(len(pts))
    gpu_ctx.blunder_detection_tin(inp, it, oncc, fb, cbl, hint, pts, det, tris, counts, zext)
    assert_same(pts, det, inp.gridpt3, counts, zext, z["pts"].view(abi.POINT3_DTYPE),
                z["detected"], z["gp3"].view(abi.UGRID_DTYPE), z["counts"], z["zext"])


@pytest.mark.skipif(not refpy.available(), reason="reference build not available")
@pytest.mark.parametrize("kw,call", [
    (dict(seed=41, size=768, nodes=40, res=7.0), (1, True, 1, 60.0)),
    (dict(seed=42, size=768, nodes=40, res=7.0, point_frac=0.15), (2, True, 4, 40.0)),
    (dict(seed=43, size=768, nodes=40, res=7.0), (4, True, 1, 60.0)),
    (dict(seed=44, size=768, nodes=24, res=12.0, L=1, template=15), (1, True, 2, 80.0)),
    (dict(seed=45, size=768, nodes=24, res=16.0, L=2, template=15), (3, False, 1, 70.0)),
    (dict(seed=46, size=768, nodes=16, res=24.0, L=3, template=15), (4, True, 1, 35.0)),
    (dict(seed=47, size=768, nodes=16, res=24.0, L=4, template=15, flagged_frac=0.3),
     (2, True, 1, 25.0)),
])
def test_matches_reference_build(gpu_ctx, kw, call, sums_mode):
    import copy
    inp, pts, tris, oncc = cases.make_tin_blunder_case(**kw)
    ref = copy.copy(inp)
    ref.gridpt3 = inp.gridpt3.copy()
    r_pts = pts.copy()
    r_det, r_counts, r_zext = fresh_out(len(pts))
    it, fb, cbl, hint = call
    refpy.blunder_detection_tin(ref, it, oncc.copy(), fb, cbl, hint, r_pts, r_det, tris.copy(),
                                r_counts, r_zext)
    det, counts, zext = fresh_out(len(pts))
    gpu_ctx.blunder_detection_tin(inp, it, oncc, fb, cbl, hint, pts, det, tris, counts, zext)
    assert_same(pts, det, inp.gridpt3, counts, zext, r_pts, r_det, ref.gridpt3, r_counts, r_zext)


@pytest.mark.skipif(not refpy.available(), reason="reference build not available")
def test_cpp_dropin_through_reference_structures(gpu_ctx):
    inp, pts, tris, oncc, z = mg.tinb_case("tinb_l3")
    it, fb, cbl, hint = mg.GOLDEN_TINB["tinb_l3"]["call"]
    fn = C.cast(getattr(vll.load(), DROPIN), C.c_void_p).value
    det, counts, zext = fresh_out(len(pts))
    assert refpy.blunder_detection_tin(inp, it, oncc, fb, cbl, hint, pts, det, tris, counts, zext,
                                       fn_addr=fn) == 1
    assert_same(pts, det, inp.gridpt3, counts, zext, z["pts"].view(abi.POINT3_DTYPE),
                z["detected"], z["gp3"].view(abi.UGRID_DTYPE), z["counts"], z["zext"])


def test_level0_iteration3_does_nothing(gpu_ctx):
    inp, pts, tris, oncc, _ = mg.tinb_case("tinb_l0")
    before = pts.copy()
    det, counts, zext = fresh_out(len(pts))
    gpu_ctx.blunder_detection_tin(inp, 3, oncc, True, 1, 60.0, pts, det, tris, counts, zext)
    assert np.array_equal(pts["flag"], before["flag"]) and not det.any() and not counts.any()


def test_device_entry_matches_fixture(gpu_ctx):
    import torch
    inp, pts, tris, oncc, z = mg.tinb_case("tinb_l1_anchor")
    it, fb, cbl, hint = mg.GOLDEN_TINB["tinb_l1_anchor"]["call"]
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).cuda()
    d_pts, d_tris, d_g, d_o = dev(pts), dev(tris), dev(inp.gridpt3), dev(oncc)
    d_det = torch.zeros(len(pts), dtype=torch.uint8, device="cuda")
    _, counts, zext = fresh_out(len(pts))
    gpu_ctx.blunder_detection_tin_device(inp.desc(), it, d_o.data_ptr(), fb, cbl, hint,
                                         d_pts.data_ptr(), d_det.data_ptr(), len(pts),
                                         d_tris.data_ptr(), len(tris), d_g.data_ptr(), counts,
                                         zext)
    torch.cuda.synchronize()
    assert_same(d_pts.cpu().numpy().view(abi.POINT3_DTYPE), d_det.cpu().numpy(),
                d_g.cpu().numpy().view(abi.UGRID_DTYPE), counts, zext,
                z["pts"].view(abi.POINT3_DTYPE), z["detected"], z["gp3"].view(abi.UGRID_DTYPE),
                z["counts"], z["zext"])


def test_wide_band_reruns_the_point_pass(gpu_ctx, monkeypatch):
    """With the band widened by 1 m some comparison falls inside it: the pass
    is undone and re-run (counted), and the result is still the reference's."""
    monkeypatch.setenv("SETSM_VLL_TIN_SUMS", "wideband")
    inp, pts, tris, oncc, z = mg.tinb_case("tinb_l0")
    it, fb, cbl, hint = mg.GOLDEN_TINB["tinb_l0"]["call"]
    det, counts, zext = fresh_out(len(pts))
    before = vll.load().vll_tin_rerun_count(gpu_ctx._h)
    gpu_ctx.blunder_detection_tin(inp, it, oncc, fb, cbl, hint, pts, det, tris, counts, zext)
    assert vll.load().vll_tin_rerun_count(gpu_ctx._h) == before + 1
    assert_same(pts, det, inp.gridpt3, counts, zext, z["pts"].view(abi.POINT3_DTYPE),
                z["detected"], z["gp3"].view(abi.UGRID_DTYPE), z["counts"], z["zext"])


@pytest.mark.skipif(not refpy.available(), reason="reference build not available")
@pytest.mark.parametrize("seed", [61, 62])
def test_crowded_points_and_repeated_vertices(gpu_ctx, seed):
    """Triangle lists beyond the Delaunay ones: two points in more than 32
    triangles (the warp's selection of the first 30 in triangle order),
    triangles listing a point twice (kept twice, as the reference's lists do)
    and a vertex past the points.  A triangle (a, a, b) has a zero normal
    when point b evaluates it, where the reference's SetNormalAngle leaves its
    angle unset (SubFunctions.cpp:2999-3007), so b is a point the pass skips
    (flag 1), and no vertex is point 0 (the unset third index)."""
    import copy
    inp, pts, tris, oncc = cases.make_tin_blunder_case(seed=seed, size=768, nodes=40, res=7.0)
    rng = np.random.default_rng(seed)
    n = len(pts)
    extra = []
    for hub in (3, n // 2):
        others = np.setdiff1d(np.arange(1, n), [hub])
        for _ in range(45):
            j, k = rng.choice(others, 2, replace=False)
            extra.append((hub, j, k) if rng.random() < 0.5 else (j, hub, k))
    skipped = np.flatnonzero(pts["flag"] == 1)
    active = np.setdiff1d(np.flatnonzero(pts["flag"] != 1), [0])
    for _ in range(12):
        extra.append((rng.choice(active),) * 2 + (rng.choice(skipped[skipped > 0]),))
    extra.append((1, 2, n + 5))
    ext = np.zeros(len(extra), dtype=tris.dtype)
    ext["a"], ext["b"], ext["c"] = np.array(extra).T
    mixed = np.concatenate([tris[:len(tris) // 2], ext, tris[len(tris) // 2:]])
    ref = copy.copy(inp)
    ref.gridpt3 = inp.gridpt3.copy()
    r_pts, (r_det, r_counts, r_zext) = pts.copy(), fresh_out(n)
    refpy.blunder_detection_tin(ref, 1, oncc.copy(), True, 1, 60.0, r_pts, r_det, mixed.copy(),
                                r_counts, r_zext)
    det, counts, zext = fresh_out(n)
    gpu_ctx.blunder_detection_tin(inp, 1, oncc, True, 1, 60.0, pts, det, mixed, counts, zext)
    assert_same(pts, det, inp.gridpt3, counts, zext, r_pts, r_det, ref.gridpt3, r_counts, r_zext)


def test_invalid_inputs_fail_and_leave_buffers(gpu_ctx):
    """A point whose grid node lies outside the grid, a negative Hinterval and
    a missing output fail with VLL_ERR_INVALID; the host buffers keep their
    contents."""
    inp, pts, tris, oncc, _ = mg.tinb_case("tinb_l0")
    it, fb, cbl, hint = mg.GOLDEN_TINB["tinb_l0"]["call"]
    g0 = inp.gridpt3.copy()
    bad = pts.copy()
    bad["y"][5] = inp.boundary[3] + 50 * inp.grid_resolution   # rows past the top
    before = bad.copy()
    det, counts, zext = fresh_out(len(pts))
    with pytest.raises(vll.VLLError) as e:
        gpu_ctx.blunder_detection_tin(inp, it, oncc, fb, cbl, hint, bad, det, tris, counts, zext)
    assert e.value.code == abi.VLL_ERR_INVALID
    # fields, not bytes: numpy's copy of a padded record leaves the padding
    for f in ("x", "y", "z", "flag"):
        assert np.array_equal(bad[f], before[f])
    assert not det.any() and not counts.any()
    assert cases.field_mismatch(inp.gridpt3, g0) == {}
    with pytest.raises(vll.VLLError):
        gpu_ctx.blunder_detection_tin(inp, it, oncc, fb, cbl, -1.0, pts, det, tris, counts, zext)
    # the context stays usable
    gpu_ctx.blunder_detection_tin(inp, it, oncc, fb, cbl, hint, pts, det, tris, counts, zext)


@pytest.mark.skipif(not refpy.available(), reason="reference build not available")
@pytest.mark.parametrize("big", [1e308, float("inf")])
def test_overflowing_height_sums_rerun_exactly(gpu_ctx, big, monkeypatch):
    """One point with a huge or infinite height makes the edges' height
    difference sums overflow: the device sets the threshold band to
    [-inf, inf], so the point pass is re-run with the sequential sums (counted)
    and the result is the reference build's."""
    import copy
    monkeypatch.delenv("SETSM_VLL_TIN_SUMS", raising=False)
    inp, pts, tris, oncc = cases.make_tin_blunder_case(seed=41, size=768, nodes=40, res=7.0)
    pts["z"][len(pts) // 2] = big
    ref = copy.copy(inp)
    ref.gridpt3 = inp.gridpt3.copy()
    r_pts = pts.copy()
    r_det, r_counts, r_zext = fresh_out(len(pts))
    refpy.blunder_detection_tin(ref, 1, oncc.copy(), True, 1, 60.0, r_pts, r_det, tris.copy(),
                                r_counts, r_zext)
    det, counts, zext = fresh_out(len(pts))
    before = vll.load().vll_tin_rerun_count(gpu_ctx._h)
    gpu_ctx.blunder_detection_tin(inp, 1, oncc, True, 1, 60.0, pts, det, tris, counts, zext)
    assert vll.load().vll_tin_rerun_count(gpu_ctx._h) == before + 1
    assert_same(pts, det, inp.gridpt3, counts, zext, r_pts, r_det, ref.gridpt3, r_counts, r_zext)
