"""The TIN-triangle orthoimage height search on the GPU (vll_orthotin.cu)
against the reference: VerticalLineLocus_Ortho (setsm_code.cpp:8234-8533)
and Ortho_blunder (:8028-8232), through the C ABI, the C++ drop-ins with the
reference's signatures, and the device entry point.  Points, triangles' effects
and every UGRID field must be identical; a single search's F_sncc (an FP64
mean of correlations) within 1e-9, as the map projection's libm calls may
differ from the host's in the last bit on rare raster cells."""
import copy
import ctypes as C

import numpy as np
import pytest

from oracle import refpy
from setsm_b200 import abi, vll
from tests import cases
from tests.golden import make_golden as mg

pytestmark = pytest.mark.gpu

SNCC_TOL = 1e-9
DROPINS = {
    "ortho": "_Z23VerticalLineLocus_OrthoP11ProjectInfoR12taglevelinfodPd11tagD3DPointS4_S4_"
             "P10UpdateGridiS3_",
    "blunder": "_Z13Ortho_blunderP11ProjectInfoR12taglevelinfodP11tagD3DPointiP12tagUI3DPointiP10"
               "UpdateGrid",
}


def same_points(a, b):
    return all(np.array_equal(a[f], b[f]) for f in ("x", "y", "z", "flag"))


@pytest.mark.parametrize("name", sorted(mg.GOLDEN_TIN))
def test_ortho_blunder_matches_reference_fixture(gpu_ctx, name):
    inp, pts, tris, z = mg.tin_case(name)
    assert mg.image_digest(inp) == str(z["img_digest"])
    rounds = gpu_ctx.ortho_blunder(inp, mg.GOLDEN_TIN[name]["mpp"], pts, tris)
    assert 1 <= rounds <= 200
    assert same_points(pts, z["pts"].view(abi.POINT3_DTYPE))
    assert cases.field_mismatch(mg.clean(inp.gridpt3), z["gp3"].view(abi.UGRID_DTYPE)) == {}


@pytest.mark.skipif(not refpy.available(), reason="reference build not available")
@pytest.mark.parametrize("kw,mpp", [
    (dict(seed=31, size=768, nodes=40, res=7.0), 1.0),
    (dict(seed=32, size=768, nodes=40, res=7.0, point_frac=0.12), 1.5),
    (dict(seed=33, size=768, nodes=24, res=12.0, L=1, template=15), 2.5),
    (dict(seed=34, size=768, nodes=24, res=16.0, L=2, template=15, range_m=80.0), 3.0),
    (dict(seed=35, size=512, nodes=32, res=8.0, n_images=3, anchor_frac=0.4), 1.5),
    # sparse points: triangles of up to ~1200 cells, many with more than the
    # 256 inside cells a warp stages (the per-height box path)
    (dict(seed=37, size=768, nodes=128, res=2.0, point_frac=0.002), 1.5),
])
def test_ortho_blunder_matches_reference_build(gpu_ctx, kw, mpp):
    inp, pts, tris = cases.make_tin_case(**kw)
    ref = copy.copy(inp)
    ref.gridpt3 = inp.gridpt3.copy()
    ref_pts = pts.copy()
    refpy.ortho_blunder(ref, mpp, ref_pts, tris.copy())
    gpu_ctx.ortho_blunder(inp, mpp, pts, tris)
    assert same_points(pts, ref_pts)
    assert cases.field_mismatch(mg.clean(inp.gridpt3), mg.clean(ref.gridpt3)) == {}


def searchable(inp, pts, tris):
    """(three points, target node) of every triangle with two anchored
    vertices, as Ortho_blunder's first round chooses them."""
    g = inp.gridpt3
    b, gs, w = inp.boundary, inp.grid_resolution, inp.grid_width
    node = (((pts["y"] - b[1]) / gs + 0.5).astype(np.int64) * w
            + ((pts["x"] - b[0]) / gs + 0.5).astype(np.int64))
    out = []
    for t in tris:
        v = [int(t["a"]), int(t["b"]), int(t["c"])]
        f = [int(g["anchor_flag"][node[i]]) for i in v]
        if sum(x in (1, 3) for x in f) != 2:
            continue
        k = 0 if f[0] == 2 else (1 if f[1] == 2 else 2)
        order = [i for j, i in enumerate(v) if j != k] + [v[k]]
        out.append((pts[order].copy(), int(node[v[k]])))
    return out


@pytest.mark.skipif(not refpy.available(), reason="reference build not available")
@pytest.mark.parametrize("kw,mpp", [
    (dict(seed=41, size=768, nodes=40, res=7.0), 1.5),
    (dict(seed=42, size=768, nodes=24, res=16.0, L=2, template=15), 1.0),
    (dict(seed=43, size=768, nodes=128, res=2.0, point_frac=0.0015), 1.5),
])
def test_single_search_matches_reference(gpu_ctx, kw, mpp):
    inp, pts, tris = cases.make_tin_case(**kw)
    jobs = searchable(inp, pts, tris)[:40]
    assert len(jobs) >= 10
    found = 0
    for three, target in jobs:
        want = refpy.vll_ortho(inp, mpp, three, target)
        got = gpu_ctx.vertical_line_locus_ortho(inp, mpp, three, target)
        assert got[0] == want[0] and got[1] == want[1], (got, want)
        if want[1] != -9999.0:
            found += 1
            assert abs(got[2] - want[2]) <= SNCC_TOL
        else:
            assert np.isnan(got[2]) and np.isnan(want[2])
    assert found > 0


@pytest.mark.skipif(not refpy.available(), reason="reference build not available")
def test_cpp_dropins_through_reference_structures(gpu_ctx):
    L = vll.load()
    inp, pts, tris, z = mg.tin_case("tin_l0")
    mpp = mg.GOLDEN_TIN["tin_l0"]["mpp"]
    three, target = searchable(inp, pts, tris)[0]
    fn = C.cast(getattr(L, DROPINS["ortho"]), C.c_void_p).value
    want = refpy.vll_ortho(inp, mpp, three, target)
    got = refpy.call_vll_ortho(fn, inp, mpp, three, target)
    assert got[:2] == want[:2] and (np.isnan(want[2]) or abs(got[2] - want[2]) <= SNCC_TOL)
    fn = C.cast(getattr(L, DROPINS["blunder"]), C.c_void_p).value
    assert refpy.call_ortho_blunder(fn, inp, mpp, pts, tris) == len(pts)
    assert same_points(pts, z["pts"].view(abi.POINT3_DTYPE))
    assert cases.field_mismatch(mg.clean(inp.gridpt3), z["gp3"].view(abi.UGRID_DTYPE)) == {}


def test_device_entry_point(gpu_ctx):
    import torch
    inp, pts, tris, z = mg.tin_case("tin_l1_3img")
    io, keep = cases.device_level(torch, inp, inp.new_nccresult())
    d_pts = torch.from_numpy(pts.view(np.uint8).copy()).cuda()
    d_tris = torch.from_numpy(tris.view(np.uint8).copy()).cuda()
    torch.cuda.synchronize()
    rounds = gpu_ctx.ortho_blunder_device(io[0], mg.GOLDEN_TIN["tin_l1_3img"]["mpp"],
                                          d_pts.data_ptr(), len(pts), d_tris.data_ptr(),
                                          len(tris), io[1])
    assert rounds >= 1
    got_pts = d_pts.cpu().numpy().view(abi.POINT3_DTYPE)
    got_gp3 = cases.from_device(keep["gp3"], abi.UGRID_DTYPE)
    assert same_points(got_pts, z["pts"].view(abi.POINT3_DTYPE))
    assert cases.field_mismatch(mg.clean(got_gp3), z["gp3"].view(abi.UGRID_DTYPE)) == {}


def test_vertex_outside_the_grid_is_an_error(gpu_ctx):
    """A vertex whose grid node index falls outside the UGRID array (the
    reference would read past it) is refused with a status code."""
    inp, pts, tris, _ = mg.tin_case("tin_l0")
    pts["y"][int(tris["a"][0])] = inp.boundary[3] + 10 * inp.grid_resolution
    with pytest.raises(vll.VLLError):
        gpu_ctx.ortho_blunder(inp, 1.5, pts, tris)
