"""SetHeightRange on the GPU (vll_heightrange.cu) against the reference
(setsm_code.cpp:9851-10255): the fixtures in tests/golden made by the
reference build, the reference build itself where present, and the C++
drop-in with the reference's signature.  Every field of the returned grid
and the height extent must be identical."""
import ctypes as C

import numpy as np
import pytest

from oracle import refpy
from setsm_b200 import abi, vll
from tests import cases
from tests.golden import make_golden as mg

pytestmark = pytest.mark.gpu

DROPIN = ("_Z14SetHeightRangeP11ProjectInfoR12taglevelinfoP12tagNCCresultiiP10UpdateGridiPdS7_"
          "P11tagD3DPointPK12tagUI3DPointdb")


@pytest.mark.parametrize("name", sorted(mg.GOLDEN_RANGE))
def test_matches_reference_fixture(gpu_ctx, name):
    v = mg.GOLDEN_RANGE[name]
    inp, pts, tris, z = mg.range_case(name)
    out, ext = gpu_ctx.set_height_range(inp, pts, tris, v["iteration"], v["mpp"], v["lcmr"],
                                        v.get("sigma", 0.0))
    assert cases.field_mismatch(mg.clean(out), z["result"].view(abi.UGRID_DTYPE)) == {}
    assert ext == tuple(z["extent"])


@pytest.mark.skipif(not refpy.available(), reason="reference build not available")
@pytest.mark.parametrize("kw,it,mpp,lcmr,dem", [
    (dict(seed=61, size=768, nodes=40, res=7.0), 1, 1.5, False, 2.0),
    (dict(seed=62, size=768, nodes=40, res=7.0, point_frac=0.1), 2, 0.8, True, 1.0),
    (dict(seed=63, size=768, nodes=24, res=12.0, L=1, template=15), 2, 2.5, False, 4.0),
    (dict(seed=64, size=768, nodes=24, res=16.0, L=2, template=15), 5, 1.5, False, 2.0),
    (dict(seed=65, size=768, nodes=16, res=24.0, L=3, template=15), 1, 3.0, False, 2.0),
    (dict(seed=66, size=768, nodes=16, res=24.0, L=4, template=15, range_m=120.0), 3, 2.0, True,
     8.0),
    (dict(seed=67, size=512, nodes=32, res=8.0, n_images=3, flag4_frac=0.5), 2, 1.2, False, 2.0),
])
def test_matches_reference_build(gpu_ctx, kw, it, mpp, lcmr, dem):
    inp, pts, tris = cases.make_range_case(**kw)
    inp.dem_resolution = dem
    want, wext = refpy.set_height_range(inp, pts, tris, it, mpp, lcmr)
    got, gext = gpu_ctx.set_height_range(inp, pts, tris, it, mpp, lcmr)
    assert cases.field_mismatch(mg.clean(got), mg.clean(want)) == {}
    assert gext == wext


@pytest.mark.skipif(not refpy.available(), reason="reference build not available")
def test_cpp_dropin_through_reference_structures(gpu_ctx):
    v = mg.GOLDEN_RANGE["range_l1_seed"]
    inp, pts, tris, z = mg.range_case("range_l1_seed")
    fn = C.cast(getattr(vll.load(), DROPIN), C.c_void_p).value
    out, ext = refpy.set_height_range(inp, pts, tris, v["iteration"], v["mpp"], v["lcmr"],
                                      v["sigma"], fn_addr=fn)
    assert cases.field_mismatch(mg.clean(out), z["result"].view(abi.UGRID_DTYPE)) == {}
    assert ext == tuple(z["extent"])


def test_empty_tin(gpu_ctx):
    """No triangles: every node goes through the neighbour pass only."""
    inp, pts, tris, _ = mg.range_case("range_l0")
    out, ext = gpu_ctx.set_height_range(inp, pts, tris[:0], 1, 1.5, False)
    assert np.all(out["Height"] == -1000)


@pytest.mark.parametrize("name", sorted(mg.GOLDEN_RANGE))
def test_device_entry_point(gpu_ctx, name):
    import torch
    v = mg.GOLDEN_RANGE[name]
    inp, pts, tris, z = mg.range_case(name)
    d_pts = torch.from_numpy(pts.view(np.uint8).copy()).cuda()
    d_tris = torch.from_numpy(tris.view(np.uint8).copy()).cuda()
    d_gp3 = torch.from_numpy(inp.gridpt3.view(np.uint8).copy()).cuda()
    d_out = torch.zeros(inp.n * 20, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    ext = gpu_ctx.set_height_range_device(inp.desc(), d_pts.data_ptr(), len(pts),
                                          d_tris.data_ptr(), len(tris), d_gp3.data_ptr(),
                                          d_out.data_ptr(), v["iteration"], v["mpp"], v["lcmr"],
                                          v.get("sigma", 0.0))
    out = d_out.cpu().numpy().view(abi.UGRID_DTYPE)
    assert cases.field_mismatch(mg.clean(out), z["result"].view(abi.UGRID_DTYPE)) == {}
    assert ext == tuple(z["extent"])
