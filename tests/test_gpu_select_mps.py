"""SelectMPs on the GPU (vll_selectmps.cu) against the reference
(setsm_code.cpp:8535-8895): the fixtures made by the reference build, the
reference build itself on the matching results of the parity cases with the
level, the SGM / RA switches and the call arguments varied, and the C++
drop-in with the reference's signature.  The points (in order) and every
UGRID field must be identical."""
import copy
import ctypes as C

import numpy as np
import pytest

from oracle import refpy
from setsm_b200 import abi, vll
from tests import cases
from tests.golden import make_golden as mg

pytestmark = pytest.mark.gpu

DROPIN = ("_Z9SelectMPsPK11ProjectInfoR12taglevelinfoPK12tagNCCresultP10UpdateGridddddididPSt6"
          "vectorI11tagD3DPointSaISA_EE")


def same_points(a, b):
    return len(a) == len(b) and all(np.array_equal(a[f], b[f]) for f in ("x", "y", "z", "flag"))


@pytest.mark.parametrize("name", sorted(mg.GOLDEN_SELECT))
def test_matches_reference_fixture(gpu_ctx, name):
    inp, ncc, z = mg.select_case(name)
    pts = gpu_ctx.select_mps(inp, ncc, *mg.GOLDEN_SELECT[name]["args"])
    assert same_points(pts, z["pts"].view(abi.POINT3_DTYPE))
    assert len(pts) == int(z["ret"])
    assert cases.field_mismatch(mg.clean(inp.gridpt3), z["gp3"].view(abi.UGRID_DTYPE)) == {}


ARGS = [(0.6, 0.2, 0.8, 0.7, 1, 1.5, 1, 10.0), (0.3, 0.25, 0.3, 0.2, 3, 2.0, 3, 3.0),
        (0.35, 0.3, 0.35, 0.25, 4, 1.0, 2, 6.0)]


@pytest.mark.skipif(not refpy.available(), reason="reference build not available")
@pytest.mark.parametrize("name", ["m7", "v7_it2", "l3_m"])
@pytest.mark.parametrize("level", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("k", range(len(ARGS)))
def test_matches_reference_build(gpu_ctx, name, level, k):
    inp, ncc = cases.make_select_case(name, seed=100 + level)
    inp.pyramid_step = level
    inp.sgm_py = 1 if k == 1 else -1
    inp.is_ra = k == 2 and level == 4
    ref = copy.copy(inp)
    ref.gridpt3 = inp.gridpt3.copy()
    r, want = refpy.select_mps(ref, ncc, *ARGS[k])
    got = gpu_ctx.select_mps(inp, ncc, *ARGS[k])
    assert r == len(want)
    assert same_points(got, want)
    assert cases.field_mismatch(mg.clean(inp.gridpt3), mg.clean(ref.gridpt3)) == {}


@pytest.mark.skipif(not refpy.available(), reason="reference build not available")
def test_cpp_dropin_through_reference_structures(gpu_ctx):
    inp, ncc, z = mg.select_case("select_l1")
    fn = C.cast(getattr(vll.load(), DROPIN), C.c_void_p).value
    r, pts = refpy.select_mps(inp, ncc, *mg.GOLDEN_SELECT["select_l1"]["args"], fn_addr=fn)
    assert r == int(z["ret"])
    assert same_points(pts, z["pts"].view(abi.POINT3_DTYPE))
    assert cases.field_mismatch(mg.clean(inp.gridpt3), z["gp3"].view(abi.UGRID_DTYPE)) == {}


def test_capacity_error_leaves_inputs(gpu_ctx):
    """More points than the buffer holds: a status code, nothing written."""
    inp, ncc, z = mg.select_case("select_l0")
    before = inp.gridpt3.copy()
    d = inp.desc()
    out = np.zeros(4, dtype=abi.POINT3_DTYPE)
    n = C.c_int64()
    rc = vll.load().vll_select_mps(gpu_ctx._h, C.byref(d), ncc.ctypes.data,
                                   inp.gridpt3.ctypes.data, *map(float, (0.6, 0.2, 0.8, 0.7)), 1,
                                   1.5, 1, 10.0, out.ctypes.data, len(out), C.byref(n))
    assert rc == abi.VLL_ERR_CAPACITY
    assert n.value == int(z["ret"]) > 4
    assert cases.field_mismatch(inp.gridpt3, before) == {}


@pytest.mark.parametrize("name", sorted(mg.GOLDEN_SELECT))
def test_device_entry_point(gpu_ctx, name):
    import torch
    inp, ncc, z = mg.select_case(name)
    io, keep = cases.device_level(torch, inp, ncc)
    d_pts = torch.zeros(inp.n * 32, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    n = gpu_ctx.select_mps_device(io[0], io[2], io[1], d_pts.data_ptr(), inp.n,
                                  *mg.GOLDEN_SELECT[name]["args"])
    assert n == int(z["ret"])
    pts = d_pts.cpu().numpy().view(abi.POINT3_DTYPE)[:n]
    assert same_points(pts, z["pts"].view(abi.POINT3_DTYPE))
    gp3 = cases.from_device(keep["gp3"], abi.UGRID_DTYPE)
    assert cases.field_mismatch(mg.clean(gp3), z["gp3"].view(abi.UGRID_DTYPE)) == {}
