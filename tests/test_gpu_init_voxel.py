"""InitializeVoxel on the GPU (vll_initvoxel.cu) against the reference's
(setsm_code.cpp:5759-6012), on the voxel-route parity cases: the first
iteration (no previous rows) and the second one from the state the
reference's own first iteration (InitializeVoxel, VerticalLineLocus, AWNCC)
leaves, through the host and the device entry points; and the device-resident
voxel route (InitializeVoxel -> VerticalLineLocus on the device) against the
reference's.  Every NCCresult / UGRID field and every voxel must be identical."""
import copy

import numpy as np
import pytest

from oracle import refpy
from setsm_b200 import abi
from tests import cases

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refpy.available(), reason="reference build not available")]

VOXEL_CASES = ["v7_gncc", "v11", "l2_combined", "l2_max", "v7_3img", "v7_3img_unsel"]


# the SGM route too (AWNCC with semi-global aggregation at level 0)
SGM_CASE = dict(size=512, nodes=24, res=8.0, n_heights=32, cmr=False, sgm=1, ortho_frac=0.5)


def first_iteration(name):
    """(inputs at iteration 2, ncc, voxels) after the reference's iteration 1
    of case `name` (a key of tests/cases.py:CASES, or "sgm")."""
    inp = cases.make_case(**(SGM_CASE if name == "sgm" else cases.CASES[name]))
    inp = copy.copy(inp)
    inp.gridpt3 = inp.gridpt3.copy()
    inp.iteration = 1
    ncc = inp.new_nccresult()
    vox = refpy.initialize_voxel(inp, ncc, None)
    refpy.vertical_line_locus(inp, ncc, vox)
    refpy.awncc(inp, ncc, vox)
    inp.iteration = 2
    return inp, ncc, vox


def compare(gpu_ctx, inp, ncc, vox):
    ref = copy.copy(inp)
    ref.gridpt3 = inp.gridpt3.copy()
    ref_ncc = ncc.copy()
    want = refpy.initialize_voxel(ref, ref_ncc, None if vox is None else vox.copy())
    got_ncc = ncc.copy()
    got = gpu_ctx.initialize_voxel(inp, got_ncc, vox)
    assert cases.field_mismatch(got_ncc, ref_ncc) == {}
    assert cases.field_mismatch(inp.gridpt3, ref.gridpt3) == {}
    assert len(got) == len(want)
    assert cases.field_mismatch(got, want) == {}
    return got_ncc, got


@pytest.mark.parametrize("name", VOXEL_CASES)
def test_first_iteration(gpu_ctx, name):
    inp = cases.make_case(**cases.CASES[name])
    inp.iteration = 1
    compare(gpu_ctx, inp, inp.new_nccresult(), None)


@pytest.mark.parametrize("name", VOXEL_CASES)
def test_second_iteration_carries_rows(gpu_ctx, name):
    inp, ncc, vox = first_iteration(name)
    compare(gpu_ctx, inp, ncc, vox)


@pytest.mark.parametrize("name", ["v7_gncc", "l2_combined", "sgm"])
def test_device_voxel_route_matches_reference(gpu_ctx, name):
    """InitializeVoxel, VerticalLineLocus and AWNCC on device-resident data,
    the offsets of the first feeding the others."""
    import torch
    inp, ncc, vox = first_iteration(name)
    ref = copy.copy(inp)
    ref.gridpt3 = inp.gridpt3.copy()
    ref_ncc = ncc.copy()
    want_vox = refpy.initialize_voxel(ref, ref_ncc, vox.copy())
    refpy.vertical_line_locus(ref, ref_ncc, want_vox)
    io, keep = cases.device_level(torch, inp, ncc)
    d_vin = torch.from_numpy(vox.view(np.uint8).copy()).cuda()
    cap = len(want_vox) + 64
    d_vout = torch.zeros(cap * 4, dtype=torch.uint8, device="cuda")
    d_off = torch.zeros(inp.n + 1, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    n = gpu_ctx.initialize_voxel_device(io[0], io[1], io[2], d_vin.data_ptr(), d_vout.data_ptr(),
                                        cap, d_off.data_ptr())
    assert n == len(want_vox)
    gpu_ctx.vertical_line_locus_device(io[0], io[1], io[2], d_vout.data_ptr(), d_off.data_ptr(),
                                       kernel="split")
    gpu_ctx.awncc_device(io[0], io[1], io[2], d_vout.data_ptr(), d_off.data_ptr())
    refpy.awncc(ref, ref_ncc, want_vox)
    torch.cuda.synchronize()
    got_ncc = cases.from_device(keep["ncc"], abi.NCCRESULT_DTYPE)
    got_vox = d_vout.cpu().numpy().view(abi.VOXEL_DTYPE)[:n]
    assert cases.field_mismatch(got_ncc, ref_ncc) == {}
    assert cases.field_mismatch(got_vox, want_vox) == {}
    assert cases.field_mismatch(cases.from_device(keep["gp3"], abi.UGRID_DTYPE),
                                ref.gridpt3) == {}


DROPIN_IV = "_Z15InitializeVoxelPK11ProjectInfoPP12tagVoxelinfoR12taglevelinfoP10UpdateGridP12tagNCCresultiPKd"
DROPIN_AWNCC = "_Z5AWNCCP11ProjectInfoPP12tagVoxelinfo8tagCSizeP10UpdateGridP12tagNCCresultdhhi"


@pytest.mark.parametrize("name", ["v7_gncc", "v7_3img"])
def test_cpp_dropins_through_reference_structures(gpu_ctx, name):
    """InitializeVoxel and AWNCC drop-ins (setsm_code.hpp:75, :91) called the
    way Matching_SETSM calls them (VOXEL** rows), around the reference's own
    VerticalLineLocus: the same NCCresult, UGRID and voxels as the
    reference's iteration."""
    import ctypes as C
    from setsm_b200 import vll
    L = vll.load()
    fn_iv = C.cast(getattr(L, DROPIN_IV), C.c_void_p).value
    fn_aw = C.cast(getattr(L, DROPIN_AWNCC), C.c_void_p).value
    inp, ncc, vox = first_iteration(name)
    ref = copy.copy(inp)
    ref.gridpt3 = inp.gridpt3.copy()
    ref_ncc = ncc.copy()
    want_vox = refpy.initialize_voxel(ref, ref_ncc, vox.copy())
    refpy.vertical_line_locus(ref, ref_ncc, want_vox)
    refpy.awncc(ref, ref_ncc, want_vox)
    got_ncc = ncc.copy()
    got_vox = refpy.call_initialize_voxel(fn_iv, inp, got_ncc, vox.copy())
    refpy.vertical_line_locus(inp, got_ncc, got_vox)
    refpy.call_awncc(fn_aw, inp, got_ncc, got_vox)
    assert cases.field_mismatch(got_ncc, ref_ncc) == {}
    assert cases.field_mismatch(got_vox, want_vox) == {}
    assert cases.field_mismatch(inp.gridpt3, ref.gridpt3) == {}
