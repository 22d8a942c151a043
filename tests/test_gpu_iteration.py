"""One Matching_SETSM iteration (setsm_code.cpp:3827-4368) device-resident
from InitializeVoxel to SetHeightRange: InitializeVoxel -> VerticalLineLocus
-> AWNCC -> SelectMPs -> TINCreate_list -> SetHeightRange on device buffers,
nothing crossing the bus between the steps, against the reference build's
same six functions on the host.  Records, voxel rows, matched points,
triangles (in order), the next iteration's grid and its height extent must be
identical."""
import copy

import numpy as np
import pytest

from oracle import refpy
from setsm_b200 import abi
from tests import cases
from tests.test_gpu_init_voxel import first_iteration

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refpy.available(), reason="reference build not available")]

SELECT_ARGS = (0.6, 0.2, 0.8, 0.7, 2, 1.5, 1, 10.0)   # iteration 2
MPP = 1.5


@pytest.mark.parametrize("name", ["v7_gncc", "v11"])
def test_iteration_on_the_device_matches_reference(gpu_ctx, name):
    import torch
    inp, ncc, vox = first_iteration(name)             # the reference's iteration 1
    it = inp.iteration
    # ---- the reference's iteration on the host ----
    ref = copy.copy(inp)
    ref.gridpt3 = inp.gridpt3.copy()
    r_ncc = ncc.copy()
    r_vox = refpy.initialize_voxel(ref, r_ncc, vox.copy())
    refpy.vertical_line_locus(ref, r_ncc, r_vox)
    refpy.awncc(ref, r_ncc, r_vox)
    _, r_pts = refpy.select_mps(ref, r_ncc, *SELECT_ARGS)
    r_tris = refpy.tin_create(r_pts, inp.boundary, inp.grid_resolution)
    r_grid, r_ext = refpy.set_height_range(ref, r_pts, r_tris, it, MPP, True)
    assert len(r_pts) >= 3 and len(r_tris) > 0
    # ---- the same iteration on device buffers ----
    io, keep = cases.device_level(torch, inp, ncc)
    desc, d_g, d_n = io
    d_vin = torch.from_numpy(vox.view(np.uint8).copy()).cuda()
    cap = len(r_vox) + 64
    d_vox = torch.zeros(cap * abi.VOXEL_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    d_off = torch.zeros(inp.n + 1, dtype=torch.int64, device="cuda")
    d_pts = torch.zeros(inp.n * abi.POINT3_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    d_res = torch.zeros(inp.n * abi.UGRID_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    n_vox = gpu_ctx.initialize_voxel_device(desc, d_g, d_n, d_vin.data_ptr(), d_vox.data_ptr(),
                                            cap, d_off.data_ptr())
    gpu_ctx.vertical_line_locus_device(desc, d_g, d_n, d_vox.data_ptr(), d_off.data_ptr(),
                                       kernel="split")
    gpu_ctx.awncc_device(desc, d_g, d_n, d_vox.data_ptr(), d_off.data_ptr())
    n_pts = gpu_ctx.select_mps_device(desc, d_n, d_g, d_pts.data_ptr(), inp.n, *SELECT_ARGS)
    tcap = 2 * n_pts + 16
    d_tris = torch.zeros(tcap * abi.TRI_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    n_tris = gpu_ctx.tin_create_device(d_pts.data_ptr(), n_pts, inp.boundary,
                                       inp.grid_resolution, d_tris.data_ptr(), tcap)
    ext = gpu_ctx.set_height_range_device(desc, d_pts.data_ptr(), n_pts, d_tris.data_ptr(),
                                          n_tris, d_g, d_res.data_ptr(), it, MPP, True)
    torch.cuda.synchronize()
    # ---- every intermediate and the result ----
    assert n_vox == len(r_vox)
    assert cases.field_mismatch(cases.from_device(keep["ncc"], abi.NCCRESULT_DTYPE), r_ncc) == {}
    assert cases.field_mismatch(d_vox.cpu().numpy().view(abi.VOXEL_DTYPE)[:n_vox], r_vox) == {}
    got_pts = d_pts.cpu().numpy().view(abi.POINT3_DTYPE)[:n_pts]
    assert len(got_pts) == len(r_pts)
    for f in ("x", "y", "z", "flag"):     # (the record's 7 padding bytes are not data)
        assert got_pts[f].tobytes() == r_pts[f].tobytes(), f
    got_tris = d_tris.cpu().numpy().view(abi.TRI_DTYPE)[:n_tris]
    assert got_tris.tobytes() == r_tris.tobytes()
    got_grid = d_res.cpu().numpy().view(abi.UGRID_DTYPE)
    from tests.golden import make_golden as mg
    assert cases.field_mismatch(mg.clean(got_grid), mg.clean(r_grid)) == {}
    assert ext == r_ext
