"""The allocation-free entry point (vll_vertical_line_locus_noalloc).

Callers that cannot allocate device memory at call time -- a pool allocator
that owns the GPU, another framework's memory manager, a latency-critical
loop -- use this variant; it takes its scratch from a fixed 64 MiB device
array instead of cudaMalloc.  These tests call it through the C ABI and check
that two calls in a row reproduce the regular split-kernel entry point
exactly, that oversize grids are rejected before any output is written, and
that unsupported routes are refused."""
import copy
import ctypes as C

import numpy as np
import pytest

from setsm_b200 import abi, vll
from tests import cases

pytestmark = pytest.mark.gpu


def _device_case(torch, inp):
    """Device copies of a case's inputs and a descriptor pointing at them."""
    keep = []
    d = inp.desc()
    for ti, im in enumerate(inp.images):
        for name, arr in (("image", im.image), ("mag", im.mag), ("ori", im.ori)):
            src = arr.view(np.int16) if arr.dtype == np.uint16 else arr
            t = torch.from_numpy(np.ascontiguousarray(src)).cuda()
            keep.append(t)
            setattr(d.images[ti], name, t.data_ptr())
    wgs = torch.from_numpy(inp.grid_wgs).cuda()
    pts = torch.from_numpy(inp.grid_pts).cuda()
    keep += [wgs, pts]
    d.grid_wgs = wgs.data_ptr()
    d.grid_pts = pts.data_ptr()
    gp3 = torch.from_numpy(inp.gridpt3.view(np.uint8).copy()).cuda()
    keep.append(gp3)
    return d, gp3, keep


def _noalloc(d, d_gp3, d_ncc, stream=None):
    L = vll.load()
    fn = L.vll_vertical_line_locus_noalloc
    fn.argtypes = [C.POINTER(abi.LevelDesc), C.c_void_p, C.c_void_p, C.c_void_p,
                   C.POINTER(C.c_int64), C.c_char_p, C.c_int]
    fn.restype = C.c_int
    acc = C.c_int64(-1)
    buf = C.create_string_buffer(256)
    rc = fn(C.byref(d), d_gp3, d_ncc, stream, C.byref(acc), buf, 256)
    return rc, acc.value, buf.value.decode()


def test_noalloc_matches_regular_entry_point(gpu_ctx):
    import torch
    inp = cases.make_case(**cases.CASES["m7"])
    d, d_gp3, keep = _device_case(torch, inp)
    n_bytes = inp.n * abi.NCCRESULT_DTYPE.itemsize
    init = inp.new_nccresult()
    d_ref = torch.from_numpy(init.view(np.uint8).copy()).cuda()
    st = gpu_ctx.vertical_line_locus_device(d, d_gp3.data_ptr(), d_ref.data_ptr(), kernel="split",
                                            stats=True)
    ref = d_ref.cpu().numpy().view(abi.NCCRESULT_DTYPE)
    assert st.accessable_grid > 0
    for _ in range(2):   # two calls in a row share (and must clear) the scratch array
        d_out = torch.from_numpy(init.view(np.uint8).copy()).cuda()
        rc, acc, msg = _noalloc(d, d_gp3.data_ptr(), d_out.data_ptr())
        assert rc == abi.VLL_OK, msg
        out = d_out.cpu().numpy().view(abi.NCCRESULT_DTYPE)
        assert acc == st.accessable_grid
        assert cases.field_mismatch(out, ref) == {}
        assert d_out.numel() == n_bytes


def test_noalloc_rejects_oversize_grid_before_writing(gpu_ctx):
    """A 2048^2 grid (4.2 M nodes): its per-node scratch arrays alone exceed
    the 64 MiB array, so the call is refused before any output is written."""
    import torch
    inp = cases.make_case(**cases.CASES["m7"])
    d, _, keep = _device_case(torch, inp)
    side = 2048
    n = side * side
    d.grid_width = side
    d.grid_height = side
    wgs = torch.zeros(n * 16, dtype=torch.uint8, device="cuda")
    pts = torch.zeros(n * 16, dtype=torch.uint8, device="cuda")
    d.grid_wgs = wgs.data_ptr()
    d.grid_pts = pts.data_ptr()
    d_gp3 = torch.zeros(n * abi.UGRID_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    init = np.zeros(n, dtype=abi.NCCRESULT_DTYPE)
    init["result0"] = 123
    d_out = torch.from_numpy(init.view(np.uint8).copy()).cuda()
    rc, acc, msg = _noalloc(d, d_gp3.data_ptr(), d_out.data_ptr())
    assert rc == abi.VLL_ERR_CAPACITY
    assert "scratch" in msg
    out = d_out.cpu().numpy().view(abi.NCCRESULT_DTYPE)
    assert out.tobytes() == init.tobytes()


def test_noalloc_refuses_voxel_route(gpu_ctx):
    import torch
    inp = cases.make_case(**cases.CASES["v7_gncc"])
    d, d_gp3, keep = _device_case(torch, inp)
    d_out = torch.zeros(inp.n * abi.NCCRESULT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    rc, acc, msg = _noalloc(d, d_gp3.data_ptr(), d_out.data_ptr())
    assert rc == abi.VLL_ERR_UNSUPPORTED
