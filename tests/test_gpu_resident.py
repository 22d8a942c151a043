"""Residency of the host-buffer calls (vll_set_residency) and of the C++
drop-ins: image planes and grid arrays kept on the device between calls,
voxel rows kept there along InitializeVoxel -> VerticalLineLocus -> AWNCC.
Results must be the ones of the calls that copy everything every time, and
of the reference (setsm_code.cpp:3743-3844)."""
import ctypes as C
import copy

import numpy as np
import pytest

from oracle import refpy
from setsm_b200 import abi, vll
from tests import cases
from tests.test_abi_layout import DROPIN
from tests.test_gpu_init_voxel import DROPIN_AWNCC, DROPIN_IV

pytestmark = pytest.mark.gpu


def test_resident_planes_give_the_same_records(gpu_ctx):
    inp = cases.make_case(**cases.CASES["m7"])
    want = inp.new_nccresult()
    gpu_ctx.set_residency()
    st0 = gpu_ctx.vertical_line_locus(inp, want, None, "split")
    try:
        gpu_ctx.set_residency(planes=True)
        for _ in range(3):
            got = inp.new_nccresult()
            st = gpu_ctx.vertical_line_locus(inp, got, None, "split")
            assert st.accessable_grid == st0.accessable_grid
            assert got.tobytes() == want.tobytes()
        # another image (a new array, or new content) is sent again
        other = cases.make_case(**dict(cases.CASES["m7"], seed=4))
        got = other.new_nccresult()
        gpu_ctx.vertical_line_locus(other, got, None, "split")
        gpu_ctx.set_residency()
        ref = other.new_nccresult()
        gpu_ctx.vertical_line_locus(other, ref, None, "split")
        assert got.tobytes() == ref.tobytes()
        assert got.tobytes() != want.tobytes()
    finally:
        gpu_ctx.set_residency()


@pytest.mark.parametrize("name", ["v7_gncc", "v11"])
def test_resident_voxel_route_matches_copies(gpu_ctx, name):
    """Two iterations of InitializeVoxel -> VerticalLineLocus -> AWNCC with
    the voxel packing resident equal the same calls with host voxel arrays."""
    base = cases.make_case(**cases.CASES[name])
    g0 = base.gridpt3.copy()
    # host copies every call
    a = copy.copy(base)
    a.gridpt3 = g0.copy()
    ncc_a = a.new_nccresult()
    vox = None
    for it in (1, 2):
        a.iteration = it
        vox = gpu_ctx.initialize_voxel(a, ncc_a, vox)
        gpu_ctx.vertical_line_locus(a, ncc_a, vox, "split")
        gpu_ctx.awncc(a, ncc_a, vox)
    # resident
    b = copy.copy(base)
    b.gridpt3 = g0.copy()
    ncc_b = b.new_nccresult()
    try:
        gpu_ctx.set_residency(planes=True, voxels=True)
        gpu_ctx.resident_reset()
        for it in (1, 2):
            b.iteration = it
            gpu_ctx.initialize_voxel_resident(b, ncc_b)
            gpu_ctx.vertical_line_locus(b, ncc_b, None, "split")
            gpu_ctx.awncc(b, ncc_b, None)
        rv = gpu_ctx.resident_voxels()
    finally:
        gpu_ctx.set_residency()
    assert cases.field_mismatch(ncc_b, ncc_a) == {}
    assert cases.field_mismatch(b.gridpt3, a.gridpt3) == {}
    assert cases.field_mismatch(rv, vox) == {}


@pytest.mark.skipif(not refpy.available(), reason="reference build not available")
@pytest.mark.parametrize("resident", ["1", None])
@pytest.mark.parametrize("name", ["v7_gncc", "v7_3img"])
def test_dropin_iterations_on_one_voxel_array(gpu_ctx, name, resident, monkeypatch):
    """The three C++ drop-ins called as Matching_SETSM calls them, two
    iterations on one VOXEL** array, with the voxel rows resident on the
    device (SETSM_VLL_RESIDENT=1) or copied every call: NCCresult, UGRID and
    Accessable_grid of the reference's own three functions."""
    if resident:
        monkeypatch.setenv("SETSM_VLL_RESIDENT", resident)
    else:
        monkeypatch.delenv("SETSM_VLL_RESIDENT", raising=False)
    L = vll.load()
    fns = tuple(C.cast(getattr(L, s), C.c_void_p).value for s in (DROPIN_IV, DROPIN, DROPIN_AWNCC))
    base = cases.make_case(**cases.CASES[name])
    g0 = base.gridpt3.copy()
    ref = copy.copy(base)
    ref.gridpt3 = g0.copy()
    ref_ncc = ref.new_nccresult()
    acc_ref = refpy.call_voxel_iterations((None, None, None), ref, ref_ncc, (1, 2))
    got = copy.copy(base)
    got.gridpt3 = g0.copy()
    got_ncc = got.new_nccresult()
    acc = refpy.call_voxel_iterations(fns, got, got_ncc, (1, 2))
    assert acc == acc_ref and acc[0] > 0
    assert cases.field_mismatch(got_ncc, ref_ncc) == {}
    assert cases.field_mismatch(got.gridpt3, ref.gridpt3) == {}
