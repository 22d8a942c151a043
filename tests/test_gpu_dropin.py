"""The C++ drop-in (VerticalLineLocus with the reference's mangled signature,
setsm_code.hpp:81) called the way SETSM calls it: ProInfo, LevelInfo, UGRID,
NCCresult and VOXEL** built by the reference's own headers (oracle/_ref
harness), handed to the function exported by libsetsm_vll.so.  Results must
equal the reference's golden outputs bit for bit."""
import ctypes as C

import pytest

from oracle import refpy
from setsm_b200 import vll
from tests import cases
from tests.test_abi_layout import DROPIN
from tests.test_oracle_golden import golden_case

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refpy.available(), reason="reference build not available")]


@pytest.mark.parametrize("name", ["m7", "v7_gncc", "l2_combined"])
def test_dropin_through_reference_structures(gpu_ctx, name):
    inp, g = golden_case(name)
    inp.gridpt3 = g["init_gp3"].copy()
    ncc = g["init_ncc"].copy()
    vox = None if g["init_vox"] is None else g["init_vox"].copy()
    fn = C.cast(getattr(vll.load(), DROPIN), C.c_void_p).value
    acc = refpy.call_vertical_line_locus(fn, inp, ncc, vox)
    assert acc == g["acc"]
    assert cases.field_mismatch(ncc, g["vll_ncc"]) == {}
    if vox is not None:
        assert cases.field_mismatch(vox, g["vll_vox"]) == {}
