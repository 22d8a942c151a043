"""The CUDA kernels against the reference's own outputs (tests/golden), replaying
the last VerticalLineLocus call of each case from the fixture's recorded
inputs: every NCCresult field and voxel bit-exact, for both kernels, and the
AWNCC peak loop on the voxel route."""
import numpy as np
import pytest

from tests import cases
from tests.golden import make_golden as mg
from tests.test_oracle_golden import golden_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kernel", ["plain", "split"])
@pytest.mark.parametrize("name", sorted(mg.GOLDEN))
def test_kernels_match_reference_golden(gpu_ctx, name, kernel):
    inp, g = golden_case(name)
    inp.gridpt3 = g["init_gp3"].copy()
    ncc = g["init_ncc"].copy()
    vox = None if g["init_vox"] is None else g["init_vox"].copy()
    st = gpu_ctx.vertical_line_locus(inp, ncc, vox, kernel)
    assert st.accessable_grid == g["acc"]
    assert cases.field_mismatch(ncc, g["vll_ncc"]) == {}
    if vox is not None:
        assert cases.field_mismatch(vox, g["vll_vox"]) == {}
        gpu_ctx.awncc(inp, ncc, vox)
        assert cases.field_mismatch(ncc, g["ncc"]) == {}
    else:
        assert np.array_equal(ncc.view(np.uint8), g["ncc"].view(np.uint8))
