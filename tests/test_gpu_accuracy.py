"""FP32 window statistics of the split kernel against the exact FP64 kernel,
slot by slot (before the split kernel's FP64 re-checks).

Tolerance (stated by the matching spec): |delta NCC| <= 1e-4 on every slot.
The split kernel's error band for re-checks (2e-5) must also cover the
observed error with margin, otherwise its exactness argument fails."""
import numpy as np
import pytest

from tests import cases

pytestmark = pytest.mark.gpu

NCC_TOL = 1e-4
BAND = 2e-5


@pytest.mark.parametrize("name", ["m7", "m11", "m7_edges", "l3_m"])
def test_fp32_rho_error(gpu_ctx, name):
    inp = cases.make_case(**cases.CASES[name])
    r32, off = gpu_ctx.debug_slot_rho(inp, inp.new_nccresult(), "split")
    r64, off2 = gpu_ctx.debug_slot_rho(inp, inp.new_nccresult(), "plain")
    assert np.array_equal(off, off2)
    both = ~np.isnan(r32) & ~np.isnan(r64)
    assert both.sum() > 1000
    # the same slots are evaluated by both kernels
    assert np.array_equal(np.isnan(r32), np.isnan(r64))
    err = np.abs(r32[both] - r64[both])
    print(f"{name}: {both.sum()} slots, max |dNCC| {err.max():.3e}, p99.99 "
          f"{np.quantile(err, 0.9999):.3e}")
    assert err.max() <= NCC_TOL
    assert err.max() < BAND / 2
