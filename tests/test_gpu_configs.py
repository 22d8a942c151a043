"""The benchmark workloads against the reference SETSM build itself.

* C1 (2048^2 pair, 256^2 grid, 64 heights at 1 m, 7x7): the whole grid
  through the reference's VerticalLineLocus (oracle/_ref, setsm_code.cpp:
  6049-6548) and through both CUDA kernels; every NCCresult field and the
  returned Accessable_grid identical.
* The reduced level-0 scene (4096^2 pair, 1024^2 grid, TIN ranges K 8-512 at
  0.5 m, the generator and distributions of the full 16384^2 scene): a band
  of grid rows through the reference with magnitude / orientation planes made
  by the reference's own MakeSobelMagnitudeImage / Orientation on a crop
  around the band, against the split kernel's whole-grid result for those
  rows, for the 7x7 and the 11x11 window; the crop planes equal the GPU-made
  planes over the band's footprint.
"""
import math

import numpy as np
import pytest

from oracle import refpy
from tests import cases

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refpy.available(), reason="reference build not available")]


def _ncc_of(wl, ctx, template, kernel):
    from setsm_b200 import workloads
    import torch
    wl.d_ncc.zero_()
    torch.cuda.synchronize()   # the library runs on its own stream
    st = ctx.vertical_line_locus_device(wl.device_desc(template), wl.d_gp3.data_ptr(),
                                        wl.d_ncc.data_ptr(), None, None, kernel, stats=True)
    return workloads.ncc_host(wl), st


@pytest.fixture(scope="module")
def c1(gpu_ctx):
    from setsm_b200 import workloads
    return workloads.build("c1", gpu_ctx, device="cuda:0", seed=1)


@pytest.mark.parametrize("kernel", ["split", "plain"])
def test_c1_whole_grid_identical_to_reference(gpu_ctx, c1, kernel):
    import os
    refpy.set_threads(os.cpu_count() or 1)
    inp = c1.host_inputs(11)
    ncc_ref = inp.new_nccresult()
    acc_ref = refpy.vertical_line_locus(inp, ncc_ref)
    ncc_gpu, st = _ncc_of(c1, gpu_ctx, 11, kernel)
    assert st.accessable_grid == acc_ref
    assert acc_ref > 0.9 * c1.n_nodes
    assert cases.field_mismatch(ncc_gpu, ncc_ref) == {}
    # the host-buffer C ABI gives the same records
    ncc_h = inp.new_nccresult()
    st_h = gpu_ctx.vertical_line_locus(inp, ncc_h, None, kernel)
    assert st_h.accessable_grid == acc_ref
    assert cases.field_mismatch(ncc_h, ncc_ref) == {}


@pytest.fixture(scope="module")
def c2s(gpu_ctx):
    from setsm_b200 import workloads
    return workloads.build("c2_small", gpu_ctx, device="cuda:0", seed=1)


def _footprint(wl, r0, rows, margin=48):
    import torch
    from setsm_b200 import synth
    W = wl.grid.width
    sl = slice(r0 * W, (r0 + rows) * W)
    wgs = torch.from_numpy(np.ascontiguousarray(wl.host["wgs"][sl]))
    n = wl.scene.spec.image_size
    out = []
    for ci in range(2):
        lines = []
        for f in ("minHeight", "maxHeight"):
            h = torch.from_numpy(wl.gp3[f][sl].astype(np.float64))
            lines.append(synth.rpc_eval(wl.scene.rpcs[ci], wgs[:, 0], wgs[:, 1], h)[1])
        line = torch.cat(lines)
        out.append((max(0, int(math.floor(float(line.min()))) - margin),
                    min(n, int(math.ceil(float(line.max()))) + margin)))
    return out


@pytest.mark.parametrize("template", [11, 15])
def test_level0_scene_band_identical_to_reference(gpu_ctx, c2s, template):
    import os
    refpy.set_threads(os.cpu_count() or 1)
    wl = c2s
    rows = 24
    r0 = wl.grid.height // 2 - rows // 2 + 101
    fp = _footprint(wl, r0, rows)
    n = wl.scene.spec.image_size
    mags = [np.zeros((n, n), np.uint16) for _ in range(2)]
    oris = [np.zeros((n, n), np.uint8) for _ in range(2)]
    for ci, (y0, y1) in enumerate(fp):
        c0, c1_ = max(0, y0 - 16), min(n, y1 + 16)
        m, o = refpy.preprocess(wl.host["img"][ci][c0:c1_], 15)
        mags[ci][y0:y1] = m[y0 - c0:y1 - c0]
        oris[ci][y0:y1] = o[y0 - c0:y1 - c0]
        # the reference's planes equal the library's over the footprint
        assert np.array_equal(mags[ci][y0:y1], wl.host["mag"][ci][y0:y1])
        assert np.array_equal(oris[ci][y0:y1], wl.host["ori"][ci][y0:y1])
    inp = wl.host_inputs(template, rows=(r0, r0 + rows), planes={"mag": mags, "ori": oris})
    ncc_ref = inp.new_nccresult()
    acc_ref = refpy.vertical_line_locus(inp, ncc_ref)
    assert acc_ref > 0
    ncc_gpu, _ = _ncc_of(wl, gpu_ctx, template, "split")
    W = wl.grid.width
    band = ncc_gpu[r0 * W:(r0 + rows) * W]
    assert cases.field_mismatch(band, ncc_ref) == {}
