"""Row-band sharding through the CUDA kernels: bands matched on cropped image
footprints (one after another on one GPU, as ranks would on their own GPUs)
concatenate to the whole-grid GPU result and to the oracle, bit for bit."""
import numpy as np
import pytest

from oracle import oraclepy as op
from setsm_b200 import shard
from tests import cases

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kernel", ["split", "plain"])
@pytest.mark.parametrize("name,world", [("m7", 2), ("m11", 3), ("m7_edges", 2)])
def test_gpu_bands_reproduce_whole_grid(gpu_ctx, name, world, kernel):
    inp = cases.make_case(**cases.CASES[name])
    ncc_o = inp.new_nccresult()
    acc_o = op.vertical_line_locus(inp, ncc_o, None)
    parts, acc = [], 0
    for rank in range(world):
        ncc, a, _ = shard.match_band(gpu_ctx, inp, rank, world, kernel=kernel)
        parts.append(ncc)
        acc += a
    got = np.concatenate(parts)
    assert acc == acc_o
    assert cases.field_mismatch(got, ncc_o) == {}


@pytest.mark.parametrize("world", [1, 3])
def test_device_bands_reproduce_whole_grid(gpu_ctx, world):
    """The sharded bench's path: bands of the C1 workload with their image
    footprints cropped on the device (Workload.device_band) give the
    whole-grid call's records and Accessable_grid, bit for bit."""
    import torch

    from setsm_b200 import workloads
    wl = workloads.build("c1", gpu_ctx, device="cuda:0", seed=3, keep_host=False)
    t = workloads.CONFIGS["c1"]["templates"][0]
    wl.d_ncc.zero_()
    torch.cuda.synchronize()
    st = gpu_ctx.vertical_line_locus_device(wl.device_desc(t), wl.d_gp3.data_ptr(),
                                            wl.d_ncc.data_ptr(), None, None, "split", stats=True)
    want = workloads.ncc_host(wl)
    parts, acc = [], 0
    for r0, r1 in shard.row_bands(wl.grid.height, world):
        band = wl.device_band(r0, r1)
        if world > 1:
            # two images of 5 bytes per pixel (intensity, magnitude, orientation)
            assert band.image_bytes() < 0.8 * 2 * 5 * wl.d_img[0].numel()
        out = torch.zeros(band.n_nodes * shard.NCC_BYTES, dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        s = gpu_ctx.vertical_line_locus_device(band.desc(t), band.d_gridpt3(), out.data_ptr(),
                                               None, None, "split", stats=True)
        parts.append(out.cpu().numpy().view(want.dtype))
        acc += int(s.accessable_grid)
    got = np.concatenate(parts)
    assert acc == int(st.accessable_grid) > 0
    assert cases.field_mismatch(got, want) == {}
