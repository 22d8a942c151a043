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
