"""Row-band sharding (setsm_b200/shard.py): the host logic on the CPU.

The bands' results, computed on footprint-cropped images with moved
py_Startpos, must concatenate to the whole-grid result bit for bit.  The
matcher itself is stood in for by the oracle here (a CPU context with the
library's call shape); tests/test_gpu_shard.py runs the same bands through the
CUDA kernels.  The world-size-2 test runs two gloo ranks that each match their
band and all-gather the rows."""
import os

import numpy as np
import pytest

from oracle import oraclepy as op
from setsm_b200 import shard
from tests import cases


class OracleContext:
    """The oracle behind the matcher's call shape (test stand-in only)."""

    class _St:
        def __init__(self, acc):
            self.accessable_grid = acc

    def vertical_line_locus(self, inputs, ncc, voxels=None, kernel="split"):
        return self._St(op.vertical_line_locus(inputs, ncc, voxels))


def full_result(inp):
    ncc = inp.new_nccresult()
    acc = op.vertical_line_locus(inp, ncc, None)
    return ncc, acc


def test_row_bands_partition():
    for h in (1, 7, 48, 4096):
        for w in (1, 2, 3, 8):
            b = shard.row_bands(h, w)
            assert len(b) == w and b[0][0] == 0 and b[-1][1] == h
            assert all(b[k][1] == b[k + 1][0] for k in range(w - 1))
            sizes = [r1 - r0 for r0, r1 in b]
            assert max(sizes) - min(sizes) <= 1


@pytest.mark.parametrize("name,world", [("m7", 2), ("m7", 3), ("m11", 2), ("m7_edges", 4),
                                        ("l3_m", 2)])
def test_bands_reproduce_whole_grid(name, world):
    inp = cases.make_case(**cases.CASES[name])
    assert shard.shardable(inp)
    ncc_full, acc_full = full_result(inp)
    ctx = OracleContext()
    parts, acc = [], 0
    for rank in range(world):
        ncc, a, (r0, r1) = shard.match_band(ctx, inp, rank, world)
        parts.append(ncc)
        acc += a
    got = np.concatenate(parts)
    assert acc == acc_full
    assert cases.field_mismatch(got, ncc_full) == {}


def test_bands_hold_only_their_footprint():
    inp = cases.make_case(**cases.CASES["m7"])
    full_px = inp.images[0].image.size
    band = shard.band_inputs(inp, inp.grid_height // 2, 3 * inp.grid_height // 4)
    for ti in range(2):
        assert band.images[ti].image.size < 0.6 * full_px
        assert band.images[ti].image.shape == band.images[ti].mag.shape == band.images[ti].ori.shape
        sx, sy = band.images[ti].startpos
        assert sx >= 0 and sy >= 0 and sx + sy > 0


GLOO_CASE = dict(size=384, nodes=20, res=8.0, n_heights=24)


def _rank_main(rank, world, port, result_path):
    import torch
    import torch.distributed as dist
    torch.set_num_threads(2)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        inp = cases.make_case(**GLOO_CASE)
        ncc, acc, _ = shard.match_band(OracleContext(), inp, rank, world)
        full, total = shard.gather_bands(ncc, acc, inp.grid_width, inp.grid_height)
        if rank == 0:
            np.save(result_path, full.view(np.uint8))
            with open(result_path + ".acc", "w") as f:
                f.write(str(total))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_gather_the_grid(tmp_path, world):
    """Bands matched by `world` gloo ranks and gathered with
    all_gather_into_tensor (3 ranks: unequal bands, padded to the largest)."""
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    path = str(tmp_path / "ncc.npy")
    mp.start_processes(_rank_main, args=(world, port, path), nprocs=world, join=True,
                       start_method="spawn")
    inp = cases.make_case(**GLOO_CASE)
    ncc_full, acc_full = full_result(inp)
    assert acc_full > 0
    got = np.load(path).view(ncc_full.dtype)
    assert int(open(path + ".acc").read()) == acc_full
    assert cases.field_mismatch(got, ncc_full) == {}
