"""Batches of levels in one pass of the split pipeline (one persistent window
launch over every level's work items), the CUDA-graph plan of a batch, and the
launch tuning: every level's outputs must equal the oracle's for that level
alone, bit for bit, whatever the mix of window sizes, pyramid levels, routes
and tuning."""
import numpy as np
import pytest

from setsm_b200 import abi, vll
from tests import cases
from tests.test_gpu_parity import oracle_run

pytestmark = pytest.mark.gpu

MIX = ["m7", "m11", "m7_edges", "l3_m", "v7_gncc", "v11", "l2_max", "v7_it2", "l2_combined"]


def build_batch(torch, names):
    levels, held = [], []
    for name in names:
        o = oracle_run(name)
        inp = o["inputs"]
        inp.gridpt3 = o["init_gp3"].copy()
        io, h = cases.device_level(torch, inp, o["init_ncc"], o["init_vox"])
        levels.append(io)
        held.append((name, o, h))
    return levels, held


def check_outputs(held, acc):
    for (name, o, h), a in zip(held, acc):
        assert a == o["acc"], name
        ncc = cases.from_device(h["ncc"], abi.NCCRESULT_DTYPE)
        assert cases.field_mismatch(ncc, o["vll_ncc"]) == {}, name
        if h["vox"] is not None:
            vox = cases.from_device(h["vox"], abi.VOXEL_DTYPE)
            assert cases.field_mismatch(vox, o["vll_vox"]) == {}, name


def reset(torch, held):
    for name, o, h in held:
        h["ncc"].copy_(torch.from_numpy(o["init_ncc"].view(np.uint8).copy()))
        if h["vox"] is not None:
            h["vox"].copy_(torch.from_numpy(o["init_vox"].view(np.uint8).copy()))


def test_batch_of_mixed_levels_matches_oracle(gpu_ctx):
    import torch
    levels, held = build_batch(torch, MIX)
    acc, st = gpu_ctx.batch(levels)
    check_outputs(held, acc)
    assert st.evals > 0 and st.accessable_grid == sum(o["acc"] for _, o, _ in held)


def test_batch_order_does_not_matter(gpu_ctx):
    import torch
    names = list(reversed(MIX))
    levels, held = build_batch(torch, names)
    acc, _ = gpu_ctx.batch(levels)
    check_outputs(held, acc)


def test_plan_replays_match_oracle(gpu_ctx):
    import torch
    levels, held = build_batch(torch, MIX)
    plan = gpu_ctx.plan(levels)
    for _ in range(3):
        reset(torch, held)
        acc, st = plan.run()
        check_outputs(held, acc)
    # replays without resetting the outputs are idempotent
    plan.run(wait=False)
    acc, st = plan.run()
    check_outputs(held, acc)
    plan.close()


def test_plan_follows_changed_ranges(gpu_ctx):
    """A plan's buffers depend on the node count only: replays after the
    height ranges changed give the same records as an unplanned batch on the
    changed ranges, and restoring the ranges restores the original results."""
    import torch
    levels, held = build_batch(torch, ["m7", "m11"])
    plan = gpu_ctx.plan(levels)
    name, o, h = held[0]
    g = o["init_gp3"].copy()
    g["maxHeight"] = g["maxHeight"] + 7      # more height slots than planned
    h["gp3"].copy_(torch.from_numpy(g.view(np.uint8).copy()))
    reset(torch, held)
    acc_p, _ = plan.run()
    got = [hh["ncc"].cpu().numpy().copy() for _, _, hh in held]
    reset(torch, held)
    acc_b, _ = gpu_ctx.batch(levels)
    want = [hh["ncc"].cpu().numpy().copy() for _, _, hh in held]
    assert list(acc_p) == list(acc_b)
    for a, b in zip(got, want):
        assert a.tobytes() == b.tobytes()
    # restoring the ranges restores the plan's original results
    h["gp3"].copy_(torch.from_numpy(o["init_gp3"].view(np.uint8).copy()))
    reset(torch, held)
    acc, _ = plan.run()
    check_outputs(held, acc)
    plan.close()


@pytest.mark.parametrize("tuning", [dict(blocks_per_sm=1, grab=1, box_margin=1.0),
                                    dict(blocks_per_sm=2, grab=16, box_margin=2.0),
                                    dict(blocks_per_sm=0, grab=64, box_margin=1.5)])
def test_tuning_does_not_change_results(gpu_ctx, tuning):
    import torch
    saved = gpu_ctx.get_tuning()
    try:
        gpu_ctx.set_tuning(**tuning)
        assert gpu_ctx.get_tuning()["grab"] == tuning["grab"]
        levels, held = build_batch(torch, ["m7", "m11", "m7_edges"])
        acc, _ = gpu_ctx.batch(levels)
        check_outputs(held, acc)
    finally:
        gpu_ctx.set_tuning(**saved)


def test_tuning_rejects_bad_values(gpu_ctx):
    with pytest.raises(vll.VLLError):
        gpu_ctx.set_tuning(grab=1000)
    with pytest.raises(vll.VLLError):
        gpu_ctx.set_tuning(box_margin=0.5)


def test_batch_refuses_unsupported_window(gpu_ctx):
    """A 17x17 window (half-size 8) is matched by the plain FP64 kernel only;
    a batch containing it is refused with a status, not run partially."""
    import torch
    levels, held = build_batch(torch, ["m7", "m11"])
    levels[1][0].template_size = 21
    with pytest.raises(vll.VLLError) as e:
        gpu_ctx.batch(levels)
    assert e.value.code == abi.VLL_ERR_UNSUPPORTED
