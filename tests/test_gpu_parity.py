"""CUDA kernels against the C oracle on the same seeded inputs.

Both kernels must reproduce the oracle (= the reference) on every field of
NCCresult and every voxel: the plain FP64 kernel by construction, the split
kernel through its FP64 re-check of every decision that lies inside the FP32
error band."""
import copy

import numpy as np
import pytest

from oracle import oraclepy as op
from setsm_b200 import abi, vll
from tests import cases

pytestmark = pytest.mark.gpu

_oracle_cache = {}


def oracle_run(name):
    if name not in _oracle_cache:
        inp = cases.make_case(**cases.CASES[name])
        _oracle_cache[name] = cases.run_cpu(op, inp, inp.iters)
    return _oracle_cache[name]


def replay(ctx, o, kernel):
    inp = copy.copy(o["inputs"])
    inp.gridpt3 = o["init_gp3"].copy()
    ncc = o["init_ncc"].copy()
    vox = None if o["init_vox"] is None else o["init_vox"].copy()
    st = ctx.vertical_line_locus(inp, ncc, vox, kernel)
    return inp, ncc, vox, st


@pytest.mark.parametrize("kernel", ["plain", "split"])
@pytest.mark.parametrize("name", sorted(cases.CASES))
def test_vertical_line_locus_matches_oracle(gpu_ctx, name, kernel):
    o = oracle_run(name)
    inp, ncc, vox, st = replay(gpu_ctx, o, kernel)
    assert st.accessable_grid == o["acc"]
    assert cases.field_mismatch(ncc, o["vll_ncc"]) == {}
    if vox is not None:
        assert cases.field_mismatch(vox, o["vll_vox"]) == {}
        gpu_ctx.awncc(inp, ncc, vox)
        assert cases.field_mismatch(ncc, o["ncc"]) == {}


@pytest.mark.parametrize("cap", ["0", "40"])
@pytest.mark.parametrize("name", ["m7", "m11", "v7_gncc", "v7_it2", "l3_m"])
def test_full_pending_buffer_stays_exact(gpu_ctx, name, cap, monkeypatch):
    """Nodes the FP32 pass cannot settle are queued with their FP32 values in
    a pending buffer of limited size; a node that finds it full is evaluated
    wholly in FP64 by the exact pass.  With no room (0) or room for a node
    or so (40 slots), every record and voxel is still the oracle's."""
    if name not in cases.CASES:
        pytest.skip(f"no case {name}")
    monkeypatch.setenv("SETSM_VLL_PENDING_SLOTS", cap)
    o = oracle_run(name)
    inp, ncc, vox, st = replay(gpu_ctx, o, "split")
    assert st.accessable_grid == o["acc"]
    assert cases.field_mismatch(ncc, o["vll_ncc"]) == {}
    if vox is not None:
        assert cases.field_mismatch(vox, o["vll_vox"]) == {}
    if cap == "0":
        assert st.fp64_nodes == st.exact_nodes


def test_split_is_deterministic_and_counts(gpu_ctx):
    o = oracle_run("m7")
    _, n1, _, s1 = replay(gpu_ctx, o, "split")
    _, n2, _, s2 = replay(gpu_ctx, o, "split")
    assert n1.tobytes() == n2.tobytes()
    _, n3, _, s3 = replay(gpu_ctx, o, "plain")
    assert s1.evals == s3.evals > 0
    assert s1.fp64_rechecks < s1.evals


@pytest.mark.parametrize("seed", [3, 5])
def test_preprocess_matches_oracle(gpu_ctx, seed):
    im = cases.scene(seed, 768).images[1].numpy().view(np.uint16)
    mag, ori = gpu_ctx.preprocess(im)
    m2, o2 = op.preprocess(im)
    assert np.array_equal(mag, m2)
    assert np.array_equal(ori, o2)
    odd = np.ascontiguousarray(im[:333, :517])
    mag, ori = gpu_ctx.preprocess(odd)
    m2, o2 = op.preprocess(odd)
    assert np.array_equal(mag, m2) and np.array_equal(ori, o2)


def test_pyramid_matches_oracle(gpu_ctx):
    im = cases.scene(3, 768).images[0].numpy().view(np.uint16)
    assert np.array_equal(gpu_ctx.pyramid_down(im), op.pyramid_down(im))
    odd = np.ascontiguousarray(im[:301, :257])
    assert np.array_equal(gpu_ctx.pyramid_down(odd), op.pyramid_down(odd))


def test_errors_are_status_codes(gpu_ctx):
    o = oracle_run("v7_gncc")
    inp = copy.copy(o["inputs"])
    ncc = o["init_ncc"].copy()
    small = np.zeros(3, dtype=abi.VOXEL_DTYPE)
    with pytest.raises(vll.VLLError) as e:
        gpu_ctx.vertical_line_locus(inp, ncc, small, "plain")
    assert e.value.code == abi.VLL_ERR_CAPACITY
    bad = copy.copy(inp)
    bad.template_size = 200   # half-size far beyond the supported windows
    with pytest.raises(vll.VLLError) as e:
        gpu_ctx.vertical_line_locus(bad, o["init_ncc"].copy(), o["init_vox"].copy(), "plain")
    assert e.value.code == abi.VLL_ERR_UNSUPPORTED
    # the context stays usable after errors
    _, n2, _, _ = replay(gpu_ctx, o, "plain")
    assert cases.field_mismatch(n2, o["vll_ncc"]) == {}
