"""AWNCC with semi-global aggregation on the GPU (vll_sgm.cu + the SGM
branch of the peak loop) against the reference's own AWNCC
(setsm_code.cpp:7001-7702): the fixtures in tests/golden made by the
reference build, and the reference build itself where it is present.  Every
NCCresult field must be identical."""
import copy

import pytest

from oracle import refpy
from tests import cases
from tests.golden import make_golden as mg
from tests.test_oracle_golden import load_fixture

pytestmark = pytest.mark.gpu


def golden_sgm(name):
    inp = cases.make_case(**mg.GOLDEN_SGM[name])
    g = load_fixture(name)
    assert mg.input_digest(inp) == g["digest"]
    return inp, g


@pytest.mark.parametrize("kernel", ["split", "plain"])
@pytest.mark.parametrize("name", sorted(mg.GOLDEN_SGM))
def test_sgm_awncc_matches_reference_fixture(gpu_ctx, name, kernel):
    inp, g = golden_sgm(name)
    inp.gridpt3 = g["init_gp3"].copy()
    ncc = g["init_ncc"].copy()
    vox = g["init_vox"].copy()
    st = gpu_ctx.vertical_line_locus(inp, ncc, vox, kernel)
    assert st.accessable_grid == g["acc"]
    assert cases.field_mismatch(ncc, g["vll_ncc"]) == {}
    assert cases.field_mismatch(vox, g["vll_vox"]) == {}
    gpu_ctx.awncc(inp, ncc, vox)
    assert cases.field_mismatch(ncc, g["ncc"]) == {}


@pytest.mark.skipif(not refpy.available(), reason="reference build not available")
@pytest.mark.parametrize("seed", [7, 11])
def test_sgm_awncc_matches_reference_build(gpu_ctx, seed):
    """A larger grid (and other seeds) straight against the reference build."""
    inp = cases.make_case(seed=seed, size=768, nodes=40, res=7.0, n_heights=48, cmr=False, sgm=1,
                          ortho_frac=0.5, it=2, iters=(1, 2))
    r = cases.run_cpu(refpy, inp, inp.iters)
    inp2 = copy.copy(r["inputs"])
    inp2.gridpt3 = r["init_gp3"].copy()
    ncc = r["init_ncc"].copy()
    vox = r["init_vox"].copy()
    gpu_ctx.vertical_line_locus(inp2, ncc, vox, "split")
    assert cases.field_mismatch(ncc, r["vll_ncc"]) == {}
    gpu_ctx.awncc(inp2, ncc, vox)
    assert cases.field_mismatch(ncc, r["ncc"]) == {}


@pytest.mark.parametrize("name", sorted(mg.GOLDEN_SGM))
def test_sgm_per_direction_form_matches_fixture(gpu_ctx, name, monkeypatch):
    """The per-direction launches (used when the 8 stored directions exceed the
    memory budget) give the same NCCresult as the all-directions form."""
    monkeypatch.setenv("SETSM_VLL_SGM_SEQUENTIAL", "1")
    inp, g = golden_sgm(name)
    inp.gridpt3 = g["init_gp3"].copy()
    ncc = g["vll_ncc"].copy()
    vox = g["vll_vox"].copy()
    gpu_ctx.awncc(inp, ncc, vox)
    assert cases.field_mismatch(ncc, g["ncc"]) == {}
