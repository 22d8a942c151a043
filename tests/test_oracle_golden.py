"""The oracle against golden vectors produced by the reference SETSM code
(tests/golden/*.npz, written by tests/golden/make_golden.py from the
reference's own InitializeVoxel / VerticalLineLocus / AWNCC).  Bit-exact on
every NCCresult, UGRID and voxel field.  This pins the oracle wherever the
reference sources are absent."""
import numpy as np
import pytest

from oracle import oraclepy as op
from setsm_b200 import abi
from tests import cases
from tests.golden import make_golden as mg


def load_fixture(name):
    z = np.load(mg.fixture_path(name))
    out = {"digest": str(z["digest"]), "acc": int(z["acc"])}
    for k, dt in (("init_ncc", abi.NCCRESULT_DTYPE), ("vll_ncc", abi.NCCRESULT_DTYPE),
                  ("ncc", abi.NCCRESULT_DTYPE), ("init_gp3", abi.UGRID_DTYPE),
                  ("init_vox", abi.VOXEL_DTYPE), ("vll_vox", abi.VOXEL_DTYPE)):
        out[k] = z[k].view(dt) if k in z.files else None
    return out


def golden_case(name):
    inp = cases.make_case(**mg.GOLDEN[name])
    g = load_fixture(name)
    assert mg.input_digest(inp) == g["digest"], \
        "regenerated inputs differ from the ones the golden vectors were made from"
    return inp, g


@pytest.mark.parametrize("name", sorted(mg.GOLDEN))
def test_oracle_matches_reference_golden(name):
    inp, g = golden_case(name)
    o = cases.run_cpu(op, inp, inp.iters)
    assert o["acc"] == g["acc"] > 0
    for k in ("init_ncc", "init_gp3", "vll_ncc", "ncc", "init_vox", "vll_vox"):
        if g[k] is None:
            assert o.get(k) is None
            continue
        assert cases.field_mismatch(o[k], g[k]) == {}, k
    # every fixture carries peaks
    assert (g["ncc"]["result4"] > 0).sum() > 0


def test_golden_set_covers_the_routes():
    routes = set()
    for name, kw in mg.GOLDEN.items():
        routes.add(("voxel" if kw.get("cmr", True) is False else "memory-tight",
                    kw.get("L", 0) > 0, kw.get("template", 11)))
    assert ("memory-tight", False, 11) in routes and ("memory-tight", False, 15) in routes
    assert ("voxel", False, 11) in routes and ("voxel", True, 15) in routes


@pytest.mark.skipif(not __import__("oracle.refpy").refpy.available(),
                    reason="reference build not available")
@pytest.mark.parametrize("name", sorted(mg.GOLDEN_SGM))
def test_sgm_fixtures_are_the_reference_output(name):
    """The SGM fixtures (checked by tests/test_gpu_sgm.py) are what the
    reference build produces on the regenerated inputs."""
    from oracle import refpy
    inp = cases.make_case(**mg.GOLDEN_SGM[name])
    g = load_fixture(name)
    assert mg.input_digest(inp) == g["digest"]
    r = cases.run_cpu(refpy, inp, inp.iters)
    assert r["acc"] == g["acc"]
    for k in ("init_ncc", "vll_ncc", "ncc", "vll_vox"):
        assert cases.field_mismatch(r[k], g[k]) == {}, k


@pytest.mark.parametrize("name", sorted(mg.GOLDEN_VARIANTS))
def test_variant_fixture_inputs_are_reproducible(name):
    """The seeded variant cases rebuild the fixtures' exact inputs."""
    inp, z = mg.variant_case(name)
    assert mg.input_digest(inp) == str(z["digest"])
    assert np.array_equal(mg.clean(inp.gridpt3).view(np.uint8), z["init_gp3"])


@pytest.mark.skipif(not __import__("oracle.refpy").refpy.available(),
                    reason="reference build not available")
@pytest.mark.parametrize("name", sorted(mg.GOLDEN_VARIANTS))
def test_variant_fixtures_are_the_reference_output(name):
    from oracle import refpy
    v = mg.GOLDEN_VARIANTS[name]
    inp, z = mg.variant_case(name)
    if v["kind"] == "seeddem":
        refpy.vll_seeddem(inp)
    else:
        ncc = refpy.vll_blunder(inp, v["iteration"], v["bblunder"])
        assert np.array_equal(ncc.view(np.uint32), z["ncc"].view(np.uint32))
    assert np.array_equal(mg.clean(inp.gridpt3).view(np.uint8), z["gp3"])


@pytest.mark.skipif(not __import__("oracle.refpy").refpy.available(),
                    reason="reference build not available")
@pytest.mark.parametrize("name", sorted(mg.GOLDEN_TIN))
def test_tin_fixtures_are_the_reference_output(name):
    from oracle import refpy
    from setsm_b200 import abi
    inp, pts, tris, z = mg.tin_case(name)
    assert mg.image_digest(inp) == str(z["img_digest"])
    refpy.ortho_blunder(inp, mg.GOLDEN_TIN[name]["mpp"], pts, tris)
    assert np.array_equal(mg.clean(pts).view(np.uint8), z["pts"])
    assert np.array_equal(mg.clean(inp.gridpt3).view(np.uint8), z["gp3"])


@pytest.mark.skipif(not __import__("oracle.refpy").refpy.available(),
                    reason="reference build not available")
@pytest.mark.parametrize("name", sorted(mg.GOLDEN_RANGE))
def test_range_fixtures_are_the_reference_output(name):
    from oracle import refpy
    from setsm_b200 import abi
    v = mg.GOLDEN_RANGE[name]
    inp, pts, tris, z = mg.range_case(name)
    out, ext = refpy.set_height_range(inp, pts, tris, v["iteration"], v["mpp"], v["lcmr"],
                                      v.get("sigma", 0.0))
    assert np.array_equal(mg.clean(out).view(np.uint8), z["result"])
    assert ext == tuple(z["extent"])


@pytest.mark.skipif(not __import__("oracle.refpy").refpy.available(),
                    reason="reference build not available")
@pytest.mark.parametrize("name", sorted(mg.GOLDEN_SELECT))
def test_select_fixtures_are_the_reference_output(name):
    from oracle import refpy
    inp, ncc, z = mg.select_case(name)
    r, pts = refpy.select_mps(inp, ncc, *mg.GOLDEN_SELECT[name]["args"])
    assert r == int(z["ret"])
    assert np.array_equal(mg.clean(pts).view(np.uint8), z["pts"])
    assert np.array_equal(mg.clean(inp.gridpt3).view(np.uint8), z["gp3"])


@pytest.mark.skipif(not __import__("oracle.refpy").refpy.available(),
                    reason="reference build not available")
@pytest.mark.parametrize("name", sorted(mg.GOLDEN_TINB))
def test_tinb_fixtures_are_the_reference_output(name):
    from oracle import refpy
    inp, pts, tris, oncc, z = mg.tinb_case(name)
    it, fb, cbl, hint = mg.GOLDEN_TINB[name]["call"]
    det = np.zeros(len(pts), np.uint8)
    counts = np.zeros(2, np.int64)
    zext = np.array([1e5, -1e5])
    refpy.blunder_detection_tin(inp, it, oncc, fb, cbl, hint, pts, det, tris, counts, zext)
    assert np.array_equal(mg.clean(pts).view(np.uint8), z["pts"])
    assert np.array_equal(det, z["detected"])
    assert np.array_equal(counts, z["counts"]) and np.array_equal(zext, z["zext"])
