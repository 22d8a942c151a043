"""The orthoimage-window variants on the GPU (vll_ortho.cu) against the
reference: VerticalLineLocus_seeddem (setsm_code.cpp:7720-7880) and
VerticalLineLocus_blunder (:7882-8026).  The fixtures in tests/golden were
made by the reference build (tests/golden/make_golden.py); larger cases run
straight against the reference build where it is present.  Every UGRID field
and every float of the blunder NCC must be identical."""
import copy

import numpy as np
import pytest

from oracle import refpy
from setsm_b200 import abi
from tests import cases
from tests.golden import make_golden as mg

pytestmark = pytest.mark.gpu


def load_variant(name):
    v = mg.GOLDEN_VARIANTS[name]
    inp, z = mg.variant_case(name)
    assert mg.input_digest(inp) == str(z["digest"])
    assert np.array_equal(mg.clean(inp.gridpt3).view(np.uint8), z["init_gp3"])
    want_ncc = z["ncc"] if "ncc" in z.files else None
    return v, inp, z["gp3"].view(abi.UGRID_DTYPE), want_ncc


def run_gpu(ctx, v, inp):
    if v["kind"] == "seeddem":
        ctx.seeddem(inp)
        return None
    return ctx.blunder(inp, v["iteration"], v["bblunder"])


# The blunder pass's float NCC inherits the map projection's last-bit
# differences from the host's C library (about one raster coordinate in a
# thousand differs by an ulp, see setsm_b200/csrc/vll_ddmath.cuh), which move
# the double NCC by ~1e-10 and, rarely, its float rounding by one ulp.  The
# tolerance: identical floats on at least 99.5% of the nodes, and adjacent
# floats (one ulp, <= 6e-8 for |NCC| < 1) on the rest.  The UGRID fields
# (quantised to 1e-3) must be identical.
NCC_MAX_ULPS = 1
NCC_EXACT_FRAC = 0.995


def assert_same(gp3, want_gp3, ncc=None, want_ncc=None):
    assert cases.field_mismatch(mg.clean(gp3), mg.clean(want_gp3)) == {}
    if want_ncc is not None:
        a = ncc.astype(np.float32).view(np.int32).astype(np.int64)
        b = want_ncc.astype(np.float32).view(np.int32).astype(np.int64)
        same = a == b
        assert same.mean() >= NCC_EXACT_FRAC, (int((~same).sum()), len(same))
        assert np.all(np.sign(ncc) == np.sign(want_ncc))
        assert np.abs(a - b).max() <= NCC_MAX_ULPS


@pytest.mark.parametrize("name", sorted(mg.GOLDEN_VARIANTS))
def test_variant_matches_reference_fixture(gpu_ctx, name):
    v, inp, want_gp3, want_ncc = load_variant(name)
    ncc = run_gpu(gpu_ctx, v, inp)
    assert_same(inp.gridpt3, want_gp3, ncc, want_ncc)


@pytest.mark.parametrize("name", sorted(mg.GOLDEN_VARIANTS))
def test_variant_device_entry_point(gpu_ctx, name):
    """The _device entry points on resident data give the same records."""
    import torch
    v, inp, want_gp3, want_ncc = load_variant(name)
    io, keep = cases.device_level(torch, inp, inp.new_nccresult())
    torch.cuda.synchronize()    # the copies ran on torch's stream, the calls use the context's
    d = io[0]
    if v["kind"] == "seeddem":
        gpu_ctx.seeddem_device(d, io[1])
        torch.cuda.synchronize()    # the device calls return before their kernels finish
    else:
        out = torch.zeros(inp.n, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        gpu_ctx.blunder_device(d, io[1], v["iteration"], v["bblunder"], out.data_ptr())
        torch.cuda.synchronize()
        assert_same(want_gp3, want_gp3, out.cpu().numpy(), want_ncc)
    gp3 = cases.from_device(keep["gp3"], abi.UGRID_DTYPE)
    assert cases.field_mismatch(mg.clean(gp3), mg.clean(want_gp3)) == {}


@pytest.mark.skipif(not refpy.available(), reason="reference build not available")
@pytest.mark.parametrize("kind,kw", [
    ("seeddem", dict(seed=21, size=768, nodes=48, res=7.0, L=0)),
    ("seeddem", dict(seed=22, size=768, nodes=40, res=9.0, L=1, template=15, matchtag=True,
                     blunder_level=1)),
    ("seeddem", dict(seed=23, size=768, nodes=32, res=12.0, L=2, template=15,
                     minmax=(0.0, 180.0))),
    ("blunder1", dict(seed=24, size=768, nodes=48, res=7.0, L=0, blunder_level=1)),
    ("blunder1", dict(seed=25, size=768, nodes=32, res=12.0, L=2, blunder_level=2)),
    ("blunder2", dict(seed=26, size=768, nodes=24, res=16.0, L=4, template=15, blunder_level=3)),
    ("blunder3", dict(seed=27, size=768, nodes=24, res=16.0, L=3, template=15, blunder_level=3)),
    # three images: ortho_ncc[2] lands on Mean_ortho_ncc as in the reference
    ("seeddem", dict(seed=28, size=512, nodes=32, res=8.0, L=0, n_images=3)),
    ("blunder1", dict(seed=29, size=512, nodes=32, res=8.0, L=0, blunder_level=1, n_images=3)),
])
def test_variant_matches_reference_build(gpu_ctx, kind, kw):
    inp = cases.make_variant_case(**kw)
    ref = copy.copy(inp)
    ref.gridpt3 = inp.gridpt3.copy()
    if kind == "seeddem":
        refpy.vll_seeddem(ref)
        gpu_ctx.seeddem(inp)
        assert_same(inp.gridpt3, ref.gridpt3)
    else:
        it, bb = {"blunder1": (1, False), "blunder2": (3, True), "blunder3": (1, True)}[kind]
        want = refpy.vll_blunder(ref, it, bb)
        got = gpu_ctx.blunder(inp, it, bb)
        assert_same(inp.gridpt3, ref.gridpt3, got, want)


def test_variant_rejects_bad_descriptor(gpu_ctx):
    from setsm_b200 import vll
    inp = cases.make_variant_case(seed=5, nodes=12, res=16.0, L=0, blunder_level=1)
    inp.images[1].image_b = inp.images[1].image_b[:1, :1].copy()
    inp.images[1].mag_b = inp.images[1].mag_b[:1, :1].copy()
    with pytest.raises(vll.VLLError):
        gpu_ctx.blunder(inp, 1, False)


@pytest.mark.skipif(not refpy.available(), reason="reference build not available")
@pytest.mark.parametrize("name", sorted(mg.GOLDEN_VARIANTS))
def test_variant_cpp_dropins_through_reference_structures(gpu_ctx, name):
    """The C++ drop-ins (setsm_code.hpp:93, :95) called with ProInfo /
    LevelInfo built by the reference's own headers."""
    import ctypes as C
    from setsm_b200 import vll
    from tests.test_abi_layout import VARIANTS
    v, inp, want_gp3, want_ncc = load_variant(name)
    sym = [k for k in VARIANTS if ("seeddem" in k) == (v["kind"] == "seeddem")][0]
    fn = C.cast(getattr(vll.load(), sym), C.c_void_p).value
    if v["kind"] == "seeddem":
        refpy.call_vll_seeddem(fn, inp)
        ncc = None
    else:
        ncc = refpy.call_vll_blunder(fn, inp, v["iteration"], v["bblunder"])
    assert_same(inp.gridpt3, want_gp3, ncc, want_ncc)


@pytest.mark.skipif(not refpy.available(), reason="reference build not available")
@pytest.mark.parametrize("use_b", [0, 1])
def test_ortho_raster_matches_reference(gpu_ctx, use_b):
    """SetOrthoImageCoord on the GPU against the reference's: identical but
    for the rare last-bit differences of the map projection's libm calls."""
    import ctypes as C
    from setsm_b200 import vll
    L = vll.load()
    L.vll_debug_ortho_raster.argtypes = [C.c_void_p, C.POINTER(abi.LevelDesc), C.c_void_p,
                                         C.c_int, C.c_double, C.c_int, C.c_void_p, C.c_int64,
                                         C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    R = refpy.lib()
    R.ref_ortho_raster.argtypes = [C.POINTER(abi.LevelDesc), C.c_void_p, C.c_int, C.c_double,
                                   C.c_int, C.c_void_p, C.c_long]
    R.ref_ortho_raster.restype = C.c_long
    inp = cases.make_variant_case(seed=24, size=768, nodes=48, res=7.0, L=0, blunder_level=1)
    d = inp.desc()
    res = inp.resolution * 2 ** (inp.blunder_level if use_b else inp.pyramid_step)
    cap = 1 << 20
    for ti in range(2):
        got = np.zeros(2 * cap)
        want = np.zeros(2 * cap)
        w, h = C.c_int64(), C.c_int64()
        rc = L.vll_debug_ortho_raster(gpu_ctx._h, C.byref(d), inp.gridpt3.ctypes.data, use_b,
                                      res, ti, got.ctypes.data, cap, C.byref(w), C.byref(h))
        assert rc == abi.VLL_OK
        n = R.ref_ortho_raster(C.byref(d), inp.gridpt3.ctypes.data, use_b, res, ti,
                               want.ctypes.data, cap)
        assert n == w.value * h.value > 0
        diff = got[:2 * n] != want[:2 * n]
        assert diff.mean() < 0.005, int(diff.sum())
        assert np.abs(got[:2 * n] - want[:2 * n]).max() < 1e-7
