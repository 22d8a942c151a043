"""The C-ABI library without a GPU: it loads, exports every entry point that
include/setsm_vll.h declares plus the C++ VerticalLineLocus drop-in, and its
compatibility structures have the reference's byte layout (the drop-in reads
the caller's ProInfo / LevelInfo / NCCresult / UGRID / VOXEL in place).
No compute call is made here."""
import ctypes as C
import os
import re
import subprocess

import pytest

from oracle import refpy
from setsm_b200 import abi, vll

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "setsm_vll.h")
# setsm_code.hpp:81 -- int VerticalLineLocus(VOXEL**, const ProInfo*, NCCresult*,
#                       LevelInfo&, const UGRID*, const uint8, const double*)
DROPIN = "_Z17VerticalLineLocusPP12tagVoxelinfoPK11ProjectInfoP12tagNCCresultR12taglevelinfoPK10UpdateGridhPKd"


def declared_functions() -> list:
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(vll_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_entry_points():
    names = declared_functions()
    for must in ("vll_create", "vll_destroy", "vll_vertical_line_locus",
                 "vll_vertical_line_locus_device", "vll_awncc_peaks",
                 "vll_vertical_line_locus_noalloc"):
        assert must in names


def test_library_loads_and_exports_every_declared_symbol():
    L = vll.load()          # dlopen only; no CUDA call is made
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert missing == []
    for n in vll.EXPORTED:
        assert hasattr(L, n), n
    assert L.vll_abi_version() == abi.VLL_ABI_VERSION


def test_cpp_dropin_symbol_is_exported():
    L = vll.load()
    assert C.cast(getattr(L, DROPIN), C.c_void_p).value
    out = subprocess.run(["nm", "-D", "--defined-only", vll.LIB_PATH], capture_output=True,
                         text=True).stdout
    assert re.search(r"\bT " + DROPIN + r"\b", out)
    demangled = subprocess.run(["c++filt", DROPIN], capture_output=True, text=True).stdout
    assert demangled.startswith("VerticalLineLocus(tagVoxelinfo**, ProjectInfo const*")


# setsm_code.hpp:93 and :95, the orthoimage-window variants
VARIANTS = {
    "_Z25VerticalLineLocus_seeddemPK11ProjectInfoR12taglevelinfoP10UpdateGridPKd":
        "VerticalLineLocus_seeddem(ProjectInfo const*, taglevelinfo&, UpdateGrid*, double const*)",
    "_Z25VerticalLineLocus_blunderPK11ProjectInfoR12taglevelinfoPfP10UpdateGridhb":
        "VerticalLineLocus_blunder(ProjectInfo const*, taglevelinfo&, float*, UpdateGrid*, "
        "unsigned char, bool)",
}


def test_cpp_variant_dropins_are_exported():
    out = subprocess.run(["nm", "-D", "--defined-only", vll.LIB_PATH], capture_output=True,
                         text=True).stdout
    for sym, sig in VARIANTS.items():
        assert re.search(r"\bT " + sym + r"\b", out), sym
        demangled = subprocess.run(["c++filt", sym], capture_output=True, text=True).stdout
        assert demangled.strip() == sig


def test_record_sizes():
    assert abi.NCCRESULT_DTYPE.itemsize == 24
    assert abi.UGRID_DTYPE.itemsize == 20
    assert abi.VOXEL_DTYPE.itemsize == 4
    assert C.sizeof(abi.TransParam) == 112


@pytest.mark.skipif(not refpy.available(), reason="reference build not available")
def test_compat_layout_matches_reference_headers():
    ours = vll.compat_layout()
    ref = refpy.layout()
    assert len(ours) == len(ref) > 40
    assert ours == ref


def test_no_gpu_call_errors_cleanly_without_gpu():
    """Creating a context on a machine without a GPU returns a status code
    (never exits the process)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    L = vll.load()
    h = C.c_void_p()
    rc = L.vll_create(0, C.byref(h))
    assert rc == abi.VLL_ERR_CUDA
    assert b"" != L.vll_last_error(None)
