"""TEST INFRASTRUCTURE ONLY: ctypes access to the reference SETSM build.

``oracle/_ref/libsetsm_ref.so`` is the reference's own code (setsm_code.cpp,
SubFunctions.cpp, CoordConversion.cpp, ...) compiled by ``make -C oracle ref``
with stubbed TIFF I/O, plus the marshalling harness oracle/ref_harness.cpp.
The same Python surface is offered by ``oracle.oraclepy`` for the C
restatement so the two can be compared call for call.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from setsm_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libsetsm_ref.so")

_lib = None


class _StdoutToStderr:
    """Sends the reference's own printf output (file descriptor 1) to stderr
    while a reference call runs, so a caller's stdout carries only its own
    output (bench.py prints one JSON line there)."""

    def __enter__(self):
        import sys
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *exc):
        C.CDLL(None).fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)
        return False


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB_PATH} not built (make -C oracle ref)")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.ref_initialize_voxel.argtypes = [C.POINTER(abi.LevelDesc), vp, vp, vp, vp, C.c_long]
        L.ref_initialize_voxel.restype = C.c_long
        L.ref_vertical_line_locus.argtypes = [C.POINTER(abi.LevelDesc), vp, vp, vp, C.c_long]
        L.ref_vertical_line_locus.restype = C.c_long
        L.ref_awncc.argtypes = [C.POINTER(abi.LevelDesc), vp, vp, vp, C.c_long]
        L.ref_awncc.restype = None
        L.ref_sobel.argtypes = [C.c_uint32, C.c_uint32, vp, vp, vp]
        L.ref_tin_create.argtypes = [vp, C.c_long, vp, C.c_double, vp, C.c_long]
        L.ref_tin_create.restype = C.c_long
        L.ref_orientation.argtypes = [C.c_uint32, C.c_uint32, vp, vp, C.c_int, vp]
        L.ref_pyramid_down.argtypes = [C.c_uint32, C.c_uint32, vp, vp]
        L.ref_rpc_project.argtypes = [C.POINTER(abi.ImageDesc), C.c_long, vp, vp, vp, vp]
        L.ref_ps2wgs.argtypes = [C.POINTER(abi.TransParam), C.c_long, vp, vp]
        L.ref_wgs2ps.argtypes = [C.POINTER(abi.TransParam), C.c_long, vp, vp]
        L.ref_set_transparam.argtypes = [C.c_int, C.c_int, C.POINTER(abi.TransParam)]
        L.ref_get_height_step.argtypes = [C.c_int, C.c_double]
        L.ref_get_height_step.restype = C.c_double
        L.ref_set_threads.argtypes = [C.c_int]
        L.ref_max_threads.restype = C.c_int
        for f in ("ref_sizeof_nccresult", "ref_sizeof_ugrid", "ref_sizeof_voxel",
                  "ref_sizeof_transparam"):
            getattr(L, f).restype = C.c_int
        _lib = L
    return _lib


def set_threads(n: int) -> None:
    lib().ref_set_threads(int(n))


def max_threads() -> int:
    return int(lib().ref_max_threads())


def sizes() -> dict:
    L = lib()
    return {"NCCresult": L.ref_sizeof_nccresult(), "UGRID": L.ref_sizeof_ugrid(),
            "VOXEL": L.ref_sizeof_voxel(), "TransParam": L.ref_sizeof_transparam()}


# ---- image preprocessing ---------------------------------------------------
def sobel(img: np.ndarray):
    img = np.ascontiguousarray(img, dtype=np.uint16)
    h, w = img.shape
    mag = np.zeros_like(img)
    d = np.zeros((h, w), dtype=np.int16)
    lib().ref_sobel(w, h, img.ctypes.data, mag.ctypes.data, d.ctypes.data)
    return mag, d


def orientation(mag: np.ndarray, direction: np.ndarray, template_size: int = 15):
    mag = np.ascontiguousarray(mag, dtype=np.uint16)
    direction = np.ascontiguousarray(direction, dtype=np.int16)
    h, w = mag.shape
    out = np.zeros((h, w), dtype=np.uint8)
    lib().ref_orientation(w, h, mag.ctypes.data, direction.ctypes.data, template_size,
                          out.ctypes.data)
    return out


def preprocess(img: np.ndarray, template_size: int = 15):
    """Magnitude and orientation images the way SetPyramidImages builds them."""
    mag, d = sobel(img)
    return mag, orientation(mag, d, template_size)


def pyramid_down(img: np.ndarray):
    img = np.ascontiguousarray(img, dtype=np.uint16)
    h, w = img.shape
    out = np.zeros((h // 2, w // 2), dtype=np.uint16)
    lib().ref_pyramid_down(w, h, img.ctypes.data, out.ctypes.data)
    return out


# ---- geometry ----------------------------------------------------------------
def rpc_project(rpc: np.ndarray, adjust, lon, lat, hgt):
    im = abi.ImageDesc()
    for k in range(90):
        im.rpc[k] = rpc[k]
    im.image_adjust[0], im.image_adjust[1] = adjust
    lon = np.ascontiguousarray(lon, dtype=np.float64).ravel()
    lat = np.ascontiguousarray(lat, dtype=np.float64).ravel()
    hgt = np.ascontiguousarray(hgt, dtype=np.float64).ravel()
    out = np.zeros((lon.size, 2))
    lib().ref_rpc_project(C.byref(im), lon.size, lon.ctypes.data, lat.ctypes.data,
                          hgt.ctypes.data, out.ctypes.data)
    return out


def ps2wgs(param: dict, xy: np.ndarray):
    tp = abi.TransParam()
    abi.set_transparam(tp, param)
    xy = np.ascontiguousarray(xy, dtype=np.float64).reshape(-1, 2)
    out = np.zeros_like(xy)
    lib().ref_ps2wgs(C.byref(tp), xy.shape[0], xy.ctypes.data, out.ctypes.data)
    return out


def wgs2ps(param: dict, lonlat: np.ndarray):
    tp = abi.TransParam()
    abi.set_transparam(tp, param)
    ll = np.ascontiguousarray(lonlat, dtype=np.float64).reshape(-1, 2)
    out = np.zeros_like(ll)
    lib().ref_wgs2ps(C.byref(tp), ll.shape[0], ll.ctypes.data, out.ctypes.data)
    return out


def transparam(north: bool = True, projection: int = 1) -> dict:
    tp = abi.TransParam()
    lib().ref_set_transparam(int(north), projection, C.byref(tp))
    return abi.transparam_dict(tp)


def height_step(pyramid_step: int, im_resolution: float) -> float:
    return float(lib().ref_get_height_step(pyramid_step, im_resolution))


# ---- the hot path --------------------------------------------------------------
def voxel_count(ncc: np.ndarray) -> int:
    return int(ncc["NumOfHeight"].astype(np.int64).sum())


def initialize_voxel(inputs, ncc: np.ndarray, voxels_in: np.ndarray | None):
    """InitializeVoxel; returns the packed voxel rows by the updated NumOfHeight.

    Modifies ``inputs.gridpt3`` and ``ncc`` in place like the reference."""
    d = inputs.desc()
    # worst case: every node gets the full range
    cap = int(((inputs.gridpt3["maxHeight"].astype(np.int64)
                - inputs.gridpt3["minHeight"].astype(np.int64) + 4)
               / inputs.height_step + 4).clip(0).sum())
    out = np.zeros(max(cap, 1), dtype=abi.VOXEL_DTYPE)
    vin = voxels_in.ctypes.data if voxels_in is not None and voxels_in.size else None
    with _StdoutToStderr():
        n = lib().ref_initialize_voxel(C.byref(d), inputs.gridpt3.ctypes.data, ncc.ctypes.data,
                                       vin, out.ctypes.data, out.size)
    assert n <= out.size
    return out[:n].copy()


def vertical_line_locus(inputs, ncc: np.ndarray, voxels: np.ndarray | None = None) -> int:
    d = inputs.desc()
    vp = voxels.ctypes.data if voxels is not None and voxels.size else None
    cap = voxels.size if voxels is not None else 0
    with _StdoutToStderr():
        return int(lib().ref_vertical_line_locus(C.byref(d), inputs.gridpt3.ctypes.data,
                                                 ncc.ctypes.data, vp, cap))


def awncc(inputs, ncc: np.ndarray, voxels: np.ndarray) -> None:
    d = inputs.desc()
    vp = voxels.ctypes.data if voxels.size else None
    with _StdoutToStderr():
        lib().ref_awncc(C.byref(d), inputs.gridpt3.ctypes.data, ncc.ctypes.data, vp, voxels.size)


def _kat_lib():
    L = lib()
    if not getattr(L, "_kat", False):
        L.ref_correlate.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        L.ref_correlate.restype = C.c_double
        L.ref_window_counts.argtypes = [C.c_int, C.c_void_p]
        L.ref_call_vertical_line_locus.argtypes = [C.c_void_p, C.POINTER(abi.LevelDesc),
                                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_long]
        L.ref_call_vertical_line_locus.restype = C.c_long
        L._kat = True
    return L


def correlate(left, right) -> float:
    """The reference's Correlate (SubFunctions.cpp:974-1018)."""
    a = np.ascontiguousarray(left, dtype=np.float64)
    b = np.ascontiguousarray(right, dtype=np.float64)
    return float(_kat_lib().ref_correlate(a.ctypes.data, b.ctypes.data, int(min(a.size, b.size))))


def window_counts(half: int) -> tuple:
    """Sub-window counts of the reference's SetVecKernelValue window loop."""
    out = np.zeros(3, dtype=np.int32)
    _kat_lib().ref_window_counts(int(half), out.ctypes.data)
    return tuple(int(x) for x in out)


def call_vertical_line_locus(fn_addr: int, inputs, ncc: np.ndarray, voxels=None) -> int:
    """Calls the function at `fn_addr` (VerticalLineLocus's C++ signature,
    setsm_code.hpp:81) with structures built from the reference's headers."""
    d = inputs.desc()
    vp = voxels.ctypes.data if voxels is not None else None
    cap = voxels.size if voxels is not None else 0
    with _StdoutToStderr():
        return int(_kat_lib().ref_call_vertical_line_locus(fn_addr, C.byref(d),
                                                          inputs.gridpt3.ctypes.data,
                                                          ncc.ctypes.data, vp, cap))


def layout() -> list:
    """Byte offsets and sizes of the reference structures the drop-in reads,
    from the reference's own headers (same order as vll_compat_layout)."""
    L = lib()
    L.ref_layout.argtypes = [C.c_void_p, C.c_int]
    L.ref_layout.restype = C.c_int
    out = np.zeros(128, dtype=np.int64)
    n = L.ref_layout(out.ctypes.data, out.size)
    return out[:n].tolist()


def vll_seeddem(inputs) -> None:
    """VerticalLineLocus_seeddem (setsm_code.cpp:7720-7880); updates
    inputs.gridpt3 in place."""
    L = lib()
    L.ref_vll_seeddem.argtypes = [C.POINTER(abi.LevelDesc), C.c_void_p]
    L.ref_vll_seeddem.restype = None
    d = inputs.desc()
    with _StdoutToStderr():
        L.ref_vll_seeddem(C.byref(d), inputs.gridpt3.ctypes.data)


def vll_blunder(inputs, iteration: int, bblunder: bool) -> np.ndarray:
    """VerticalLineLocus_blunder (setsm_code.cpp:7882-8026); updates
    inputs.gridpt3 in place and returns the per-node ortho NCC."""
    L = lib()
    L.ref_vll_blunder.argtypes = [C.POINTER(abi.LevelDesc), C.c_void_p, C.c_int, C.c_int,
                                  C.c_void_p]
    L.ref_vll_blunder.restype = None
    d = inputs.desc()
    out = np.zeros(inputs.n, dtype=np.float32)
    with _StdoutToStderr():
        L.ref_vll_blunder(C.byref(d), inputs.gridpt3.ctypes.data, int(iteration), int(bblunder),
                          out.ctypes.data)
    return out


def call_vll_seeddem(fn_addr: int, inputs) -> None:
    """Calls the function at `fn_addr` (VerticalLineLocus_seeddem's C++
    signature, setsm_code.hpp:93) with the reference's structures."""
    L = lib()
    L.ref_call_vll_seeddem.argtypes = [C.c_void_p, C.POINTER(abi.LevelDesc), C.c_void_p]
    L.ref_call_vll_seeddem.restype = None
    d = inputs.desc()
    with _StdoutToStderr():
        L.ref_call_vll_seeddem(fn_addr, C.byref(d), inputs.gridpt3.ctypes.data)


def call_vll_blunder(fn_addr: int, inputs, iteration: int, bblunder: bool) -> np.ndarray:
    """Calls the function at `fn_addr` (VerticalLineLocus_blunder's C++
    signature, setsm_code.hpp:95) with the reference's structures."""
    L = lib()
    L.ref_call_vll_blunder.argtypes = [C.c_void_p, C.POINTER(abi.LevelDesc), C.c_void_p, C.c_int,
                                       C.c_int, C.c_void_p]
    L.ref_call_vll_blunder.restype = C.c_int
    d = inputs.desc()
    out = np.zeros(inputs.n, dtype=np.float32)
    with _StdoutToStderr():
        ok = L.ref_call_vll_blunder(fn_addr, C.byref(d), inputs.gridpt3.ctypes.data,
                                    int(iteration), int(bblunder), out.ctypes.data)
    assert ok == 1
    return out


def vll_ortho(inputs, mpp: float, three: np.ndarray, target_index: int):
    """VerticalLineLocus_Ortho (setsm_code.cpp:8234-8533) for the triangle
    three = (ref1, ref2, target) (abi.POINT3_DTYPE); returns (return value,
    F_Height, F_sncc) with F_sncc NaN when the function leaves it unset."""
    L = lib()
    L.ref_vll_ortho.argtypes = [C.POINTER(abi.LevelDesc), C.c_double, C.c_void_p, C.c_void_p,
                                C.c_int, C.c_void_p]
    L.ref_vll_ortho.restype = C.c_int
    d = inputs.desc()
    three = np.ascontiguousarray(three, dtype=abi.POINT3_DTYPE)
    out = np.array([0.0, np.nan])
    with _StdoutToStderr():
        r = L.ref_vll_ortho(C.byref(d), float(mpp), three.ctypes.data, inputs.gridpt3.ctypes.data,
                            int(target_index), out.ctypes.data)
    return int(r), float(out[0]), float(out[1])


def ortho_blunder(inputs, mpp: float, pts: np.ndarray, tris: np.ndarray) -> int:
    """Ortho_blunder (setsm_code.cpp:8028-8232); pts, tris and
    inputs.gridpt3 are updated in place."""
    L = lib()
    L.ref_ortho_blunder.argtypes = [C.POINTER(abi.LevelDesc), C.c_double, C.c_void_p, C.c_int,
                                    C.c_void_p, C.c_int, C.c_void_p]
    L.ref_ortho_blunder.restype = C.c_int
    d = inputs.desc()
    with _StdoutToStderr():
        return int(L.ref_ortho_blunder(C.byref(d), float(mpp), pts.ctypes.data, len(pts),
                                       tris.ctypes.data, len(tris), inputs.gridpt3.ctypes.data))


def call_vll_ortho(fn_addr: int, inputs, mpp: float, three: np.ndarray, target_index: int):
    """As vll_ortho, through the function at fn_addr (setsm_code.hpp:97 signature)."""
    L = lib()
    L.ref_call_vll_ortho.argtypes = [C.c_void_p, C.POINTER(abi.LevelDesc), C.c_double, C.c_void_p,
                                     C.c_void_p, C.c_int, C.c_void_p]
    L.ref_call_vll_ortho.restype = C.c_int
    d = inputs.desc()
    three = np.ascontiguousarray(three, dtype=abi.POINT3_DTYPE)
    out = np.array([0.0, np.nan])
    with _StdoutToStderr():
        r = L.ref_call_vll_ortho(fn_addr, C.byref(d), float(mpp), three.ctypes.data,
                                 inputs.gridpt3.ctypes.data, int(target_index), out.ctypes.data)
    return int(r), float(out[0]), float(out[1])


def call_ortho_blunder(fn_addr: int, inputs, mpp: float, pts: np.ndarray, tris: np.ndarray) -> int:
    """As ortho_blunder, through the function at fn_addr (setsm_code.hpp:118)."""
    L = lib()
    L.ref_call_ortho_blunder.argtypes = [C.c_void_p, C.POINTER(abi.LevelDesc), C.c_double,
                                         C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p]
    L.ref_call_ortho_blunder.restype = C.c_int
    d = inputs.desc()
    with _StdoutToStderr():
        return int(L.ref_call_ortho_blunder(fn_addr, C.byref(d), float(mpp), pts.ctypes.data,
                                            len(pts), tris.ctypes.data, len(tris),
                                            inputs.gridpt3.ctypes.data))


def set_height_range(inputs, pts, tris, iteration: int, mpp: float, lcmr: bool,
                     seed_sigma: float = 0.0, fn_addr: int | None = None):
    """SetHeightRange (setsm_code.cpp:9851-10255), or the function at
    fn_addr with its signature (setsm_code.hpp:122); inputs.gridpt3 is left
    unchanged.  Returns (result grid, (minH_grid, maxH_grid))."""
    L = lib()
    L.ref_set_height_range.argtypes = [C.c_void_p, C.POINTER(abi.LevelDesc), C.c_void_p, C.c_int,
                                       C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                       C.c_double, C.c_int, C.c_double, C.c_void_p]
    L.ref_set_height_range.restype = C.c_int
    d = inputs.desc()
    out = np.zeros(inputs.n, dtype=abi.UGRID_DTYPE)
    ext = np.zeros(2)
    with _StdoutToStderr():
        L.ref_set_height_range(fn_addr, C.byref(d), pts.ctypes.data, len(pts), tris.ctypes.data,
                               len(tris), inputs.gridpt3.ctypes.data, out.ctypes.data,
                               int(iteration), float(mpp), int(bool(lcmr)), float(seed_sigma),
                               ext.ctypes.data)
    return out, (float(ext[0]), float(ext[1]))


def select_mps(inputs, ncc, th_roh, th_roh_min, th_roh_start, th_roh_next, iteration, mpp,
               final_level_iteration, mpp_stereo_angle, fn_addr: int | None = None):
    """SelectMPs (setsm_code.cpp:8535-8895), or the function at fn_addr with
    its signature (setsm_code.hpp:99); inputs.gridpt3 updated in place.
    Returns (return value, points)."""
    L = lib()
    L.ref_select_mps.argtypes = [C.c_void_p, C.POINTER(abi.LevelDesc), C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_void_p, C.c_void_p, C.c_long,
                                 C.POINTER(C.c_long)]
    L.ref_select_mps.restype = C.c_long
    d = inputs.desc()
    params = np.array([th_roh, th_roh_min, th_roh_start, th_roh_next, mpp, mpp_stereo_angle],
                      dtype=np.float64)
    iparams = np.array([iteration, final_level_iteration], dtype=np.int32)
    out = np.zeros(inputs.n, dtype=abi.POINT3_DTYPE)
    n = C.c_long()
    with _StdoutToStderr():
        r = L.ref_select_mps(fn_addr, C.byref(d), ncc.ctypes.data, inputs.gridpt3.ctypes.data,
                             params.ctypes.data, iparams.ctypes.data, out.ctypes.data, len(out),
                             C.byref(n))
    return int(r), out[: n.value].copy()


def call_initialize_voxel(fn_addr: int, inputs, ncc, voxels_in):
    """InitializeVoxel through the function at fn_addr (setsm_code.hpp:75)."""
    L = lib()
    L.ref_call_initialize_voxel.argtypes = [C.c_void_p, C.POINTER(abi.LevelDesc), C.c_void_p,
                                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_long]
    L.ref_call_initialize_voxel.restype = C.c_long
    d = inputs.desc()
    cap = int(((inputs.gridpt3["maxHeight"].astype(np.int64)
                - inputs.gridpt3["minHeight"].astype(np.int64) + 4)
               / inputs.height_step + 4).clip(0).sum())
    cap = max(cap, int(ncc["NumOfHeight"].astype(np.int64).sum()), 1)
    out = np.zeros(cap, dtype=abi.VOXEL_DTYPE)
    vin = voxels_in.ctypes.data if voxels_in is not None and voxels_in.size else None
    with _StdoutToStderr():
        n = L.ref_call_initialize_voxel(fn_addr, C.byref(d), inputs.gridpt3.ctypes.data,
                                        ncc.ctypes.data, vin, out.ctypes.data, out.size)
    assert n <= out.size
    return out[:n].copy()


def call_awncc(fn_addr: int, inputs, ncc, voxels) -> None:
    """AWNCC through the function at fn_addr (setsm_code.hpp:91)."""
    L = lib()
    L.ref_call_awncc.argtypes = [C.c_void_p, C.POINTER(abi.LevelDesc), C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_long]
    L.ref_call_awncc.restype = None
    d = inputs.desc()
    with _StdoutToStderr():
        L.ref_call_awncc(fn_addr, C.byref(d), inputs.gridpt3.ctypes.data, ncc.ctypes.data,
                         voxels.ctypes.data, voxels.size)


def blunder_detection_tin(inputs, iteration, ortho_ncc, flag_blunder, count_bl, hinterval, pts,
                          detected, tris, counts, zext, fn_addr: int | None = None) -> int:
    """blunder_detection_TIN (setsm_code.cpp:9158-9787), or the function at
    fn_addr with its signature (setsm_code.hpp:116).  pts, detected (uint8),
    inputs.gridpt3, counts (int64[2]) and zext (float64[2]: min, max) are
    updated in place."""
    L = lib()
    L.ref_blunder_detection_tin.argtypes = [C.c_void_p, C.POINTER(abi.LevelDesc), C.c_int,
                                            C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_void_p,
                                            C.c_void_p, C.c_long, C.c_void_p, C.c_long,
                                            C.c_void_p, C.c_void_p, C.c_void_p]
    L.ref_blunder_detection_tin.restype = C.c_int
    d = inputs.desc()
    with _StdoutToStderr():
        return int(L.ref_blunder_detection_tin(
            fn_addr, C.byref(d), int(iteration), ortho_ncc.ctypes.data, int(bool(flag_blunder)),
            int(count_bl), float(hinterval), pts.ctypes.data, detected.ctypes.data, len(pts),
            tris.ctypes.data, len(tris), inputs.gridpt3.ctypes.data, counts.ctypes.data,
            zext.ctypes.data))


def tin_create(pts: np.ndarray, min_max, resolution: float) -> np.ndarray:
    """The reference's TINCreate_list (SubFunctions.cpp:2768-2846): its ordered
    triangle list (vertex indices) of the points."""
    pts = np.ascontiguousarray(pts, dtype=abi.POINT3_DTYPE)
    mm = np.ascontiguousarray(min_max, dtype=np.float64)
    cap = 2 * len(pts) + 16
    while True:
        out = np.zeros(cap, dtype=abi.TRI_DTYPE)
        with _StdoutToStderr():
            n = lib().ref_tin_create(pts.ctypes.data, len(pts), mm.ctypes.data, float(resolution),
                                     out.ctypes.data, cap)
        if n <= cap:
            return out[:n]
        cap = n


def call_voxel_iterations(fns, inputs, ncc: np.ndarray, iters) -> list:
    """InitializeVoxel -> VerticalLineLocus -> AWNCC per iteration on one
    VOXEL** array, through the functions at fns = (init, vll, awncc)
    addresses (None: the reference's own); gridpt3 / ncc in place.  Returns
    each iteration's Accessable_grid."""
    L = lib()
    vp = C.c_void_p
    L.ref_call_voxel_iterations.argtypes = [vp, vp, vp, C.POINTER(abi.LevelDesc), vp, vp, C.c_int,
                                            vp, vp]
    L.ref_call_voxel_iterations.restype = None
    d = inputs.desc()
    it = np.ascontiguousarray(iters, dtype=np.int32)
    acc = np.zeros(len(it), dtype=np.int64)
    with _StdoutToStderr():
        L.ref_call_voxel_iterations(fns[0], fns[1], fns[2], C.byref(d), inputs.gridpt3.ctypes.data,
                                    ncc.ctypes.data, len(it), it.ctypes.data, acc.ctypes.data)
    return [int(a) for a in acc]
