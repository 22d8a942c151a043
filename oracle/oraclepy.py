"""TEST INFRASTRUCTURE ONLY: ctypes access to the C restatement oracle.

Same Python surface as ``oracle.refpy`` (the reference build), so tests can
call both with identical arguments.  ``oracle/liboracle_vll.so`` is built by
``make -C oracle oracle`` (``__graft_entry__.build()`` does this).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from setsm_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_vll.so")

_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.vo_set_threads.argtypes = [C.c_int]
        L.vo_max_threads.restype = C.c_int
        L.vo_sobel.argtypes = [C.c_uint32, C.c_uint32, vp, vp, vp]
        L.vo_orientation.argtypes = [C.c_uint32, C.c_uint32, vp, vp, C.c_int, vp]
        L.vo_pyramid_down.argtypes = [C.c_uint32, C.c_uint32, vp, vp]
        L.vo_rpc_project.argtypes = [C.POINTER(abi.ImageDesc), C.c_long, vp, vp, vp, vp]
        L.vo_ps2wgs.argtypes = [C.POINTER(abi.TransParam), C.c_long, vp, vp]
        L.vo_initialize_voxel.argtypes = [C.POINTER(abi.LevelDesc), vp, vp, vp, vp, C.c_long]
        L.vo_initialize_voxel.restype = C.c_long
        L.vo_vertical_line_locus.argtypes = [C.POINTER(abi.LevelDesc), vp, vp, vp, C.c_long,
                                             vp, vp, vp]
        L.vo_vertical_line_locus.restype = C.c_long
        L.vo_awncc_peaks.argtypes = [C.POINTER(abi.LevelDesc), vp, vp, vp, C.c_long]
        L.vo_correlate.argtypes = [vp, vp, C.c_int]
        L.vo_correlate.restype = C.c_double
        L.vo_quantize_result.argtypes = [C.c_double]
        L.vo_quantize_result.restype = C.c_int16
        L.vo_quantize_voxel.argtypes = [C.c_double]
        L.vo_quantize_voxel.restype = C.c_int16
        L.vo_window_counts.argtypes = [C.c_int, vp]
        _lib = L
    return _lib


def set_threads(n: int) -> None:
    lib().vo_set_threads(int(n))


def max_threads() -> int:
    return int(lib().vo_max_threads())


def sobel(img: np.ndarray):
    img = np.ascontiguousarray(img, dtype=np.uint16)
    h, w = img.shape
    mag = np.zeros_like(img)
    d = np.zeros((h, w), dtype=np.int16)
    lib().vo_sobel(w, h, img.ctypes.data, mag.ctypes.data, d.ctypes.data)
    return mag, d


def orientation(mag: np.ndarray, direction: np.ndarray, template_size: int = 15):
    mag = np.ascontiguousarray(mag, dtype=np.uint16)
    direction = np.ascontiguousarray(direction, dtype=np.int16)
    h, w = mag.shape
    out = np.zeros((h, w), dtype=np.uint8)
    lib().vo_orientation(w, h, mag.ctypes.data, direction.ctypes.data, template_size,
                         out.ctypes.data)
    return out


def preprocess(img: np.ndarray, template_size: int = 15):
    mag, d = sobel(img)
    return mag, orientation(mag, d, template_size)


def pyramid_down(img: np.ndarray):
    img = np.ascontiguousarray(img, dtype=np.uint16)
    h, w = img.shape
    out = np.zeros((h // 2, w // 2), dtype=np.uint16)
    lib().vo_pyramid_down(w, h, img.ctypes.data, out.ctypes.data)
    return out


def rpc_project(rpc: np.ndarray, adjust, lon, lat, hgt):
    im = abi.ImageDesc()
    for k in range(90):
        im.rpc[k] = rpc[k]
    im.image_adjust[0], im.image_adjust[1] = adjust
    lon = np.ascontiguousarray(lon, dtype=np.float64).ravel()
    lat = np.ascontiguousarray(lat, dtype=np.float64).ravel()
    hgt = np.ascontiguousarray(hgt, dtype=np.float64).ravel()
    out = np.zeros((lon.size, 2))
    lib().vo_rpc_project(C.byref(im), lon.size, lon.ctypes.data, lat.ctypes.data,
                         hgt.ctypes.data, out.ctypes.data)
    return out


def ps2wgs(param: dict, xy: np.ndarray):
    tp = abi.TransParam()
    abi.set_transparam(tp, param)
    xy = np.ascontiguousarray(xy, dtype=np.float64).reshape(-1, 2)
    out = np.zeros_like(xy)
    lib().vo_ps2wgs(C.byref(tp), xy.shape[0], xy.ctypes.data, out.ctypes.data)
    return out


def voxel_count(ncc: np.ndarray) -> int:
    return int(ncc["NumOfHeight"].astype(np.int64).sum())


def initialize_voxel(inputs, ncc: np.ndarray, voxels_in: np.ndarray | None):
    d = inputs.desc()
    cap = int(((inputs.gridpt3["maxHeight"].astype(np.int64)
                - inputs.gridpt3["minHeight"].astype(np.int64) + 4)
               / inputs.height_step + 4).clip(0).sum())
    cap = max(cap, voxel_count(ncc), 1)
    out = np.zeros(cap, dtype=abi.VOXEL_DTYPE)
    vin = voxels_in.ctypes.data if voxels_in is not None and voxels_in.size else None
    n = lib().vo_initialize_voxel(C.byref(d), inputs.gridpt3.ctypes.data, ncc.ctypes.data,
                                  vin, out.ctypes.data, out.size)
    assert n <= out.size
    return out[:n].copy()


def heights_per_node(inputs, ncc: np.ndarray) -> np.ndarray:
    """Number of height slots per node that VerticalLineLocus will scan."""
    if inputs.check_matching_rate or inputs.is_ra:
        span = (inputs.gridpt3["maxHeight"].astype(np.int64)
                - inputs.gridpt3["minHeight"].astype(np.int64))
        return np.maximum((span / inputs.height_step).astype(np.int64), 0) & 0xFFFF
    return ncc["NumOfHeight"].astype(np.int64)


def vertical_line_locus(inputs, ncc: np.ndarray, voxels: np.ndarray | None = None,
                        want_rho: bool = False, want_evals: bool = False):
    """Returns Accessable_grid, or (Accessable_grid, rho, offsets, evals), or
    with `want_evals` (Accessable_grid, evals)."""
    d = inputs.desc()
    vp = voxels.ctypes.data if voxels is not None and voxels.size else None
    cap = voxels.size if voxels is not None else 0
    offs = rho = None
    ev = np.zeros(1, dtype=np.int64)
    if want_rho:
        k = heights_per_node(inputs, ncc)
        offs = np.concatenate([[0], np.cumsum(k)]).astype(np.int64)
        rho = np.full(max(int(offs[-1]), 1), np.nan)
    acc = int(lib().vo_vertical_line_locus(
        C.byref(d), inputs.gridpt3.ctypes.data, ncc.ctypes.data, vp, cap,
        offs.ctypes.data if offs is not None else None,
        rho.ctypes.data if rho is not None else None, ev.ctypes.data))
    if want_rho:
        return acc, rho, offs, int(ev[0])
    if want_evals:
        return acc, int(ev[0])
    return acc


def awncc(inputs, ncc: np.ndarray, voxels: np.ndarray) -> None:
    d = inputs.desc()
    vp = voxels.ctypes.data if voxels.size else None
    lib().vo_awncc_peaks(C.byref(d), inputs.gridpt3.ctypes.data, ncc.ctypes.data, vp,
                         voxels.size)


def correlate(left, right) -> float:
    """Correlate (SubFunctions.cpp:974-1018) on two equal-length vectors."""
    a = np.ascontiguousarray(left, dtype=np.float64)
    b = np.ascontiguousarray(right, dtype=np.float64)
    return float(lib().vo_correlate(a.ctypes.data, b.ctypes.data, int(min(a.size, b.size))))


def quantize_result(v: float) -> int:
    return int(lib().vo_quantize_result(float(v)))


def quantize_voxel(v: float) -> int:
    return int(lib().vo_quantize_voxel(float(v)))


def window_counts(half: int) -> tuple:
    out = np.zeros(3, dtype=np.int32)
    lib().vo_window_counts(int(half), out.ctypes.data)
    return tuple(int(x) for x in out)
