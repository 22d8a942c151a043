"""Python host interface of the B200 vertical-line-locus matcher.

Mirrors the reference's operator surface for this path
(VerticalLineLocus, setsm_code.cpp:6049; AWNCC's peak loop, :7511;
MakeSobelMagnitudeImage + Orientation, SubFunctions.cpp:2418/:2473;
CreateImagePyramid, Template.hpp:82) over the C ABI of include/setsm_vll.h.
Everything runs in ``setsm_b200/lib/libsetsm_vll.so`` on the GPU; if that
library is missing or no GPU is present the calls raise -- there is no CPU
path in the product.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
# SETSM_VLL_LIB selects another build of the library (e.g. a tuning variant)
LIB_PATH = os.environ.get("SETSM_VLL_LIB") or os.path.join(HERE, "lib", "libsetsm_vll.so")

KERNELS = {"plain": abi.VLL_KERNEL_FP64_PLAIN, "split": abi.VLL_KERNEL_SPLIT}

EXPORTED = [
    "vll_abi_version", "vll_last_error", "vll_create", "vll_destroy", "vll_set_stream",
    "vll_get_stream", "vll_voxel_count", "vll_vertical_line_locus",
    "vll_vertical_line_locus_device", "vll_awncc_peaks", "vll_preprocess_level",
    "vll_preprocess_level_device", "vll_pyramid_down", "vll_pyramid_down_device",
    "vll_compat_layout", "vll_launch_count", "vll_debug_slot_rho",
    "vll_vertical_line_locus_batch", "vll_plan_create", "vll_plan_run", "vll_plan_destroy",
    "vll_set_tuning", "vll_get_tuning",
    "vll_vertical_line_locus_seeddem", "vll_vertical_line_locus_seeddem_device",
    "vll_vertical_line_locus_blunder", "vll_vertical_line_locus_blunder_device",
    "vll_vertical_line_locus_ortho", "vll_ortho_blunder", "vll_ortho_blunder_device",
    "vll_set_height_range", "vll_select_mps", "vll_initialize_voxel",
    "vll_initialize_voxel_device", "vll_awncc_peaks_device", "vll_select_mps_device",
    "vll_set_height_range_device", "vll_blunder_detection_tin",
    "vll_blunder_detection_tin_device", "vll_tin_rerun_count", "vll_debug_tin_threshold",
    "vll_tin_create", "vll_tin_create_device",
    "vll_set_residency", "vll_get_residency", "vll_resident_reset", "vll_resident_voxels",
]

_lib = None


class VLLError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{abi.STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def load():
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(
            f"{LIB_PATH} is missing: build it with `python -m setsm_b200.build` "
            "(the matcher has no CPU implementation)")
    L = C.CDLL(LIB_PATH)
    vp, i64, i32 = C.c_void_p, C.c_int64, C.c_int
    L.vll_abi_version.restype = i32
    L.vll_last_error.argtypes = [vp]
    L.vll_last_error.restype = C.c_char_p
    L.vll_create.argtypes = [i32, C.POINTER(vp)]
    L.vll_destroy.argtypes = [vp]
    L.vll_destroy.restype = None
    L.vll_set_stream.argtypes = [vp, vp]
    L.vll_get_stream.argtypes = [vp]
    L.vll_get_stream.restype = vp
    L.vll_voxel_count.argtypes = [vp, i64]
    L.vll_voxel_count.restype = i64
    L.vll_vertical_line_locus.argtypes = [vp, C.POINTER(abi.LevelDesc), vp, vp, vp, i64, i32,
                                          C.POINTER(abi.Stats)]
    L.vll_vertical_line_locus_device.argtypes = [vp, C.POINTER(abi.LevelDesc), vp, vp, vp, vp, i32,
                                                 C.POINTER(abi.Stats)]
    L.vll_awncc_peaks.argtypes = [vp, C.POINTER(abi.LevelDesc), vp, vp, vp, i64,
                                  C.POINTER(abi.Stats)]
    L.vll_preprocess_level.argtypes = [vp, vp, C.c_uint32, C.c_uint32, i32, vp, vp]
    L.vll_preprocess_level_device.argtypes = [vp, vp, C.c_uint32, C.c_uint32, i32, vp, vp]
    L.vll_pyramid_down.argtypes = [vp, vp, C.c_uint32, C.c_uint32, vp]
    L.vll_pyramid_down_device.argtypes = [vp, vp, C.c_uint32, C.c_uint32, vp]
    L.vll_debug_slot_rho.argtypes = [vp, C.POINTER(abi.LevelDesc), vp, vp, i32, vp, i64, vp]
    L.vll_launch_count.argtypes = [vp]
    L.vll_launch_count.restype = i64
    L.vll_compat_layout.argtypes = [vp, i32]
    L.vll_compat_layout.restype = i32
    L.vll_vertical_line_locus_batch.argtypes = [vp, C.POINTER(abi.LevelIO), i32, vp,
                                                C.POINTER(abi.Stats)]
    L.vll_plan_create.argtypes = [vp, C.POINTER(abi.LevelIO), i32, C.POINTER(vp)]
    L.vll_plan_run.argtypes = [vp, vp, C.POINTER(abi.Stats)]
    L.vll_plan_destroy.argtypes = [vp]
    L.vll_plan_destroy.restype = None
    L.vll_set_tuning.argtypes = [vp, C.POINTER(abi.Tuning)]
    L.vll_get_tuning.argtypes = [vp, C.POINTER(abi.Tuning)]
    D, S = C.POINTER(abi.LevelDesc), C.POINTER(abi.Stats)
    L.vll_vertical_line_locus_seeddem.argtypes = [vp, D, vp, S]
    L.vll_vertical_line_locus_seeddem_device.argtypes = [vp, D, vp, S]
    L.vll_vertical_line_locus_blunder.argtypes = [vp, D, vp, i32, i32, vp, S]
    L.vll_vertical_line_locus_blunder_device.argtypes = [vp, D, vp, i32, i32, vp, S]
    L.vll_vertical_line_locus_ortho.argtypes = [vp, D, C.c_double, vp, vp, vp, vp, i64, vp, vp,
                                                vp]
    L.vll_ortho_blunder.argtypes = [vp, D, C.c_double, vp, i64, vp, i64, vp, vp]
    L.vll_ortho_blunder_device.argtypes = [vp, D, C.c_double, vp, i64, vp, i64, vp, vp]
    L.vll_set_height_range.argtypes = [vp, D, vp, i64, vp, i64, vp, vp, i32, C.c_double, i32,
                                       C.c_double, vp, vp]
    dbl = C.c_double
    L.vll_initialize_voxel.argtypes = [vp, D, vp, vp, vp, vp, i64, C.POINTER(i64)]
    L.vll_initialize_voxel_device.argtypes = [vp, D, vp, vp, vp, vp, i64, vp, C.POINTER(i64)]
    L.vll_awncc_peaks_device.argtypes = [vp, D, vp, vp, vp, vp, S]
    L.vll_select_mps.argtypes = [vp, D, vp, vp, dbl, dbl, dbl, dbl, i32, dbl, i32, dbl, vp, i64,
                                 C.POINTER(i64)]
    L.vll_select_mps_device.argtypes = L.vll_select_mps.argtypes
    L.vll_blunder_detection_tin.argtypes = [vp, D, i32, vp, i32, i32, dbl, vp, vp, i64, vp, i64,
                                            vp, vp, vp, vp]
    L.vll_blunder_detection_tin_device.argtypes = L.vll_blunder_detection_tin.argtypes
    L.vll_tin_rerun_count.argtypes = [vp]
    L.vll_tin_rerun_count.restype = i64
    L.vll_debug_tin_threshold.argtypes = [i32, i32, i32, dbl, dbl, dbl, dbl, i64, i64, vp,
                                          C.c_uint32, i32, C.POINTER(dbl), C.POINTER(dbl)]
    L.vll_set_height_range_device.argtypes = L.vll_set_height_range.argtypes
    L.vll_tin_create.argtypes = [vp, vp, i64, vp, dbl, vp, i64, C.POINTER(i64)]
    L.vll_tin_create_device.argtypes = L.vll_tin_create.argtypes
    L.vll_set_residency.argtypes = [vp, i32]
    L.vll_get_residency.argtypes = [vp]
    L.vll_resident_reset.argtypes = [vp]
    L.vll_resident_voxels.argtypes = [vp, vp, i64, C.POINTER(i64)]
    _lib = L
    return L


def compat_layout() -> list[int]:
    out = np.zeros(128, dtype=np.int64)
    n = load().vll_compat_layout(out.ctypes.data, out.size)
    return out[:n].tolist()


class Context:
    """One GPU context (stream + device buffers) of the matcher."""

    def __init__(self, device: int = 0):
        L = load()
        h = C.c_void_p()
        rc = L.vll_create(int(device), C.byref(h))
        if rc != abi.VLL_OK:
            raise VLLError(rc, L.vll_last_error(None).decode())
        self._h = h
        self.device = int(device)

    @property
    def handle(self):
        return self._h

    def close(self) -> None:
        if self._h:
            load().vll_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int) -> None:
        if rc != abi.VLL_OK:
            raise VLLError(rc, load().vll_last_error(self._h).decode())

    def launch_count(self) -> int:
        return int(load().vll_launch_count(self._h))

    def set_stream(self, stream_ptr: int | None) -> None:
        self._check(load().vll_set_stream(self._h, stream_ptr))

    # ---- the hot path ---------------------------------------------------------
    def vertical_line_locus(self, inputs, nccresult: np.ndarray, voxels: np.ndarray | None = None,
                            kernel: str = "split") -> abi.Stats:
        """VerticalLineLocus on host arrays (nccresult / voxels updated in place)."""
        d = inputs.desc()
        assert nccresult.dtype == abi.NCCRESULT_DTYPE and nccresult.flags.c_contiguous
        st = abi.Stats()
        vptr = voxels.ctypes.data if voxels is not None and voxels.size else None
        cap = voxels.size if voxels is not None else 0
        self._check(load().vll_vertical_line_locus(
            self._h, C.byref(d), inputs.gridpt3.ctypes.data, nccresult.ctypes.data, vptr, cap,
            KERNELS[kernel], C.byref(st)))
        return st

    def vertical_line_locus_device(self, desc: abi.LevelDesc, d_gridpt3: int, d_ncc: int,
                                   d_vox: int | None = None, d_voxoff: int | None = None,
                                   kernel: str = "split", stats: bool = False):
        st = abi.Stats() if stats else None
        self._check(load().vll_vertical_line_locus_device(
            self._h, C.byref(desc), d_gridpt3, d_ncc, d_vox, d_voxoff, KERNELS[kernel],
            C.byref(st) if st is not None else None))
        return st

    DIAG_NAMES = ("cyc_setup", "cyc_coords", "cyc_stage", "cyc_window", "cyc_scan", "cyc_recheck",
                  "cyc_fold", "_", "nodes", "chunks", "slow_lanes", "unstaged_chunks",
                  "plain_nodes", "rounds", "rechecks", "_")

    def debug_slot_rho(self, inputs, nccresult: np.ndarray, kernel: str, diag: dict | None = None) -> tuple:
        """Per-slot rho of `kernel` (FP32 values before re-checks for the split
        kernel); returns (rho, offsets) with NaN for slots not evaluated."""
        k = ((inputs.gridpt3["maxHeight"].astype(np.int64) - inputs.gridpt3["minHeight"])
             / inputs.height_step).astype(np.int64) & 0xFFFF
        off = np.concatenate([[0], np.cumsum(k)]).astype(np.int64)
        out = np.empty(max(int(off[-1]), 1))
        d = inputs.desc()
        dg = np.zeros(16, dtype=np.uint64)
        self._check(load().vll_debug_slot_rho(self._h, C.byref(d), inputs.gridpt3.ctypes.data,
                                              nccresult.ctypes.data, KERNELS[kernel],
                                              out.ctypes.data, out.size, dg.ctypes.data))
        if diag is not None:
            diag.update({n: int(v) for n, v in zip(self.DIAG_NAMES, dg) if n != "_"})
        return out[:off[-1]], off

    def awncc(self, inputs, nccresult: np.ndarray, voxels: np.ndarray | None) -> abi.Stats:
        """AWNCC over the packed voxel rows (setsm_code.cpp:7001-7702): the
        semi-global aggregation when Pyramid_step <= SGM_py, then the peak loop."""
        d = inputs.desc()
        st = abi.Stats()
        vptr = voxels.ctypes.data if voxels is not None and voxels.size else None
        cap = voxels.size if voxels is not None else 0
        self._check(load().vll_awncc_peaks(self._h, C.byref(d), inputs.gridpt3.ctypes.data,
                                           nccresult.ctypes.data, vptr, cap, C.byref(st)))
        return st

    # ---- orthoimage-window variants ------------------------------------------------
    def seeddem(self, inputs, gridpt3: np.ndarray | None = None) -> abi.Stats:
        """VerticalLineLocus_seeddem (setsm_code.cpp:7720-7880): updates
        `gridpt3` (default: inputs.gridpt3) in place."""
        g = inputs.gridpt3 if gridpt3 is None else gridpt3
        d = inputs.desc()
        st = abi.Stats()
        self._check(load().vll_vertical_line_locus_seeddem(self._h, C.byref(d), g.ctypes.data,
                                                           C.byref(st)))
        return st

    def blunder(self, inputs, iteration: int, bblunder: bool,
                gridpt3: np.ndarray | None = None) -> np.ndarray:
        """VerticalLineLocus_blunder (setsm_code.cpp:7882-8026): updates
        `gridpt3` in place and returns the per-node float NCC."""
        g = inputs.gridpt3 if gridpt3 is None else gridpt3
        d = inputs.desc()
        out = np.zeros(len(g), dtype=np.float32)
        self._check(load().vll_vertical_line_locus_blunder(
            self._h, C.byref(d), g.ctypes.data, int(iteration), int(bool(bblunder)),
            out.ctypes.data, None))
        return out

    def seeddem_device(self, desc, d_gridpt3: int) -> None:
        self._check(load().vll_vertical_line_locus_seeddem_device(self._h, C.byref(desc),
                                                                  d_gridpt3, None))

    def blunder_device(self, desc, d_gridpt3: int, iteration: int, bblunder: bool,
                       d_ncc: int) -> None:
        self._check(load().vll_vertical_line_locus_blunder_device(
            self._h, C.byref(desc), d_gridpt3, int(iteration), int(bool(bblunder)), d_ncc, None))

    # ---- TIN orthoimage height search ----------------------------------------------
    def vertical_line_locus_ortho(self, inputs, mpp: float, three: np.ndarray,
                                  target_index: int):
        """VerticalLineLocus_Ortho (setsm_code.cpp:8234-8533) for the triangle
        three = (ref1, ref2, target) (abi.POINT3_DTYPE): returns (selected
        count, F_Height, F_sncc or NaN when unset)."""
        three = np.ascontiguousarray(three, dtype=abi.POINT3_DTYPE)
        d = inputs.desc()
        fh, fs, sc = C.c_double(), C.c_double(float("nan")), C.c_int()
        self._check(load().vll_vertical_line_locus_ortho(
            self._h, C.byref(d), float(mpp), three[0:1].ctypes.data, three[1:2].ctypes.data,
            three[2:3].ctypes.data, inputs.gridpt3.ctypes.data, int(target_index),
            C.byref(fh), C.byref(fs), C.byref(sc)))
        return sc.value, fh.value, fs.value

    def ortho_blunder(self, inputs, mpp: float, pts: np.ndarray, tris: np.ndarray) -> int:
        """Ortho_blunder (setsm_code.cpp:8028-8232): updates pts
        (abi.POINT3_DTYPE), tris' effect and inputs.gridpt3 in place; returns
        the number of rounds run."""
        assert pts.dtype == abi.POINT3_DTYPE and tris.dtype == abi.TRI_DTYPE
        d = inputs.desc()
        rounds = C.c_int()
        self._check(load().vll_ortho_blunder(self._h, C.byref(d), float(mpp), pts.ctypes.data,
                                             len(pts), tris.ctypes.data, len(tris),
                                             inputs.gridpt3.ctypes.data, C.byref(rounds)))
        return rounds.value

    # ---- residency of the host-buffer calls -----------------------------------------
    def set_residency(self, planes: bool = False, voxels: bool = False) -> None:
        """Image planes / grid arrays kept on the device between calls
        (re-sent when their pointer, size or sampled fingerprint changes), and
        the voxel packing kept between InitializeVoxel, VerticalLineLocus and
        AWNCC calls given no voxel array (initialize_voxel_resident)."""
        self._check(load().vll_set_residency(self._h, (abi.VLL_RESIDENT_PLANES if planes else 0)
                                             | (abi.VLL_RESIDENT_VOXELS if voxels else 0)))

    def resident_reset(self) -> None:
        self._check(load().vll_resident_reset(self._h))

    def resident_voxels(self) -> np.ndarray:
        """A host copy of the resident voxel packing."""
        n = C.c_int64(0)
        rc = load().vll_resident_voxels(self._h, None, 0, C.byref(n))
        if rc not in (abi.VLL_OK, abi.VLL_ERR_CAPACITY):
            self._check(rc)
        out = np.zeros(max(n.value, 1), dtype=abi.VOXEL_DTYPE)
        self._check(load().vll_resident_voxels(self._h, out.ctypes.data, out.size, C.byref(n)))
        return out[: n.value]

    def initialize_voxel_resident(self, inputs, ncc: np.ndarray,
                                  voxels_in: np.ndarray | None = None) -> int:
        """InitializeVoxel keeping the new packing on the device (residency
        with voxels on); returns its length."""
        d = inputs.desc()
        n = C.c_int64()
        vin = voxels_in.ctypes.data if voxels_in is not None and voxels_in.size else None
        self._check(load().vll_initialize_voxel(self._h, C.byref(d), inputs.gridpt3.ctypes.data,
                                                ncc.ctypes.data, vin, None, 0, C.byref(n)))
        return n.value

    def initialize_voxel(self, inputs, ncc: np.ndarray,
                         voxels_in: np.ndarray | None = None) -> np.ndarray:
        """InitializeVoxel (setsm_code.cpp:5759-6012): updates inputs.gridpt3
        and ncc in place; returns the voxel rows packed by the new
        NumOfHeight (voxels_in: the rows packed by the incoming one)."""
        d = inputs.desc()
        g = inputs.gridpt3
        cap = int(((g["maxHeight"].astype(np.int64) - g["minHeight"].astype(np.int64) + 4)
                   / inputs.height_step + 4).clip(0).sum())
        cap = max(cap, int(ncc["NumOfHeight"].astype(np.int64).sum()), 1)
        out = np.zeros(cap, dtype=abi.VOXEL_DTYPE)
        n = C.c_int64()
        vin = voxels_in.ctypes.data if voxels_in is not None and voxels_in.size else None
        self._check(load().vll_initialize_voxel(self._h, C.byref(d), g.ctypes.data,
                                                ncc.ctypes.data, vin, out.ctypes.data, cap,
                                                C.byref(n)))
        return out[: n.value].copy()

    def awncc_device(self, desc, d_gridpt3: int, d_ncc: int, d_vox: int, d_offsets: int) -> None:
        """AWNCC on device data (asynchronous on the context's stream)."""
        self._check(load().vll_awncc_peaks_device(self._h, C.byref(desc), d_gridpt3, d_ncc, d_vox,
                                                  d_offsets, None))

    def initialize_voxel_device(self, desc, d_gridpt3: int, d_ncc: int, d_vox_in: int | None,
                                d_vox_out: int, capacity: int, d_offsets: int) -> int:
        n = C.c_int64()
        self._check(load().vll_initialize_voxel_device(self._h, C.byref(desc), d_gridpt3, d_ncc,
                                                       d_vox_in, d_vox_out, int(capacity),
                                                       d_offsets, C.byref(n)))
        return n.value

    def select_mps(self, inputs, ncc: np.ndarray, th_roh: float, th_roh_min: float,
                   th_roh_start: float, th_roh_next: float, iteration: int, mpp: float,
                   final_level_iteration: int, mpp_stereo_angle: float) -> np.ndarray:
        """SelectMPs (setsm_code.cpp:8535-8895): updates inputs.gridpt3 in
        place and returns the matched points (abi.POINT3_DTYPE, node order)."""
        d = inputs.desc()
        out = np.zeros(inputs.n, dtype=abi.POINT3_DTYPE)
        n = C.c_int64()
        self._check(load().vll_select_mps(
            self._h, C.byref(d), ncc.ctypes.data, inputs.gridpt3.ctypes.data, float(th_roh),
            float(th_roh_min), float(th_roh_start), float(th_roh_next), int(iteration),
            float(mpp), int(final_level_iteration), float(mpp_stereo_angle), out.ctypes.data,
            len(out), C.byref(n)))
        return out[: n.value].copy()

    def blunder_detection_tin(self, inputs, iteration: int, ortho_ncc: np.ndarray,
                              flag_blunder: bool, count_bl: int, hinterval: float,
                              pts: np.ndarray, detected: np.ndarray, tris: np.ndarray,
                              counts: np.ndarray, zext: np.ndarray) -> None:
        """blunder_detection_TIN (setsm_code.cpp:9158-9787): pts, detected
        (uint8), inputs.gridpt3, counts (int64[2]) and zext (float64[2]: min,
        max) updated in place."""
        d = inputs.desc()
        self._check(load().vll_blunder_detection_tin(
            self._h, C.byref(d), int(iteration), ortho_ncc.ctypes.data, int(bool(flag_blunder)),
            int(count_bl), float(hinterval), pts.ctypes.data, detected.ctypes.data, len(pts),
            tris.ctypes.data, len(tris), inputs.gridpt3.ctypes.data, counts.ctypes.data,
            zext[0:1].ctypes.data, zext[1:2].ctypes.data))

    def blunder_detection_tin_device(self, desc, iteration: int, d_ortho_ncc: int,
                                     flag_blunder: bool, count_bl: int, hinterval: float,
                                     d_pts: int, d_detected: int, n_pts: int, d_tris: int,
                                     n_tris: int, d_gridpt3: int, counts: np.ndarray,
                                     zext: np.ndarray) -> None:
        """blunder_detection_TIN on device buffers (pointers); counts (int64[2])
        and zext (float64[2]) are host arrays updated in place."""
        self._check(load().vll_blunder_detection_tin_device(
            self._h, C.byref(desc), int(iteration), d_ortho_ncc, int(bool(flag_blunder)),
            int(count_bl), float(hinterval), d_pts, d_detected, int(n_pts), d_tris, int(n_tris),
            d_gridpt3, counts.ctypes.data, zext[0:1].ctypes.data, zext[1:2].ctypes.data))

    def select_mps_device(self, desc, d_ncc: int, d_gridpt3: int, d_points: int, capacity: int,
                          *args) -> int:
        """SelectMPs on device data (desc.grid_pts a device pointer); args as
        select_mps's after ncc.  Returns the number of points."""
        th_roh, th_min, th_start, th_next, it, mpp, fli, angle = args
        n = C.c_int64()
        self._check(load().vll_select_mps_device(
            self._h, C.byref(desc), d_ncc, d_gridpt3, float(th_roh), float(th_min),
            float(th_start), float(th_next), int(it), float(mpp), int(fli), float(angle),
            d_points, int(capacity), C.byref(n)))
        return n.value

    def set_height_range_device(self, desc, d_pts: int, n_pts: int, d_tris: int, n_tris: int,
                                d_gridpt3: int, d_result: int, iteration: int, mpp: float,
                                lcmr: bool, seed_dem_sigma: float = 0.0):
        lo, hi = C.c_double(), C.c_double()
        self._check(load().vll_set_height_range_device(
            self._h, C.byref(desc), d_pts, n_pts, d_tris, n_tris, d_gridpt3, d_result,
            int(iteration), float(mpp), int(bool(lcmr)), float(seed_dem_sigma), C.byref(lo),
            C.byref(hi)))
        return lo.value, hi.value

    def tin_create(self, pts: np.ndarray, min_max, resolution: float) -> np.ndarray:
        """TINCreate_list (SubFunctions.cpp:2768-2846): the ordered triangle list
        (vertex indices into `pts`, POINT3_DTYPE records) of the points
        snapped to the grid of `resolution` cells from min_max[0:2]."""
        pts = np.ascontiguousarray(pts, dtype=abi.POINT3_DTYPE)
        mm = np.ascontiguousarray(min_max, dtype=np.float64)
        cap = 2 * len(pts) + 16
        while True:
            out = np.zeros(cap, dtype=abi.TRI_DTYPE)
            n = C.c_int64(0)
            rc = load().vll_tin_create(self._h, pts.ctypes.data, len(pts), mm.ctypes.data,
                                       float(resolution), out.ctypes.data, cap, C.byref(n))
            if rc == abi.VLL_ERR_CAPACITY and n.value > cap:
                cap = n.value
                continue
            self._check(rc)
            return out[:n.value]

    def tin_create_device(self, d_pts: int, n_pts: int, min_max, resolution: float, d_tris: int,
                          capacity: int) -> int:
        """TINCreate_list on device buffers; returns the number of triangles."""
        mm = np.ascontiguousarray(min_max, dtype=np.float64)
        n = C.c_int64(0)
        self._check(load().vll_tin_create_device(self._h, d_pts, int(n_pts), mm.ctypes.data,
                                                 float(resolution), d_tris, int(capacity),
                                                 C.byref(n)))
        return n.value

    def set_height_range(self, inputs, pts: np.ndarray, tris: np.ndarray, iteration: int,
                         mpp: float, level_check_matching_rate: bool,
                         seed_dem_sigma: float = 0.0):
        """SetHeightRange (setsm_code.cpp:9851-10255): updates inputs.gridpt3
        in place and returns (the new grid, (minH_grid, maxH_grid))."""
        d = inputs.desc()
        out = np.zeros(inputs.n, dtype=abi.UGRID_DTYPE)
        lo, hi = C.c_double(), C.c_double()
        self._check(load().vll_set_height_range(
            self._h, C.byref(d), pts.ctypes.data, len(pts), tris.ctypes.data, len(tris),
            inputs.gridpt3.ctypes.data, out.ctypes.data, int(iteration), float(mpp),
            int(bool(level_check_matching_rate)), float(seed_dem_sigma), C.byref(lo),
            C.byref(hi)))
        return out, (lo.value, hi.value)

    def ortho_blunder_device(self, desc, mpp: float, d_pts: int, n_pts: int, d_tris: int,
                             n_tris: int, d_gridpt3: int) -> int:
        rounds = C.c_int()
        self._check(load().vll_ortho_blunder_device(self._h, C.byref(desc), float(mpp), d_pts,
                                                    n_pts, d_tris, n_tris, d_gridpt3,
                                                    C.byref(rounds)))
        return rounds.value

    # ---- preprocessing -----------------------------------------------------------
    def preprocess(self, image: np.ndarray, template_size: int = 15):
        """Sobel magnitude + orientation images (SetPyramidImages' per-level step)."""
        image = np.ascontiguousarray(image, dtype=np.uint16)
        h, w = image.shape
        mag = np.zeros_like(image)
        ori = np.zeros((h, w), dtype=np.uint8)
        self._check(load().vll_preprocess_level(self._h, image.ctypes.data, w, h, template_size,
                                                mag.ctypes.data, ori.ctypes.data))
        return mag, ori

    def preprocess_device(self, d_image: int, w: int, h: int, d_mag: int, d_ori: int,
                          template_size: int = 15) -> None:
        self._check(load().vll_preprocess_level_device(self._h, d_image, w, h, template_size,
                                                       d_mag, d_ori))

    def pyramid_down(self, image: np.ndarray) -> np.ndarray:
        image = np.ascontiguousarray(image, dtype=np.uint16)
        h, w = image.shape
        out = np.zeros((h // 2, w // 2), dtype=np.uint16)
        self._check(load().vll_pyramid_down(self._h, image.ctypes.data, w, h, out.ctypes.data))
        return out

    def pyramid_down_device(self, d_image: int, w: int, h: int, d_out: int) -> None:
        self._check(load().vll_pyramid_down_device(self._h, d_image, w, h, d_out))

    # ---- batches of levels -------------------------------------------------
    @staticmethod
    def _level_ios(levels) -> tuple:
        """levels: sequence of (desc, d_gridpt3, d_nccresult[, d_voxels, d_voxel_offsets])."""
        n = len(levels)
        arr = (abi.LevelIO * n)()
        keep = []
        for i, lv in enumerate(levels):
            desc = lv[0]
            keep.append(desc)
            arr[i].desc = C.pointer(desc)
            arr[i].d_gridpt3 = lv[1]
            arr[i].d_nccresult = lv[2]
            arr[i].d_voxels = lv[3] if len(lv) > 3 else None
            arr[i].d_voxel_offsets = lv[4] if len(lv) > 4 else None
        return arr, keep

    def batch(self, levels) -> tuple:
        """VerticalLineLocus on every level of `levels` in one pass of the
        split pipeline (one persistent window launch).  Returns (per-level
        Accessable_grid array, Stats)."""
        arr, keep = self._level_ios(levels)
        acc = np.zeros(len(levels), dtype=np.int64)
        st = abi.Stats()
        self._check(load().vll_vertical_line_locus_batch(self._h, arr, len(levels),
                                                         acc.ctypes.data, C.byref(st)))
        del keep
        return acc, st

    def plan(self, levels) -> "Plan":
        """CUDA-graph plan of a batch (see vll_plan_create)."""
        return Plan(self, levels)

    def set_tuning(self, blocks_per_sm: int = 0, grab: int = 8, box_margin: float = 1.1) -> None:
        t = abi.Tuning(int(blocks_per_sm), int(grab), float(box_margin), 0)
        self._check(load().vll_set_tuning(self._h, C.byref(t)))

    def get_tuning(self) -> dict:
        t = abi.Tuning()
        self._check(load().vll_get_tuning(self._h, C.byref(t)))
        return t.as_dict()


class Plan:
    """A batch captured as a CUDA graph; run() replays it on the context's stream."""

    def __init__(self, ctx: Context, levels):
        self.ctx = ctx
        self.n = len(levels)
        arr, self._keep = ctx._level_ios(levels)
        self._arr = arr
        h = C.c_void_p()
        ctx._check(load().vll_plan_create(ctx._h, arr, self.n, C.byref(h)))
        self._h = h

    def run(self, wait: bool = True):
        """Replays the graph; with `wait`, returns (per-level Accessable_grid, Stats)."""
        if not wait:
            self.ctx._check(load().vll_plan_run(self._h, None, None))
            return None
        acc = np.zeros(self.n, dtype=np.int64)
        st = abi.Stats()
        self.ctx._check(load().vll_plan_run(self._h, acc.ctypes.data, C.byref(st)))
        return acc, st

    def close(self) -> None:
        if getattr(self, "_h", None):
            load().vll_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default: Context | None = None


def default_context() -> Context:
    global _default
    if _default is None:
        _default = Context(int(os.environ.get("SETSM_VLL_DEVICE", "0")))
    return _default


def VerticalLineLocus(inputs, nccresult: np.ndarray, voxels: np.ndarray | None = None,
                      kernel: str = "split") -> int:
    """Drop-in for VerticalLineLocus (setsm_code.cpp:6049): returns
    Accessable_grid and updates ``nccresult`` (and the voxel rows) in place."""
    return int(default_context().vertical_line_locus(inputs, nccresult, voxels, kernel).accessable_grid)


def AWNCC(inputs, nccresult: np.ndarray, voxels: np.ndarray) -> None:
    """AWNCC (setsm_code.cpp:7001-7702): SGM aggregation when the level asks
    for it, then the first / second peak selection."""
    default_context().awncc(inputs, nccresult, voxels)
