"""ctypes mirror of include/setsm_vll.h.

The record types are byte-identical to the reference's ``NCCresult``, ``UGRID``,
``VOXEL`` and ``TransParam`` (Typedefine.hpp:214-293); matching numpy dtypes are
provided so that grids can be built and inspected as structured arrays and
handed to the library without copies.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

VLL_ABI_VERSION = 3
VLL_MAX_IMAGES = 8

VLL_OK = 0
VLL_RESIDENT_PLANES = 1
VLL_RESIDENT_VOXELS = 2
VLL_ERR_INVALID = -1
VLL_ERR_UNSUPPORTED = -2
VLL_ERR_CUDA = -3
VLL_ERR_NOMEM = -4
VLL_ERR_TIMEOUT = -5
VLL_ERR_CAPACITY = -6

VLL_KERNEL_FP64_PLAIN = 0
VLL_KERNEL_SPLIT = 1

STATUS_NAMES = {
    VLL_OK: "VLL_OK",
    VLL_ERR_INVALID: "VLL_ERR_INVALID",
    VLL_ERR_UNSUPPORTED: "VLL_ERR_UNSUPPORTED",
    VLL_ERR_CUDA: "VLL_ERR_CUDA",
    VLL_ERR_NOMEM: "VLL_ERR_NOMEM",
    VLL_ERR_TIMEOUT: "VLL_ERR_TIMEOUT",
    VLL_ERR_CAPACITY: "VLL_ERR_CAPACITY",
}

# ---- record dtypes (identical layout to the reference structs) -------------
NCCRESULT_DTYPE = np.dtype(
    {
        "names": ["result2", "result3", "minHeight", "maxHeight", "result0", "result1",
                  "max_WNCC", "GNCC", "NumOfHeight", "result4", "check_height_change"],
        "formats": ["<f4", "<f4", "<i2", "<i2", "<i2", "<i2", "<i2", "<i2", "<u2", "u1", "u1"],
        "offsets": [0, 4, 8, 10, 12, 14, 16, 18, 20, 22, 23],
        "itemsize": 24,
    }
)

UGRID_DTYPE = np.dtype(
    {
        "names": ["Height", "minHeight", "maxHeight", "roh", "ortho_ncc", "Mean_ortho_ncc",
                  "Matched_flag", "anchor_flag"],
        "formats": ["<f4", "<i2", "<i2", "<i2", ("<i2", (2,)), "<i2", "u1", "u1"],
        "offsets": [0, 4, 6, 8, 10, 14, 16, 17],
        "itemsize": 20,
    }
)

VOXEL_DTYPE = np.dtype(
    {"names": ["flag_cal", "INCC"], "formats": ["u1", "<i2"], "offsets": [0, 2], "itemsize": 4}
)

# vll_point3 (D3DPOINT, 32 B) and vll_tri (UI3DPOINT, 12 B)
POINT3_DTYPE = np.dtype(
    {"names": ["x", "y", "z", "flag"], "formats": ["<f8", "<f8", "<f8", "u1"],
     "offsets": [0, 8, 16, 24], "itemsize": 32}
)
TRI_DTYPE = np.dtype({"names": ["a", "b", "c"], "formats": ["<u4", "<u4", "<u4"],
                      "offsets": [0, 4, 8], "itemsize": 12})


class TransParam(C.Structure):
    _fields_ = [
        ("t_c", C.c_double), ("m_c", C.c_double),
        ("sa", C.c_double), ("sb", C.c_double), ("e2", C.c_double),
        ("e2cuadrada", C.c_double), ("c", C.c_double),
        ("a", C.c_double), ("e", C.c_double),
        ("phi_c", C.c_double), ("lambda_0", C.c_double),
        ("pm", C.c_int32), ("projection", C.c_int32), ("utm_zone", C.c_int32),
        ("direction", C.c_char * 2), ("bHemisphere", C.c_int32),
    ]


class ImageDesc(C.Structure):
    _fields_ = [
        ("image", C.c_void_p), ("mag", C.c_void_p), ("ori", C.c_void_p),
        ("width", C.c_uint32), ("height", C.c_uint32),
        ("startpos", C.c_double * 2),
        ("image_next", C.c_void_p), ("mag_next", C.c_void_p), ("ori_next", C.c_void_p),
        ("width_next", C.c_uint32), ("height_next", C.c_uint32),
        ("startpos_next", C.c_double * 2),
        ("rpc", C.c_double * 90),
        ("image_adjust", C.c_double * 2),
        ("selected", C.c_int32), ("_pad", C.c_int32),
        ("image_b", C.c_void_p), ("mag_b", C.c_void_p),
        ("width_b", C.c_uint32), ("height_b", C.c_uint32),
        ("startpos_b", C.c_double * 2),
    ]


class LevelDesc(C.Structure):
    _fields_ = [
        ("num_images", C.c_int32), ("reference_id", C.c_int32),
        ("pyramid_step", C.c_int32), ("template_size", C.c_int32),
        ("py_combined_level", C.c_int32), ("iteration", C.c_int32),
        ("check_matching_rate", C.c_int32), ("is_ra", C.c_int32),
        ("pre_dem_tif", C.c_int32), ("check_matchtag", C.c_int32),
        ("sgm_py", C.c_int32), ("sensor_type", C.c_int32),
        ("resolution", C.c_double), ("dem_resolution", C.c_double),
        ("height_step", C.c_double), ("grid_resolution", C.c_double),
        ("bin_angle", C.c_double),
        ("boundary", C.c_double * 4),
        ("minmax_height", C.c_double * 2),
        ("grid_width", C.c_int64), ("grid_height", C.c_int64),
        ("grid_pts", C.c_void_p), ("grid_wgs", C.c_void_p),
        ("param", TransParam),
        ("images", ImageDesc * VLL_MAX_IMAGES),
        ("blunder_level", C.c_int32), ("_pad2", C.c_int32),
    ]


class LevelIO(C.Structure):
    """vll_level_io: one level of a batch (device pointers)."""
    _fields_ = [
        ("desc", C.POINTER(LevelDesc)), ("d_gridpt3", C.c_void_p), ("d_nccresult", C.c_void_p),
        ("d_voxels", C.c_void_p), ("d_voxel_offsets", C.c_void_p),
    ]


class Tuning(C.Structure):
    """vll_tuning: launch parameters of the window kernel."""
    _fields_ = [("blocks_per_sm", C.c_int32), ("grab", C.c_int32), ("box_margin", C.c_float),
                ("_pad", C.c_int32)]

    def as_dict(self) -> dict:
        return {"blocks_per_sm": self.blocks_per_sm, "grab": self.grab,
                "box_margin": round(float(self.box_margin), 4)}


class Stats(C.Structure):
    _fields_ = [
        ("accessable_grid", C.c_int64), ("evals", C.c_int64),
        ("fp64_rechecks", C.c_int64), ("kernel_ms", C.c_double),
        ("window_ms", C.c_double), ("slots", C.c_int64), ("launches", C.c_int64),
        ("stage_ms", C.c_double * 8),
        ("exact_nodes", C.c_int64), ("fp64_nodes", C.c_int64), ("scan_rounds", C.c_int64),
    ]

    STAGES = ("gncc", "prep", "prefix", "items", "window", "scan", "exact", "tail")

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "stage_ms"}
        d["stage_ms"] = dict(zip(self.STAGES, list(self.stage_ms)))
        return d


def ptr(a) -> int | None:
    """Address of a numpy array's data (None for None)."""
    if a is None:
        return None
    return a.ctypes.data


def set_transparam(tp: TransParam, p: dict) -> None:
    for k, v in p.items():
        if k == "direction":
            tp.direction = bytes(v)[:2]
        else:
            setattr(tp, k, v)


def transparam_dict(tp: TransParam) -> dict:
    out = {}
    for name, _ in TransParam._fields_:
        out[name] = bytes(tp.direction) if name == "direction" else getattr(tp, name)
    return out
