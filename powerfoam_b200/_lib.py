"""ctypes binding of libpfoam (include/pfoam.h).

The library is the only compute path: if it is missing or fails to load, every
operation raises.  Tensors cross the boundary as raw device pointers; the
current torch stream is passed as the cudaStream_t.
"""

import ctypes
import os

import torch

from . import build as _build

LIB_PATH = _build.LIB_PATH

PF_OK = 0
PF_ERR_OVERFLOW = 1
PF_ERR_STEP_CAP = 2
PF_ERR_ARGS = 3
PF_ERR_CUDA = 4
PF_ERR_SEED = 5
PF_ERR_CELL = 6
PF_ERR_NONFINITE = 7

_ERR_NAMES = {
    PF_ERR_OVERFLOW: "PF_ERR_OVERFLOW",
    PF_ERR_STEP_CAP: "PF_ERR_STEP_CAP",
    PF_ERR_ARGS: "PF_ERR_ARGS",
    PF_ERR_CUDA: "PF_ERR_CUDA",
    PF_ERR_SEED: "PF_ERR_SEED",
    PF_ERR_CELL: "PF_ERR_CELL",
    PF_ERR_NONFINITE: "PF_ERR_NONFINITE",
}

c_f = ctypes.c_float
c_i32 = ctypes.c_int32
c_i64 = ctypes.c_int64
c_vp = ctypes.c_void_p


class PfCamera(ctypes.Structure):
    _fields_ = [("eye", c_f * 3), ("right", c_f * 3), ("up", c_f * 3), ("width", c_i32), ("height", c_i32)]


class PfRasterInputs(ctypes.Structure):
    _fields_ = [
        ("cam", PfCamera),
        ("tile_width", c_i32),
        ("n_sites", c_i32),
        ("n_prims", c_i64),
        ("spheres", c_vp),
        ("nsigmas", c_vp),
        ("texel_sites", c_vp),
        ("texel_rgb", c_vp),
        ("texel_height", c_vp),
        ("attr_half", c_i32),
        ("adjacency", c_vp),
        ("adjacency_offsets", c_vp),
        ("adjacency_diff", c_vp),
        ("tile_offsets", c_vp),
        ("tile_prims", c_vp),
        ("depth_quantiles", c_vp),
        ("n_quantiles", c_i32),
        ("ray_gt", c_vp),
        ("transmittance_threshold", c_f),
        ("tile_order", c_vp),
        ("scratch", c_vp),
        ("ray_maps", c_vp),
        ("segments", c_vp),
        ("segment_masks", c_vp),
        ("segment_offsets", c_vp),
        ("segment_count", c_vp),
        ("segment_pairs", c_i64),
        ("segment_capacity", c_i64),
        ("segment_planes", c_i32),
    ]


class PfTraceInputs(ctypes.Structure):
    _fields_ = [
        ("cam", PfCamera),
        ("n_sites", c_i32),
        ("attr_half", c_i32),
        ("n_prims", c_i64),
        ("spheres", c_vp),
        ("nsigmas", c_vp),
        ("texel_sites", c_vp),
        ("texel_rgb", c_vp),
        ("texel_height", c_vp),
        ("adjacency", c_vp),
        ("adjacency_offsets", c_vp),
        ("adjacency_diff", c_vp),
        ("start_idx", c_i32),
        ("start_cells", c_vp),
        ("transmittance_threshold", c_f),
        ("max_steps", c_i32),
        ("depth_quantile", c_f),
    ]


class PfBatchScene(ctypes.Structure):
    _fields_ = [
        ("n_sites", c_i32),
        ("n_prims", c_i64),
        ("spheres", c_vp),
        ("nsigmas", c_vp),
        ("texel_sites", c_vp),
        ("texel_height", c_vp),
        ("adjacency", c_vp),
        ("adjacency_offsets", c_vp),
        ("adjacency_diff", c_vp),
        ("transmittance_threshold", c_f),
        ("segments", c_vp),
        ("segment_masks", c_vp),
        ("segment_offsets", c_vp),
        ("segment_count", c_vp),
        ("segment_capacity", c_i64),
        ("segment_planes", c_i32),
    ]


class PfBatchView(ctypes.Structure):
    _fields_ = [
        ("cam", PfCamera),
        ("tile_offsets", c_vp),
        ("tile_prims", c_vp),
        ("texel_rgb", c_vp),
        ("target", c_vp),
        ("color", c_vp),
        ("log_t", c_vp),
        ("normal_distance", c_vp),
        ("normal", c_vp),
        ("grad_color", c_vp),
        ("contrib", c_vp),
        ("early_stop", c_vp),
        ("tile_contrib_pairs", c_vp),
        ("grad_texel_rgb", c_vp),
        ("segment_pair_base", c_i64),
        ("segment_pairs", c_i64),
        ("segment_group", c_i32),
    ]


class PfBatchSchedule(ctypes.Structure):
    _fields_ = [("chunk", c_i32), ("order", c_i32), ("split", c_i32), ("ms", c_f)]


PF_BATCH_MAX_VIEWS = 64
PF_BATCH_ORDER_LONGEST = 0
PF_BATCH_ORDER_VIEW = 1

# name -> argtypes (all return int)
_SIGS = {
    "pf_abi_version": [],
    "pf_pack_prims": [c_vp, c_vp, c_vp, c_vp, c_i64, c_vp, c_vp, c_vp, c_vp],
    "pf_bin_workspace_size": [c_i64, c_i64, c_i64, ctypes.POINTER(ctypes.c_size_t)],
    "pf_bin": [ctypes.POINTER(PfCamera), c_i32, c_vp, c_i64, c_vp, ctypes.c_size_t, c_i64, c_vp, c_vp, c_vp, c_vp,
               c_vp, c_vp, c_vp, c_vp],
    "pf_bin_generic_workspace_size": [c_i64, c_i64, c_i32, c_i32, c_i32, c_vp],
    "pf_bin_generic": [ctypes.POINTER(PfCamera), c_vp, c_i32, c_vp, c_i64, c_vp, ctypes.c_size_t, c_i64, c_vp, c_vp,
                       c_vp, c_vp, c_vp, c_vp, c_vp, c_vp],
    "pf_bin_noalloc": [ctypes.POINTER(PfCamera), c_i32, c_vp, c_i64, c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp,
                       c_vp, c_vp],
    "pf_adjacency_prefetch": [c_vp, c_vp, c_vp, c_i64, c_vp, c_vp],
    "pf_adjacency_power_diff": [c_vp, c_vp, c_vp, c_vp, c_i64, c_vp, c_vp],
    "pf_raster_forward": [ctypes.POINTER(PfRasterInputs), c_i32, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp,
                          c_vp, c_vp, c_vp],
    "pf_raster_backward": [ctypes.POINTER(PfRasterInputs), c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp,
                           c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp],
    "pf_raster_benchmark": [ctypes.POINTER(PfRasterInputs), c_vp, c_vp],
    "pf_raster_visualize": [ctypes.POINTER(PfRasterInputs), c_i32, c_f, c_f, c_f, c_f, c_vp, c_vp, c_vp, c_vp, c_vp,
                            c_vp],
    "pf_trace_forward": [ctypes.POINTER(PfTraceInputs), c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_i32, c_vp, c_vp,
                         c_vp],
    "pf_trace_backward_workspace_size": [ctypes.POINTER(PfTraceInputs), c_i32, ctypes.POINTER(ctypes.c_size_t)],
    "pf_trace_backward": [ctypes.POINTER(PfTraceInputs), c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp,
                          c_vp, c_vp, c_vp, c_vp, c_vp, c_i32, c_vp, ctypes.c_size_t, c_vp],
    "pf_trace_forward_record": [ctypes.POINTER(PfTraceInputs), c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_i32,
                                c_vp, ctypes.c_size_t, c_vp],
    "pf_trace_backward_recorded": [ctypes.POINTER(PfTraceInputs), c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp,
                                   c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_i32, c_vp, ctypes.c_size_t, c_vp],
    "pf_start_cell_workspace_size": [c_i64, ctypes.POINTER(ctypes.c_size_t)],
    "pf_start_cell": [c_vp, c_vp, c_i64, ctypes.POINTER(c_f), c_vp, ctypes.c_size_t, c_vp, c_vp],
    "pf_sh_texel_rgb": [c_vp, c_vp, c_i64, c_i32, ctypes.POINTER(c_f), c_vp, c_vp],
    "pf_sh_texel_rgb_backward": [c_vp, c_vp, c_i64, c_i32, ctypes.POINTER(c_f), c_vp, c_vp, c_vp],
    "pf_batch_workspace_size": [ctypes.POINTER(PfBatchView), c_i32, c_i32, ctypes.POINTER(ctypes.c_size_t)],
    "pf_batch_render": [ctypes.POINTER(PfBatchScene), ctypes.POINTER(PfBatchView), c_i32, c_i32, c_i32, c_i32, c_i32,
                        c_vp, ctypes.c_size_t, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp],
    "pf_occupancy_words": [c_i32, ctypes.POINTER(c_i64)],
    "pf_occupancy_build": [c_vp, c_vp, c_vp, c_i64, ctypes.POINTER(c_f), ctypes.POINTER(c_f), c_i32, c_f, c_vp, c_vp,
                           c_vp],
    "pf_occupancy_entry": [c_vp, ctypes.POINTER(c_f), ctypes.POINTER(c_f), c_i32, ctypes.POINTER(PfCamera), c_f, c_vp,
                           c_vp, c_vp],
    "pf_batch_autotune": [ctypes.POINTER(PfBatchScene), ctypes.POINTER(PfBatchView), c_i32, c_i32,
                          ctypes.POINTER(PfBatchSchedule), c_i32, c_i32, c_i32, c_vp, ctypes.c_size_t, c_vp, c_vp,
                          c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.POINTER(c_i32), c_vp],
    "pf_trace_labels": [ctypes.POINTER(PfTraceInputs), c_f, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp],
    "pf_locator_workspace_size": [c_i64, ctypes.POINTER(ctypes.c_size_t)],
    "pf_locator_build": [c_vp, c_vp, c_i64, c_vp, ctypes.c_size_t, c_vp],
    "pf_locate_cells": [c_vp, c_vp, c_i64, c_vp, c_vp, c_i64, c_vp, c_vp, c_vp],
    "pf_seed_start_cells": [c_vp, c_vp, c_i64, c_vp, ctypes.POINTER(PfCamera), c_vp, c_vp, c_f, c_i32, c_vp, c_vp,
                            c_vp],
    "pf_voxel_map_build": [c_vp, c_vp, c_i64, c_vp, ctypes.POINTER(c_f), ctypes.POINTER(c_f), c_i32, c_vp, c_vp,
                           c_vp],
    "pf_seed_start_cells_vmap": [c_vp, c_vp, c_i64, c_vp, c_vp, c_vp, ctypes.POINTER(c_f), ctypes.POINTER(c_f), c_i32,
                                 ctypes.POINTER(PfCamera), c_vp, c_vp, c_f, c_i32, c_i32, c_vp, c_vp, c_vp],
    "pf_locate_cells_vmap": [c_vp, c_vp, c_i64, c_vp, c_vp, c_vp, ctypes.POINTER(c_f), ctypes.POINTER(c_f), c_i32,
                             c_vp, c_i64, c_i32, c_vp, c_vp],
    "pf_mlp_param_count": [],
    "pf_mlp_image_bytes": [],
    "pf_mlp_pack": [c_vp, c_vp, c_vp],
    "pf_mlp_forward": [c_vp, c_vp, c_i64, ctypes.POINTER(PfCamera), c_vp, c_vp, c_vp, c_vp],
    "pf_mlp_train_step": [c_vp, c_vp, c_i64, c_i32, c_vp, ctypes.c_uint32, c_f, c_f, c_vp, c_vp, c_vp, c_vp],
    "pf_mlp_adam": [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_f, c_f, c_f, c_f, c_vp],
    "pf_mlp_gemm_selftest": [c_vp, c_vp, c_i32, c_vp, c_vp, c_vp],
    "pf_cech_workspace_size": [c_i64, ctypes.POINTER(ctypes.c_size_t)],
    "pf_cech_adjacency": [c_vp, c_vp, c_i64, c_vp, ctypes.c_size_t, c_i64, c_vp, c_vp, c_vp, c_vp, c_vp],
    "pf_morton_workspace_size": [c_i64, ctypes.POINTER(ctypes.c_size_t)],
    "pf_morton_sort": [c_vp, c_i64, c_vp, ctypes.c_size_t, c_vp, c_vp],
    "pf_power_workspace_size": [c_i64, c_vp],
    "pf_sv_forward": [c_vp, c_vp, c_vp, ctypes.c_float, c_vp, c_vp, c_vp, c_i64, c_i32, c_i32, c_vp, c_vp, c_vp],
    "pf_sv_backward": [c_vp, c_vp, c_vp, ctypes.c_float, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_i64, c_i32, c_i32,
                       c_vp, c_vp, c_vp, c_vp],
    "pf_steiner_knn": [c_vp, c_vp, c_i64, c_vp, c_vp, c_i64, c_i32, c_vp, c_vp, c_vp, c_vp],
    "pf_steiner_select": [c_vp, c_vp, c_i64, c_i64, ctypes.c_float, c_vp, c_vp, c_vp, c_vp],
    "pf_power_adjacency": [c_vp, c_vp, c_i64, ctypes.c_int32, c_vp, ctypes.c_size_t, c_i64, c_vp, c_vp, c_vp, c_vp,
                           c_vp],
    "pf_interpenetration": [c_vp, c_vp, c_vp, c_i64, c_i64, c_vp, c_vp, c_vp],
    "pf_interpenetration_backward": [c_vp, c_vp, c_vp, c_i64, c_i64, c_vp, c_vp, c_vp, c_vp],
}

_lib = None


def load(build_if_missing=True):
    """Load libpfoam.so (building it first when the toolchain is here)."""
    global _lib
    if _lib is not None:
        return _lib
    if build_if_missing and _build.needs_build():
        try:
            _build.build()
        except Exception as e:  # noqa: BLE001
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(f"libpfoam.so is missing and could not be built: {e}") from e
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libpfoam.so not found at {LIB_PATH}; run python -m powerfoam_b200.build")
    lib = ctypes.CDLL(LIB_PATH)
    for name, args in _SIGS.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = ctypes.c_int
    lib.pf_last_error.restype = ctypes.c_char_p
    lib.pf_last_error.argtypes = []
    _lib = lib
    return lib


def exported_symbols():
    return sorted(_SIGS) + ["pf_last_error"]


class PfError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{_ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


def check(rc):
    if rc != PF_OK:
        raise PfError(rc, load().pf_last_error().decode())


def call(name, *args):
    check(getattr(load(), name)(*args))


def ptr(t):
    """Device pointer of a tensor (None -> NULL)."""
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("Only CUDA tensors are supported as inputs")
    return t.data_ptr()


def stream_ptr():
    return torch.cuda.current_stream().cuda_stream


def make_camera(eye, right, up, width, height):
    c = PfCamera()
    e, r, u = (torch.as_tensor(v).detach().float().cpu().tolist() for v in (eye, right, up))
    for i in range(3):
        c.eye[i] = e[i]
        c.right[i] = r[i]
        c.up[i] = u[i]
    c.width = int(width)
    c.height = int(height)
    return c
