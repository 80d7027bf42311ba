"""ctypes binding of libturbo_hot.so, the C ABI declared in include/turbo_hot.h.

There is no fallback: if the shared library is missing or cannot be loaded, importing this
module raises. Build it with `python -m turbonerf_b200.csrc.build` (or
`__graft_entry__.build()`).
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libturbo_hot.so")

TN_OK = 0
TN_E_INVALID = -1
TN_E_NULL = -2
TN_E_CAPACITY = -3
TN_E_CUDA = -4
TN_E_NO_RAYS = -5
TN_E_NO_SAMPLES = -6
TN_E_LEVELS = -7
TN_E_DEVICE = -8
TN_E_STATE = -9

TN_FLAG_GUARD = 1
TN_FLAG_CAPACITY = 2
TN_FLAG_NO_RAYS = 4
TN_FLAG_NO_SAMPLES = 8
TN_FLAG_SPIN = 16

TN_ACT_SIGMA = 0
TN_ACT_DENSITY = 1

_STATUS_NAMES = {
    TN_E_INVALID: "TN_E_INVALID", TN_E_NULL: "TN_E_NULL", TN_E_CAPACITY: "TN_E_CAPACITY", TN_E_CUDA: "TN_E_CUDA",
    TN_E_NO_RAYS: "TN_E_NO_RAYS", TN_E_NO_SAMPLES: "TN_E_NO_SAMPLES", TN_E_LEVELS: "TN_E_LEVELS",
    TN_E_DEVICE: "TN_E_DEVICE", TN_E_STATE: "TN_E_STATE",
}


class TurboError(RuntimeError):
    """A turbo_hot call returned a non-zero status."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{_STATUS_NAMES.get(status, status)}: {message}")


class NoRaysError(TurboError):
    """Raised like the reference's "No rays were generated for this training batch!"."""


class NoSamplesError(TurboError):
    """Raised like the reference's "No samples were generated for this training batch!"."""


class Bbox(ctypes.Structure):
    _fields_ = [(n, ctypes.c_float) for n in ("min_x", "min_y", "min_z", "max_x", "max_y", "max_z")]


class GridDesc(ctypes.Structure):
    _fields_ = [("n_levels", ctypes.c_int32), ("resolution", ctypes.c_int32), ("base_size", ctypes.c_float),
                ("reserved", ctypes.c_int32)]


class HashgridDesc(ctypes.Structure):
    _fields_ = [("n_levels", ctypes.c_uint32), ("log2_hashmap_size", ctypes.c_uint32),
                ("base_resolution", ctypes.c_float), ("per_level_scale", ctypes.c_float)]


class MarchDesc(ctypes.Structure):
    _fields_ = [("cone_angle", ctypes.c_float), ("dt_min", ctypes.c_float), ("dt_max", ctypes.c_float),
                ("max_steps", ctypes.c_uint32), ("max_iterations", ctypes.c_uint32)]


class SceneDesc(ctypes.Structure):
    """tn_scene: one scene of a multi-scene launch."""
    _fields_ = [("grid", GridDesc), ("bitfield", ctypes.c_void_p), ("bbox", Bbox), ("march", MarchDesc),
                ("inv_aabb_size", ctypes.c_float), ("ray_begin", ctypes.c_uint32), ("n_rays", ctypes.c_uint32)]


class RayBatchDesc(ctypes.Structure):
    _fields_ = [("n_rays", ctypes.c_uint32), ("ray_stride", ctypes.c_uint32), ("sample_stride", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32), ("counts", ctypes.c_void_p), ("offsets", ctypes.c_void_p),
                ("n_rays_dev", ctypes.c_void_p)]


class Tuning(ctypes.Structure):
    """tn_tuning: launch shapes of the tunable kernels."""
    _fields_ = [("count_rays_per_block", ctypes.c_uint32), ("emit_warps_per_block", ctypes.c_uint32),
                ("emit_rays_per_warp", ctypes.c_uint32), ("loss_rays_per_block", ctypes.c_uint32),
                ("compact_tile", ctypes.c_uint32), ("multi_chunk_rays", ctypes.c_uint32),
                ("side_sms", ctypes.c_uint32)]

    def as_dict(self):
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


class TuneReport(ctypes.Structure):
    """tn_tune_report: candidates tried, median ms before and with the chosen shape."""
    _fields_ = [("n_candidates", ctypes.c_uint32), ("before_ms", ctypes.c_float), ("best_ms", ctypes.c_float)]

    def as_dict(self):
        return {"n_candidates": int(self.n_candidates), "before_ms": float(self.before_ms),
                "best_ms": float(self.best_ms)}


TN_PATH_FUSED = 0
TN_PATH_PLAIN = 1


class TrainerDesc(ctypes.Structure):
    _fields_ = [("grid", GridDesc), ("bbox", Bbox), ("batch_size", ctypes.c_uint32),
                ("n_rays_per_step", ctypes.c_uint32), ("min_step_size", ctypes.c_float),
                ("cone_angle", ctypes.c_float), ("max_steps_per_ray", ctypes.c_uint32),
                ("min_transmittance", ctypes.c_float), ("use_distortion_loss", ctypes.c_int32),
                ("distortion_lambda", ctypes.c_float), ("loss_scale", ctypes.c_float),
                ("occupancy_decay", ctypes.c_float), ("occupancy_threshold", ctypes.c_float),
                ("occupancy_cells_per_step", ctypes.c_uint32), ("n_grid_params", ctypes.c_uint32),
                ("n_mlp_params", ctypes.c_uint32), ("learning_rate", ctypes.c_float),
                ("learning_rate_decay", ctypes.c_float), ("beta1", ctypes.c_float), ("beta2", ctypes.c_float),
                ("epsilon", ctypes.c_float), ("l2_reg", ctypes.c_float), ("path", ctypes.c_int32),
                ("use_cuda_graph", ctypes.c_int32), ("seed", ctypes.c_uint32), ("ray_radius", ctypes.c_float),
                ("ray_jitter", ctypes.c_float)]


class TurboInfoC(ctypes.Structure):
    """tn_turbo_info: a .turbo file's header and resume block."""
    _fields_ = [("n_params", ctypes.c_uint64), ("file_bytes", ctypes.c_uint64), ("n_occ_grid_bits", ctypes.c_uint32),
                ("aabb_scale", ctypes.c_uint32), ("has_resume", ctypes.c_uint32), ("step_count", ctypes.c_uint32),
                ("n_levels", ctypes.c_uint32), ("resolution", ctypes.c_uint32), ("dataset_path", ctypes.c_char * 256)]


class CameraC(ctypes.Structure):
    """tn_camera: pinhole camera, transform = camera to world, row-major 3 x 4 [R | t]."""
    _fields_ = [("width", ctypes.c_int32), ("height", ctypes.c_int32), ("near", ctypes.c_float),
                ("far", ctypes.c_float), ("focal_x", ctypes.c_float), ("focal_y", ctypes.c_float),
                ("principal_x", ctypes.c_float), ("principal_y", ctypes.c_float), ("shift_x", ctypes.c_float),
                ("shift_y", ctypes.c_float), ("transform", ctypes.c_float * 12)]


class RenderDescC(ctypes.Structure):
    _fields_ = [("grid", GridDesc), ("bitfield", ctypes.c_void_p), ("render_bbox", Bbox),
                ("training_bbox", Bbox), ("dt_min", ctypes.c_float), ("cone_angle", ctypes.c_float),
                ("min_transmittance", ctypes.c_float), ("batch_size", ctypes.c_uint32)]


class RenderStatsC(ctypes.Structure):
    _fields_ = [("rays_hit", ctypes.c_uint32), ("iterations", ctypes.c_uint32), ("samples", ctypes.c_uint64),
                ("steps", ctypes.c_uint64), ("tests", ctypes.c_uint64)]


class TrainingMetricsC(ctypes.Structure):
    _fields_ = [("step", ctypes.c_uint32), ("n_rays", ctypes.c_uint32), ("n_samples", ctypes.c_uint32),
                ("loss", ctypes.c_float)]


class OccupancyMetricsC(ctypes.Structure):
    _fields_ = [("n_occupied", ctypes.c_uint32), ("n_total", ctypes.c_uint32)]


_vp = ctypes.c_void_p
_u32 = ctypes.c_uint32
_u64 = ctypes.c_uint64
_i32 = ctypes.c_int
_f32 = ctypes.c_float
_P = ctypes.POINTER

# name -> argtypes (all return int status unless listed in _RESTYPE)
SIGNATURES = {
    "tn_version": [],
    "tn_last_error": [],
    "tn_ctx_create": [_P(_vp)],
    "tn_ctx_destroy": [_vp],
    "tn_ctx_reserve": [_vp, _u32, _u32],
    "tn_ctx_check": [_vp, _vp, _P(_u32)],
    "tn_ctx_flags_ptr": [_vp, _P(_vp)],
    "tn_tuning_default": [_P(Tuning)],
    "tn_tuning_validate": [_P(Tuning)],
    "tn_ctx_set_tuning": [_vp, _P(Tuning)],
    "tn_ctx_get_tuning": [_vp, _P(Tuning)],
    "tn_autotune_march": [_vp, _vp, _P(GridDesc), _vp, _P(Bbox), _P(MarchDesc), _f32, _u32, _u32, _vp, _vp, _vp,
                          _vp, _vp, _vp, _vp, _u32, _vp, _u32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                          _P(TuneReport), _P(TuneReport)],
    "tn_autotune_multi": [_vp, _vp, _u32, _vp, _u32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _u32, _vp, _vp,
                          _vp, _vp, _vp, _vp, _vp, _vp, _P(TuneReport), _P(TuneReport)],
    "tn_autotune_losses": [_vp, _vp, _P(RayBatchDesc), _i32, _f32, _f32, _vp, _f32, _f32, _vp, _vp, _vp, _vp, _vp,
                           _vp, _vp, _vp, _vp, _vp, _vp, _vp, _P(TuneReport)],
    "tn_autotune_compact": [_vp, _vp, _u32, _vp, _vp, _vp, _P(TuneReport)],
    "tn_trainer_autotune": [_vp, _P(TuneReport)],
    "tn_trainer_get_tuning": [_vp, _P(Tuning)],
    "tn_trainer_flush": [_vp],
    "tn_trainer_reset": [_vp],
    "tn_trainer_set_tuning": [_vp, _P(Tuning)],
    "tn_rays_init_bbox": [_vp, _u32, _u32, _P(Bbox), _f32, _vp, _vp, _vp, _vp, _vp],
    "tn_march_count": [_vp, _vp, _P(GridDesc), _vp, _P(Bbox), _P(MarchDesc), _u32, _u32, _vp, _vp, _vp, _vp, _vp,
                       _vp, _vp, _u32, _vp],
    "tn_march_emit": [_vp, _vp, _P(GridDesc), _vp, _P(Bbox), _P(MarchDesc), _f32, _u32, _u32, _u32, _vp, _vp, _vp,
                      _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "tn_scan_offsets": [_vp, _vp, _u32, _vp, _vp, _u32, _vp],
    "tn_multi_march_count": [_vp, _vp, _u32, _vp, _u32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "tn_multi_march_emit": [_vp, _vp, _u32, _vp, _u32, _u32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                            _vp, _vp, _vp],
    "tn_scan_offsets_noalloc": [_vp, _u32, _vp, _vp, _u32, _vp, _vp],
    "tn_compact_nonzero": [_vp, _vp, _u32, _vp, _vp, _vp],
    "tn_composite_fwd": [_vp, _vp, _P(RayBatchDesc), _i32, _f32, _vp, _vp, _vp, _vp, _vp, _vp],
    "tn_composite_bwd": [_vp, _vp, _P(RayBatchDesc), _i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "tn_composite_fwd_store": [_vp, _vp, _P(RayBatchDesc), _i32, _f32, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "tn_composite_bwd_stored": [_vp, _vp, _P(RayBatchDesc), _i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "tn_recon_loss_fwd_bwd": [_vp, _vp, _P(RayBatchDesc), _i32, _f32, _f32, _f32, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                              _vp, _vp, _vp],
    "tn_distortion_fwd_bwd": [_vp, _vp, _P(RayBatchDesc), _i32, _f32, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "tn_grad_epilogue": [_vp, _u32, _vp, _f32, _vp, _vp, _vp, _vp],
    "tn_train_losses": [_vp, _vp, _P(RayBatchDesc), _i32, _f32, _f32, _vp, _f32, _f32, _vp, _vp, _vp, _vp, _vp, _vp,
                        _vp, _vp, _vp, _vp, _vp, _vp],
    "tn_occupancy_sample_points": [_vp, _P(GridDesc), _u32, _vp, _vp, _vp, _u32, _f32, _vp, _u32],
    "tn_occupancy_update": [_vp, _vp, _P(GridDesc), _vp, _vp, _u32, _vp, _vp, _vp, _vp, _i32, _i32, _f32, _f32, _vp],
    "tn_popcount": [_vp, _vp, _u64, _vp, _vp],
    "tn_adam_step": [_vp, _u32, _u32, _u32, _f32, _f32, _f32, _f32, _f32, _f32, _vp, _vp, _vp, _vp, _vp, _vp],
    "tn_plain_march_count": [_vp, _P(GridDesc), _vp, _P(Bbox), _P(MarchDesc), _u32, _u32, _vp, _vp, _vp, _vp, _vp,
                             _vp],
    "tn_plain_scan_cut_sync": [_vp, _u32, _vp, _vp, _u32, _P(_u32), _P(_u32)],
    "tn_plain_march_emit": [_vp, _P(GridDesc), _vp, _P(Bbox), _P(MarchDesc), _f32, _u32, _u32, _u32, _vp, _vp, _vp,
                            _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "tn_plain_recon_loss_sync": [_vp, _P(RayBatchDesc), _i32, _f32, _f32, _f32, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                 _vp, _P(_f32)],
    "tn_plain_distortion_sync": [_vp, _P(RayBatchDesc), _i32, _f32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _P(_f32)],
    "tn_plain_grad_epilogue": [_vp, _u32, _f32, _vp, _vp, _vp, _vp],
    "tn_plain_occupancy_update_sync": [_vp, _P(GridDesc), _vp, _vp, _u32, _vp, _vp, _vp, _vp, _i32, _i32, _f32, _f32,
                                       _vp, _P(_u32)],
    "tn_plain_adam_step": [_vp, _u32, _u32, _u32, _f32, _f32, _f32, _f32, _f32, _f32, _vp, _vp, _vp, _vp, _vp, _vp],
    "tn_synth_field": [_vp, _u32, _vp, _u32, _vp, _f32, _u32, _vp, _vp, _vp, _vp, _u32],
    "tn_render": [_vp, _vp, _P(RenderDescC), _P(CameraC), _vp, _vp, _P(RenderStatsC)],
    "tn_trainer_render": [_vp, _P(CameraC), _P(Bbox), _f32, _u32, _vp, _P(RenderStatsC)],
    "tn_dataset_rays": [_vp, _u32, _u32, _u32, _i32, _i32, _vp, _vp, _P(Bbox), _vp, _f32, _f32, _vp, _vp, _vp, _vp,
                        _vp, _vp, _vp],
    "tn_trainer_set_dataset": [_vp, _u32, _i32, _i32, _vp, _vp],
    "tn_trainer_set_alpha_selection": [_vp, _f32, _f32],
    "tn_trainer_save": [_vp, ctypes.c_char_p, ctypes.c_char_p],
    "tn_trainer_load": [_vp, ctypes.c_char_p],
    "tn_turbo_file_info": [ctypes.c_char_p, _P(TurboInfoC)],
    "tn_trainer_default_desc": [_vp],
    "tn_trainer_create": [_P(_vp), _vp, _vp],
    "tn_trainer_destroy": [_vp],
    "tn_trainer_set_synthetic_field": [_vp, _u32, _vp, _vp],
    "tn_trainer_set_grid": [_vp, _vp, _vp],
    "tn_trainer_init_synthetic_gradients": [_vp, _f32, _P(_u32)],
    "tn_trainer_use_hashgrid": [_vp, _vp],
    "tn_hashgrid_n_params": [_vp, _P(_u64), _P(_u32)],
    "tn_hashgrid_level_resolution": [_vp, _u32, _P(_u32), _P(_i32)],
    "tn_hashgrid_encode": [_vp, _vp, _u32, _vp, _u32, _vp, _vp, _vp],
    "tn_hashgrid_backward": [_vp, _vp, _u32, _vp, _u32, _vp, _vp, _vp, _vp, _vp, _vp],
    "tn_hashgrid_clear_touched": [_vp, _vp, _vp, _u32, _vp, _vp],
    "tn_trainer_train_step": [_vp, _vp],
    "tn_trainer_train_step_rays": [_vp, _u32, _vp, _vp, _vp, _vp, _vp],
    "tn_trainer_train_step_rays_pipelined": [_vp, _u32, _vp, _vp, _vp, _vp, _vp],
    "tn_trainer_profile_step": [_vp, _vp, _u32, _P(_u32)],
    "tn_trainer_stat": [_vp, _i32, _P(_u64)],
    "tn_trainer_update_occupancy_grid": [_vp, _u32, _vp],
    "tn_trainer_sync_metrics": [_vp, _vp],
    "tn_trainer_stream": [_vp, _P(_vp)],
    "tn_trainer_buffer": [_vp, _i32, _P(_vp), _P(_u64)],
}
_RESTYPE = {"tn_last_error": ctypes.c_char_p, "tn_tuning_default": None}

_lib = None


def lib() -> ctypes.CDLL:
    """The loaded library (raises if it is missing: there is no CPU or eager fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m turbonerf_b200.csrc.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = _RESTYPE.get(name, ctypes.c_int)
        _lib = L
    return _lib


def last_error() -> str:
    msg = lib().tn_last_error()
    return msg.decode() if msg else ""


def check(status: int) -> None:
    if status == TN_OK:
        return
    msg = last_error()
    if status == TN_E_NO_RAYS:
        raise NoRaysError(status, msg)
    if status == TN_E_NO_SAMPLES:
        raise NoSamplesError(status, msg)
    raise TurboError(status, msg)


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args))
