"""ctypes declaration of the C ABI in include/sgs_b200.h and the loader of libsgs_b200.so.

The library is required: importing this module raises if it is missing or was built for another
ABI version. There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

LIB_NAME = "libsgs_b200.so"
ABI_VERSION = 4

SGS_OK = 0
SGS_ERROR_INVALID_ARGUMENT = -1
SGS_ERROR_WORKSPACE = -2
SGS_ERROR_CUDA = -3


class Gaussians(ctypes.Structure):
    _fields_ = [
        ("means", ctypes.c_void_p),
        ("scales", ctypes.c_void_p),
        ("rotations", ctypes.c_void_p),
        ("opacities", ctypes.c_void_p),
        ("sh_coefficients", ctypes.c_void_p),
        ("n_gaussians", ctypes.c_uint32),
        ("sh_bases", ctypes.c_uint32),
        ("preactivated", ctypes.c_void_p),
        ("quantized", ctypes.c_void_p),
        ("quantized_chunks", ctypes.c_void_p),
        ("sh_half", ctypes.c_void_p),
    ]


class Camera(ctypes.Structure):
    _fields_ = [
        ("w2c", ctypes.c_void_p),
        ("cam_position", ctypes.c_void_p),
        ("width", ctypes.c_uint32),
        ("height", ctypes.c_uint32),
        ("focal_x", ctypes.c_float),
        ("focal_y", ctypes.c_float),
        ("center_x", ctypes.c_float),
        ("center_y", ctypes.c_float),
        ("near_plane", ctypes.c_float),
        ("far_plane", ctypes.c_float),
    ]


class SettingsC(ctypes.Structure):
    _fields_ = [
        ("proper_antialiasing", ctypes.c_int32),
        ("supersampling_factor", ctypes.c_int32),
        ("use_gps", ctypes.c_int32),
        ("hybrid_scheduling", ctypes.c_int32),
        ("spatial_reuse", ctypes.c_int32),
        ("temporal_mode", ctypes.c_int32),
        ("blue_noise", ctypes.c_void_p),
        ("view_to_previous_view", ctypes.c_void_p),
        ("max_fragments", ctypes.c_uint32),
        ("max_binned", ctypes.c_uint32),
        ("frame_index_device", ctypes.c_void_p),
    ]


class HistoryC(ctypes.Structure):
    _fields_ = [
        ("image", ctypes.c_void_p),
        ("depth", ctypes.c_void_p),
        ("alpha", ctypes.c_void_p),
        ("weight_mass", ctypes.c_void_p),
        ("k_buffer_primitives", ctypes.c_void_p),
        ("k_buffer_occlusion", ctypes.c_void_p),
    ]


class Outputs(ctypes.Structure):
    _fields_ = [
        ("image", ctypes.c_void_p),
        ("depth", ctypes.c_void_p),
        ("alpha", ctypes.c_void_p),
        ("weight_mass", ctypes.c_void_p),
    ]


class WorkspaceLayout(ctypes.Structure):
    _fields_ = [
        ("framebuffer", ctypes.c_size_t),
        ("samples", ctypes.c_size_t),
        ("reuse_weights", ctypes.c_size_t),
        ("queue", ctypes.c_size_t),
        ("total", ctypes.c_size_t),
    ]


class Conv3x3Args(ctypes.Structure):
    _fields_ = [
        ("input", ctypes.c_void_p),
        ("output", ctypes.c_void_p),
        ("weights", ctypes.c_void_p),
        ("bias", ctypes.c_void_p),
        ("mask", ctypes.c_void_p),
        ("residual", ctypes.c_void_p),
        ("batch", ctypes.c_int32),
        ("height", ctypes.c_int32),
        ("width", ctypes.c_int32),
        ("in_channels", ctypes.c_int32),
        ("out_channels", ctypes.c_int32),
        ("epilogue", ctypes.c_int32),
    ]


SGS_CONV_RELU = 0
SGS_CONV_FINAL = 1
SGS_CONV_MASK = 2

# every entry point of include/sgs_b200.h: name -> (restype, argtypes)
SIGNATURES = {
    "sgs_quantized_chunks": (ctypes.c_uint32, [ctypes.c_uint32]),
    "sgs_quantize": (ctypes.c_int, [ctypes.POINTER(Gaussians), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_void_p]),
    "sgs_composite": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_void_p]),
    "sgs_workspace_size": (ctypes.c_size_t, [ctypes.POINTER(Gaussians), ctypes.POINTER(Camera), ctypes.POINTER(SettingsC)]),
    "sgs_get_workspace_layout": (ctypes.c_int, [ctypes.POINTER(Gaussians), ctypes.POINTER(Camera),
                                                ctypes.POINTER(SettingsC), ctypes.POINTER(WorkspaceLayout)]),
    "sgs_render": (ctypes.c_int, [ctypes.POINTER(Gaussians), ctypes.POINTER(Camera), ctypes.POINTER(SettingsC),
                                  ctypes.POINTER(HistoryC), ctypes.POINTER(Outputs), ctypes.c_void_p, ctypes.c_size_t,
                                  ctypes.c_void_p]),
    "sgs_render_split": (ctypes.c_int, [ctypes.POINTER(Gaussians), ctypes.POINTER(Camera), ctypes.POINTER(SettingsC),
                                        ctypes.POINTER(HistoryC), ctypes.POINTER(Outputs), ctypes.c_void_p,
                                        ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p]),
    "sgs_samples_workspace_size": (ctypes.c_size_t, [ctypes.POINTER(Gaussians), ctypes.POINTER(Camera),
                                                   ctypes.POINTER(SettingsC), ctypes.c_uint32]),
    "sgs_render_samples": (ctypes.c_int, [ctypes.POINTER(Gaussians), ctypes.POINTER(Camera), ctypes.POINTER(SettingsC),
                                          ctypes.POINTER(HistoryC), ctypes.POINTER(Outputs), ctypes.c_uint32,
                                          ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]),
    "sgs_render_no_alloc": (ctypes.c_int, [ctypes.POINTER(Gaussians), ctypes.POINTER(Camera),
                                           ctypes.POINTER(SettingsC), ctypes.POINTER(HistoryC),
                                           ctypes.POINTER(Outputs), ctypes.c_void_p]),
    "sgs_backward_workspace_size": (ctypes.c_size_t, [ctypes.c_uint32]),
    "sgs_backward_accumulate": (ctypes.c_int, [ctypes.POINTER(Gaussians), ctypes.POINTER(Camera),
                                               ctypes.POINTER(SettingsC), ctypes.c_void_p, ctypes.c_void_p,
                                               ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float, ctypes.c_int,
                                               ctypes.c_void_p, ctypes.c_void_p]),
    "sgs_backward_finish": (ctypes.c_int, [ctypes.POINTER(Gaussians), ctypes.POINTER(Camera),
                                           ctypes.POINTER(SettingsC), ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_void_p]),
    "sgs_backward_samples_scratch_size": (ctypes.c_size_t, [ctypes.POINTER(Camera), ctypes.POINTER(SettingsC),
                                                          ctypes.c_uint32]),
    "sgs_backward_sample_terms": (ctypes.c_int, [ctypes.POINTER(Gaussians), ctypes.POINTER(Camera),
                                                 ctypes.POINTER(SettingsC), ctypes.c_void_p, ctypes.c_void_p,
                                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float, ctypes.c_uint32,
                                                 ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p]),
    "sgs_backward_accumulate_samples": (ctypes.c_int, [ctypes.POINTER(Gaussians), ctypes.POINTER(Camera),
                                                       ctypes.POINTER(SettingsC), ctypes.c_void_p, ctypes.c_void_p,
                                                       ctypes.c_void_p, ctypes.c_float, ctypes.c_uint32, ctypes.c_int,
                                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "sgs_backward_accumulate_framebuffers": (ctypes.c_int, [ctypes.POINTER(Gaussians), ctypes.POINTER(Camera),
                                                            ctypes.POINTER(SettingsC), ctypes.c_void_p, ctypes.c_uint32,
                                                            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                            ctypes.c_float, ctypes.c_int, ctypes.c_void_p,
                                                            ctypes.c_void_p, ctypes.c_void_p]),
    "sgs_gps_count_law_size": (ctypes.c_size_t, []),
    "sgs_gps_count_law": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "sgs_conv3x3_weights_size": (ctypes.c_size_t, [ctypes.c_int32, ctypes.c_int32]),
    "sgs_conv3x3": (ctypes.c_int, [ctypes.POINTER(Conv3x3Args), ctypes.c_void_p]),
    "sgs_conv3x3_wgrad": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32,
                                         ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_void_p]),
    "sgs_denoise_features_accumulate": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                                       ctypes.c_int32, ctypes.c_void_p]),
    "sgs_denoise_features_finalize": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32,
                                                     ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p]),
    "sgs_denoise_weights_size": (ctypes.c_size_t, []),
    "sgs_denoise_scratch_size": (ctypes.c_size_t, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
    "sgs_denoise": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                                   ctypes.c_void_p]),
    "sgs_denoise_status": (ctypes.c_int, [ctypes.c_void_p]),
    "sgs_set_stage_events": (None, [ctypes.c_void_p, ctypes.c_void_p]),
    "sgs_set_queue_limit": (None, [ctypes.c_uint32]),
    "sgs_preactivate": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "sgs_probe_atomic_min": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32,
                                             ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p]),
    "sgs_get_frame_index": (ctypes.c_uint32, []),
    "sgs_set_frame_index": (None, [ctypes.c_uint32]),
    "sgs_k_buffer_size": (ctypes.c_uint32, []),
    "sgs_abi_version": (ctypes.c_int, []),
    "sgs_last_error": (ctypes.c_char_p, []),
}


def library_path() -> Path:
    return Path(__file__).resolve().parent / LIB_NAME


_lib = None


def load() -> ctypes.CDLL:
    """Loads the library once and declares every entry point; raises when it is unusable."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not path.is_file():
        raise ImportError(f"{path} is missing: build it with `python stochastic-gaussian-splatting_b200/sgs_build.py`")
    lib = ctypes.CDLL(str(path))
    for name, (restype, argtypes) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    version = lib.sgs_abi_version()
    if version != ABI_VERSION:
        raise ImportError(f"{path} has ABI version {version}, expected {ABI_VERSION}")
    _lib = lib
    return lib


def last_error(lib: ctypes.CDLL) -> str:
    msg = lib.sgs_last_error()
    return msg.decode() if msg else ""
