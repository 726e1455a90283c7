"""ctypes binding of libacoustic_rt.so (include/acoustic_rt.h).

Loading fails loudly: if the shared library is missing or does not export
the ABI, importing the backend raises instead of falling back to any CPU
path.  Host-only entry points (``ac_bvh_build``, ``ac_last_error``) work on a
machine without a GPU.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path
from typing import Any

import numpy as np

PACKAGE_DIR = Path(__file__).resolve().parent
LIBRARY_PATH = PACKAGE_DIR / "libacoustic_rt.so"

AC_OK = 0
AC_ERR_INVALID = -1
AC_ERR_CUDA = -2
AC_ERR_NOMEM = -3
AC_ERR_UNSUPPORTED = -4
AC_ERR_CAPACITY = -5
AC_PRECISION_FP32 = 0
AC_PRECISION_FP64 = 1
AC_RNG_REFERENCE = 0
AC_RNG_PHILOX = 1
AC_BVH_STATUS_NONFINITE = 1
AC_BVH_STATUS_ORDER = 2
AC_BVH_STATUS_TIMEOUT = 4
AC_BVH_STATUS_INTERNAL = 8
AC_SYNTH_STATIC_BYTES = 16 << 20

c_double_p = ctypes.POINTER(ctypes.c_double)
c_int64_p = ctypes.POINTER(ctypes.c_int64)
c_int32_p = ctypes.POINTER(ctypes.c_int32)
c_float_p = ctypes.POINTER(ctypes.c_float)


class ACBvh(ctypes.Structure):
    _fields_ = [
        ("bounds_min", c_double_p), ("bounds_max", c_double_p), ("start", c_int64_p), ("count", c_int64_p),
        ("escape", c_int64_p), ("primitives", c_int64_p), ("node_count", ctypes.c_int64),
        ("leaf_count", ctypes.c_int64), ("max_depth", ctypes.c_int64),
    ]


class ACSceneDesc(ctypes.Structure):
    _fields_ = [
        ("num_surfaces", ctypes.c_int64), ("kinds", c_int64_p), ("wall_a", c_double_p), ("wall_delta", c_double_p),
        ("wall_z", c_double_p), ("z_values", c_double_p), ("box_center", c_double_p), ("box_axis_u", c_double_p),
        ("box_axis_v", c_double_p), ("box_half", c_double_p), ("box_z", c_double_p), ("normals", c_double_p),
        ("reflection", c_double_p), ("scattering", c_double_p), ("num_corners", ctypes.c_int64),
        ("corners", c_double_p), ("surface_bounds_min", c_double_p), ("surface_bounds_max", c_double_p),
        ("bvh_node_count", ctypes.c_int64), ("bvh_bounds_min", c_double_p), ("bvh_bounds_max", c_double_p),
        ("bvh_start", c_int64_p), ("bvh_count", c_int64_p), ("bvh_escape", c_int64_p),
        ("bvh_primitives", c_int64_p), ("device", ctypes.c_int32), ("cluster_size", ctypes.c_int32),
        ("traversal", ctypes.c_int32), ("bvh_leaf", ctypes.c_int32), ("bvh_width", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class ACSceneInfo(ctypes.Structure):
    _fields_ = [
        ("num_surfaces", ctypes.c_int64), ("num_corners", ctypes.c_int64), ("node_count", ctypes.c_int64),
        ("leaf_count", ctypes.c_int64), ("device_bytes", ctypes.c_int64), ("device", ctypes.c_int32),
        ("max_leaf", ctypes.c_int32), ("num_clusters", ctypes.c_int64), ("traversal", ctypes.c_int32),
        ("bvh_depth", ctypes.c_int32), ("bvh_nodes", ctypes.c_int64), ("bvh_width", ctypes.c_int32),
        ("bvh_stack_need", ctypes.c_int32),
    ]


class ACTraceParams(ctypes.Structure):
    _fields_ = [
        ("source", ctypes.c_double * 3), ("listener", ctypes.c_double * 3), ("source_forward", ctypes.c_double * 3),
        ("num_rays", ctypes.c_int64), ("num_bounces", ctypes.c_int32), ("num_bins", ctypes.c_int32),
        ("bin_duration", ctypes.c_double), ("speed_of_sound", ctypes.c_double),
        ("max_path_length", ctypes.c_double), ("direct_delay", ctypes.c_double),
        ("listener_radius", ctypes.c_double), ("source_radius", ctypes.c_double),
        ("irradiance_min_distance", ctypes.c_double), ("specular_exponent", ctypes.c_double),
        ("dipole_weight", ctypes.c_double), ("dipole_power", ctypes.c_double),
        ("use_bvh", ctypes.c_int32), ("render_ambisonics", ctypes.c_int32), ("precision", ctypes.c_int32),
        ("rng_mode", ctypes.c_int32), ("seed", ctypes.c_uint64), ("stream_key", ctypes.c_uint64),
        ("directions", ctypes.c_void_p), ("diffuse_random", ctypes.c_void_p), ("diffuse_indices", ctypes.c_void_p),
        ("diffuse_bank", ctypes.c_void_p), ("num_bank", ctypes.c_int32), ("block_size", ctypes.c_int32),
        ("energy_scale", ctypes.c_double), ("grid_blocks", ctypes.c_int32), ("visual_limit", ctypes.c_int32),
        ("visual_stride", ctypes.c_int32), ("stack_entries", ctypes.c_int32),
    ]


class ACTraceOutputs(ctypes.Structure):
    _fields_ = [
        ("echogram_fx", ctypes.c_void_p), ("ambisonic_fx", ctypes.c_void_p), ("hit_counts", ctypes.c_void_p),
        ("contrib_counts", ctypes.c_void_p), ("surface_energy_fx", ctypes.c_void_p), ("counters", ctypes.c_void_p),
        ("echogram", ctypes.c_void_p), ("ambisonic", ctypes.c_void_p), ("surface_energy", ctypes.c_void_p),
        ("ray_surfaces", ctypes.c_void_p), ("scale_out", c_double_p),
        ("visual_hit_points", ctypes.c_void_p), ("visual_surfaces", ctypes.c_void_p),
        ("visual_rays", ctypes.c_void_p), ("visual_orders", ctypes.c_void_p),
        ("visual_distances", ctypes.c_void_p), ("visual_gains", ctypes.c_void_p),
    ]


class ACJob(ctypes.Structure):
    _fields_ = [("scene", ctypes.c_void_p), ("params", ACTraceParams), ("outputs", ACTraceOutputs)]


class ACBatchConfig(ctypes.Structure):
    _fields_ = [("block_size", ctypes.c_int32), ("chunk_rays", ctypes.c_int32), ("grid_blocks", ctypes.c_int32),
                ("stack_entries", ctypes.c_int32)]


class ACServiceConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("capacity", ctypes.c_int32), ("blocks_per_sm", ctypes.c_int32),
                ("block_size", ctypes.c_int32), ("chunk_rays", ctypes.c_int32), ("stack_entries", ctypes.c_int32),
                ("idle_timeout_ns", ctypes.c_int64), ("reserve_blocks", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class ACServiceStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_int64), ("in_flight", ctypes.c_int64), ("launches", ctypes.c_int64),
                ("running_launches", ctypes.c_int32), ("grid_blocks", ctypes.c_int32), ("capacity", ctypes.c_int64),
                ("warps_alive", ctypes.c_int64), ("warps_waiting", ctypes.c_int64)]


class ACServiceJobState(ctypes.Structure):
    _fields_ = [("seq", ctypes.c_int64), ("chunks", ctypes.c_int64), ("chunks_taken", ctypes.c_int64),
                ("rays", ctypes.c_int64), ("rays_finished", ctypes.c_int64), ("done_seq", ctypes.c_int64),
                ("low_water", ctypes.c_int64), ("in_flight", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class ACSynthParams(ctypes.Structure):
    _fields_ = [
        ("num_rirs", ctypes.c_int32), ("num_bins", ctypes.c_int32), ("samples_per_bin", ctypes.c_int32),
        ("sample_rate", ctypes.c_int32), ("rng_mode", ctypes.c_int32), ("white_shared", ctypes.c_int32),
        ("white", ctypes.c_void_p), ("seed", ctypes.c_uint64), ("air", ctypes.c_void_p),
        ("direct_delays", ctypes.c_void_p), ("air_coefficients", ctypes.c_double * 6),
        ("speed_of_sound", ctypes.c_double), ("crossover", ctypes.c_double * 100),
    ]


AC_SYNTH_MAX_RATES = 4
AC_TRAVERSAL_AUTO, AC_TRAVERSAL_SCAN, AC_TRAVERSAL_BVH, AC_TRAVERSAL_HYBRID = 0, 1, 2, 3


class ACSynthJob(ctypes.Structure):
    _fields_ = [
        ("echogram", ctypes.c_void_p), ("band_irs", ctypes.c_void_p), ("white", ctypes.c_void_p),
        ("air", ctypes.c_void_p), ("seed", ctypes.c_uint64), ("direct_delay", ctypes.c_double),
        ("speed_of_sound", ctypes.c_double), ("num_bins", ctypes.c_int32), ("samples_per_bin", ctypes.c_int32),
        ("rate_index", ctypes.c_int32), ("rng_mode", ctypes.c_int32),
    ]


class ACSynthBatchConfig(ctypes.Structure):
    _fields_ = [
        ("num_rates", ctypes.c_int32), ("sample_rates", ctypes.c_int32 * AC_SYNTH_MAX_RATES),
        ("crossover", (ctypes.c_double * 100) * AC_SYNTH_MAX_RATES), ("air_coefficients", ctypes.c_double * 6),
    ]


AC_FDN_LINES, AC_FDN_ALLPASS, AC_FDN_MIN_DELAY, AC_FDN_MAX_ALLPASS = 16, 4, 128, 4096
AC_LATE_STATS = 8
(AC_LATE_SCALE, AC_LATE_POWER, AC_LATE_FDN_ENERGY, AC_LATE_TRACED_TAIL, AC_LATE_RENDERED_TAIL, AC_LATE_COMPONENT,
 AC_LATE_CHANGED) = range(7)


class ACFdnJob(ctypes.Structure):
    _fields_ = [
        ("absorptive", ctypes.c_double * (AC_FDN_LINES * 6 * 5)), ("tone", ctypes.c_double * 30),
        ("delays", ctypes.c_int32 * AC_FDN_LINES), ("allpass_delays", ctypes.c_int32 * AC_FDN_ALLPASS),
        ("num_samples", ctypes.c_int32), ("preroll", ctypes.c_int32), ("out", ctypes.c_void_p),
    ]


class ACLateTailJob(ctypes.Structure):
    _fields_ = [
        ("traced", ctypes.c_void_p), ("fdn", ctypes.c_void_p), ("out", ctypes.c_void_p),
        ("fdn_component", ctypes.c_void_p), ("stats", ctypes.c_void_p), ("rt60", ctypes.c_double * 6),
        ("start", ctypes.c_int32 * 6), ("end", ctypes.c_int32 * 6), ("anchor", ctypes.c_int32 * 6),
        ("changed_from", ctypes.c_int32), ("num_samples", ctypes.c_int32), ("bin_samples", ctypes.c_int32),
        ("rate_index", ctypes.c_int32),
    ]


AC_DIRECT_MAX_LAYERS = 64


class ACDirectQuery(ctypes.Structure):
    _fields_ = [
        ("source", ctypes.c_double * 3), ("listener", ctypes.c_double * 3), ("radius", ctypes.c_double),
        ("occlusion", ctypes.c_int32), ("volumetric", ctypes.c_int32), ("transmission", ctypes.c_int32),
        ("max_layers", ctypes.c_int32),
    ]


class ACDirectResult(ctypes.Structure):
    _fields_ = [("occlusion", ctypes.c_double), ("transmission", ctypes.c_double * 6),
                ("occlusion_surface", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class ACDirectTables(ctypes.Structure):
    _fields_ = [("unit_samples", ctypes.c_void_p), ("num_samples", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("transmission", ctypes.c_void_p), ("surface_group", ctypes.c_void_p)]


# Every symbol include/acoustic_rt.h declares, with (restype, argtypes).
SIGNATURES: dict[str, tuple[Any, list[Any]]] = {
    "ac_last_error": (ctypes.c_char_p, []),
    "ac_abi_version": (ctypes.c_int, []),
    "ac_bvh_build": (ctypes.c_int, [c_double_p, c_double_p, ctypes.c_int64, ctypes.c_int32, ctypes.POINTER(ACBvh)]),
    "ac_bvh_device_workspace_size": (ctypes.c_int, [ctypes.c_int64, ctypes.c_int32, ctypes.POINTER(ctypes.c_size_t),
                                                    ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_int64)]),
    "ac_bvh_barrier_probe": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int64, ctypes.c_void_p,
                                            ctypes.c_void_p, ctypes.c_void_p]),
    "ac_bvh_build_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32,
                                           ctypes.POINTER(ACBvh), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                           ctypes.c_void_p, ctypes.c_void_p]),
    "ac_device_info": (ctypes.c_int, [ctypes.c_int32, ctypes.c_char_p, ctypes.c_size_t, c_int32_p, c_int32_p,
                                      c_int32_p]),
    "ac_scene_create": (ctypes.c_int, [ctypes.POINTER(ACSceneDesc), ctypes.POINTER(ctypes.c_void_p)]),
    "ac_scene_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "ac_scene_get_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ACSceneInfo)]),
    "ac_energy_scale": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ACTraceParams), c_double_p]),
    "ac_trace": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ACTraceParams), ctypes.POINTER(ACTraceOutputs),
                                ctypes.c_void_p]),
    "ac_batch_workspace_size": (ctypes.c_int, [ctypes.POINTER(ACJob), ctypes.c_int32, ctypes.POINTER(ACBatchConfig),
                                               ctypes.POINTER(ctypes.c_size_t)]),
    "ac_trace_batch": (ctypes.c_int, [ctypes.POINTER(ACJob), ctypes.c_int32, ctypes.POINTER(ACBatchConfig),
                                      ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p]),
    "ac_batch_submit": (ctypes.c_int, [ctypes.POINTER(ACJob), ctypes.c_int32, ctypes.POINTER(ACBatchConfig),
                                       ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.POINTER(ctypes.c_void_p)]),
    "ac_batch_poll": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32)]),
    "ac_batch_wait": (ctypes.c_int, [ctypes.c_void_p]),
    "ac_batch_release": (ctypes.c_int, [ctypes.c_void_p]),
    "ac_synth_workspace_size": (ctypes.c_int, [ctypes.POINTER(ACSynthParams), ctypes.POINTER(ctypes.c_size_t)]),
    "ac_synthesize": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ACSynthParams), ctypes.c_void_p,
                                     ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]),
    "ac_synth_batch_workspace_size": (ctypes.c_int, [ctypes.POINTER(ACSynthJob), ctypes.c_int32,
                                                     ctypes.POINTER(ACSynthBatchConfig),
                                                     ctypes.POINTER(ctypes.c_size_t)]),
    "ac_synthesize_batch": (ctypes.c_int, [ctypes.POINTER(ACSynthJob), ctypes.c_int32,
                                           ctypes.POINTER(ACSynthBatchConfig), ctypes.c_void_p, ctypes.c_size_t,
                                           ctypes.c_void_p, ctypes.c_void_p]),
    "ac_synthesize_batch_raw": (ctypes.c_int, [ctypes.POINTER(ACSynthJob), ctypes.c_int32,
                                               ctypes.POINTER(ACSynthBatchConfig), ctypes.c_void_p, ctypes.c_size_t,
                                               ctypes.c_void_p, ctypes.c_void_p]),
    "ac_synthesize_batch_filter": (ctypes.c_int, [ctypes.POINTER(ACSynthJob), ctypes.c_int32,
                                                  ctypes.POINTER(ACSynthBatchConfig), ctypes.c_void_p,
                                                  ctypes.c_size_t, ctypes.c_void_p]),
    "ac_fdn_workspace_size": (ctypes.c_int, [ctypes.POINTER(ACFdnJob), ctypes.c_int32,
                                             ctypes.POINTER(ctypes.c_size_t)]),
    "ac_fdn_impulse": (ctypes.c_int, [ctypes.POINTER(ACFdnJob), ctypes.c_int32, ctypes.c_void_p, ctypes.c_size_t,
                                      ctypes.c_void_p, ctypes.c_void_p]),
    "ac_late_tail_workspace_size": (ctypes.c_int, [ctypes.POINTER(ACLateTailJob), ctypes.c_int32,
                                                   ctypes.POINTER(ACSynthBatchConfig),
                                                   ctypes.POINTER(ctypes.c_size_t)]),
    "ac_late_tail": (ctypes.c_int, [ctypes.POINTER(ACLateTailJob), ctypes.c_int32,
                                    ctypes.POINTER(ACSynthBatchConfig), ctypes.c_void_p, ctypes.c_size_t,
                                    ctypes.c_void_p, ctypes.c_void_p]),
    "ac_direct_workspace_size": (ctypes.c_int, [ctypes.c_int32, ctypes.POINTER(ctypes.c_size_t)]),
    "ac_direct": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ACDirectQuery), ctypes.c_int32,
                                 ctypes.POINTER(ACDirectTables), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                 ctypes.c_void_p, ctypes.c_void_p]),
    "ac_fp64_rate_probe": (ctypes.c_int, [ctypes.c_int32, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64),
                                          ctypes.c_void_p]),
    "ac_read_bandwidth_probe": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int32, ctypes.c_void_p,
                                               ctypes.c_void_p]),
    "ac_synthesize_static": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ACSynthParams), ctypes.c_void_p,
                                            ctypes.c_void_p]),
    "ac_philox_workspace": (ctypes.c_int, [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int64, ctypes.c_int32,
                                           ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_void_p, ctypes.c_void_p]),
    "ac_service_create": (ctypes.c_int, [ctypes.POINTER(ACServiceConfig), ctypes.POINTER(ctypes.c_void_p)]),
    "ac_service_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ACJob), ctypes.c_int32,
                                         ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p]),
    "ac_service_poll": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64), ctypes.c_int32,
                                       ctypes.POINTER(ctypes.c_int32)]),
    "ac_service_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ACServiceStats)]),
    "ac_service_inspect": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ACServiceJobState)]),
    "ac_service_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "ac_reference_stream": (ctypes.c_int, [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
                                           ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
}


class BackendError(RuntimeError):
    """A libacoustic_rt call failed; carries the library's status code."""

    def __init__(self, code: int, message: str) -> None:
        super().__init__(message)
        self.code = code


_LIB: ctypes.CDLL | None = None


def load() -> ctypes.CDLL:
    global _LIB
    if _LIB is not None:
        return _LIB
    path = Path(os.environ.get("ACOUSTIC_RT_LIBRARY", str(LIBRARY_PATH)))
    if not path.exists():
        raise ImportError(
            f"{path} is missing: build the CUDA backend first (python acoustic-agent_b200/build.py); "
            "there is no CPU fallback")
    lib = ctypes.CDLL(str(path))
    for name, (restype, argtypes) in SIGNATURES.items():
        fn = getattr(lib, name)  # AttributeError if the ABI is incomplete
        fn.restype = restype
        fn.argtypes = argtypes
    _LIB = lib
    return lib


def check(code: int, what: str) -> None:
    if code != AC_OK:
        message = load().ac_last_error().decode("utf-8", "replace")
        if code == AC_ERR_INVALID:
            raise ValueError(f"{what}: {message}")
        raise BackendError(code, f"{what} failed ({code}): {message}")


def _ptr(array: np.ndarray, ctype):
    return array.ctypes.data_as(ctypes.POINTER(ctype))


def device_bvh_plan(num_surfaces: int, leaf_size: int = 4) -> tuple[int, int, int]:
    """(device workspace bytes, plan staging bytes, node count) of ac_bvh_build_device; host only."""
    ws, staging, nodes = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_int64()
    check(load().ac_bvh_device_workspace_size(int(num_surfaces), int(leaf_size), ctypes.byref(ws),
                                              ctypes.byref(staging), ctypes.byref(nodes)),
          "ac_bvh_device_workspace_size")
    return int(ws.value), int(staging.value), int(nodes.value)


def build_bvh(bounds_min: np.ndarray, bounds_max: np.ndarray, leaf_size: int = 4) -> dict[str, Any]:
    """BVH of bvh.py:8-77, built natively (host only)."""
    lower = np.ascontiguousarray(bounds_min, dtype=np.float64)
    upper = np.ascontiguousarray(bounds_max, dtype=np.float64)
    if lower.shape != upper.shape or lower.ndim != 2 or lower.shape[1] != 3:
        raise ValueError("BVH bounds must have shape [surface, 3]")
    n = lower.shape[0]
    if n < 1:
        raise ValueError("BVH requires at least one surface")
    cap = 2 * n
    out = {
        "bounds_min": np.zeros((cap, 3)), "bounds_max": np.zeros((cap, 3)), "start": np.zeros(cap, np.int64),
        "count": np.zeros(cap, np.int64), "escape": np.zeros(cap, np.int64), "primitives": np.zeros(n, np.int64),
    }
    bvh = ACBvh(_ptr(out["bounds_min"], ctypes.c_double), _ptr(out["bounds_max"], ctypes.c_double),
                _ptr(out["start"], ctypes.c_int64), _ptr(out["count"], ctypes.c_int64),
                _ptr(out["escape"], ctypes.c_int64), _ptr(out["primitives"], ctypes.c_int64), 0, 0, 0)
    check(load().ac_bvh_build(_ptr(lower, ctypes.c_double), _ptr(upper, ctypes.c_double), n, int(leaf_size),
                              ctypes.byref(bvh)), "ac_bvh_build")
    nodes = int(bvh.node_count)
    return {
        "bounds_min": out["bounds_min"][:nodes].copy(), "bounds_max": out["bounds_max"][:nodes].copy(),
        "start": out["start"][:nodes].copy(), "count": out["count"][:nodes].copy(),
        "escape": out["escape"][:nodes].copy(), "primitives": out["primitives"].copy(),
        "node_count": nodes, "leaf_count": int(bvh.leaf_count), "max_depth": int(bvh.max_depth),
        "leaf_size": max(1, int(leaf_size)),
    }
