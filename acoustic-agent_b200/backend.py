"""Drop-in reflection backend for Acoustic Agent.

``trace_energy_field`` has the signature, argument meaning, error behaviour
and result dictionary of ``acoustic_agent.steam_rt.trace_energy_field``
(steam_rt.py:1757-1804; result layout of its CUDA branch, :1892-1923).
``install()`` wires it into a running Acoustic Agent so that
``SimConfig(rt_accelerator="b200")`` (and, on request, ``"cuda"``) routes the
reflection trace of ``AcousticAgent.create(...).run()`` here, with the rest of
the solver (direct sound, diffraction, FDN tail, band synthesis) unchanged.

Differences from the reference CUDA backend, all deliberate:
* ``rt_precision="float64"`` is accepted and runs the float64 parity kernel
  (the reference CUDA backend rejects it);
* echogram bins are accumulated as int64 fixed point, so repeated runs are
  bit-identical;
* the random stream is the reference's own host arrays by default
  (``rng="reference"``), or an on-device Philox stream (``rng="philox"``).
"""
from __future__ import annotations

import math
import time
from collections import OrderedDict
from threading import Lock
from typing import Any, Mapping

import numpy as np
import torch

from acoustic_agent_b200 import runtime
from acoustic_agent_b200.directivity import source_directivity, source_forward
from acoustic_agent_b200.scene import SceneArrays, from_reference_arrays

ACCELERATOR_NAME = "b200"
_DEFAULT_RNG = "reference"
_VISUAL_RETAIN_LIMIT = 512  # steam_rt.py:42 _RT_VISUAL_RETAIN_LIMIT


def set_default_rng(mode: str) -> None:
    """Choose the random stream of drop-in traces: 'reference' (default) or 'philox'."""
    global _DEFAULT_RNG
    if mode not in ("reference", "philox"):
        raise ValueError("rng must be 'reference' or 'philox'")
    _DEFAULT_RNG = mode


def normalize_precision(value: str) -> str:
    """steam_rt.py:1814-1819 ``_normalize_rt_precision``."""
    aliases = {"fp32": "float32", "single": "float32", "fp64": "float64", "double": "float64"}
    precision = aliases.get(str(value).strip().lower(), str(value).strip().lower())
    if precision not in {"float32", "float64"}:
        raise ValueError("rt_precision must be float32 or float64")
    return precision


def resolve_intersection_backend(value: str, surface_count: int, min_surfaces: int) -> str:
    """steam_rt.py:222-231."""
    backend = str(value).strip().lower()
    if backend not in {"auto", "linear", "bvh"}:
        raise ValueError("intersection_backend must be auto, linear, or bvh")
    threshold = max(1, int(min_surfaces))
    return "bvh" if backend == "bvh" or (backend == "auto" and int(surface_count) >= threshold) else "linear"


class _SceneCache:
    """Resident device scenes keyed by the identity of their array dict (cf. steam_rt_cuda.py:229-261).

    ``acquire`` hands out a scene with a user count; ``release`` returns it.
    Only scenes without users are evicted (least recently used first), so a
    thread tracing a scene never sees it destroyed under it; while every entry
    is in use the cache holds more than ``limit`` scenes until they are
    released.  Work already enqueued on a stream is ordered before the memory
    is freed by ac_scene_destroy itself.
    """

    def __init__(self, limit: int = 32) -> None:
        self.limit = limit
        # key -> [array dict (kept alive so its id is not reused), scene, users]
        self.entries: OrderedDict[tuple[int, int], list[Any]] = OrderedDict()
        self.lock = Lock()

    def acquire(self, arrays: Mapping[str, Any] | SceneArrays, device: int) -> tuple[runtime.DeviceScene, bool]:
        key = (id(arrays), int(device))
        with self.lock:
            hit = self.entries.get(key)
            if hit is not None and hit[0] is arrays:
                hit[2] += 1
                self.entries.move_to_end(key)
                return hit[1], True
        scene = runtime.DeviceScene(arrays, device=device)
        evicted: list[runtime.DeviceScene] = []
        with self.lock:
            hit = self.entries.get(key)
            if hit is not None and hit[0] is arrays:
                # another thread uploaded the same arrays meanwhile: use its scene, drop ours
                hit[2] += 1
                self.entries.move_to_end(key)
                evicted.append(scene)
                scene, found = hit[1], True
            else:
                if hit is not None:
                    if hit[2] == 0:
                        evicted.append(hit[1])
                    del self.entries[key]
                self.entries[key] = [arrays, scene, 1]
                found = False
            for k in [k for k, e in self.entries.items() if e[2] == 0]:
                if len(self.entries) <= self.limit:
                    break
                evicted.append(self.entries.pop(k)[1])
        for old in evicted:
            old.close()
        return scene, found

    def release(self, scene: runtime.DeviceScene) -> None:
        with self.lock:
            for entry in self.entries.values():
                if entry[1] is scene:
                    entry[2] -= 1
                    return


SCENES = _SceneCache()


def _scene_arrays(scene: Any) -> Mapping[str, Any] | SceneArrays:
    if isinstance(scene, SceneArrays):
        return scene
    if isinstance(scene, Mapping):
        return from_reference_arrays(scene)
    # A reference RoomRayScene: reuse the reference's own cached SoA arrays.
    import sys

    steam_rt = sys.modules.get("acoustic_agent.steam_rt")
    if steam_rt is None or not hasattr(steam_rt, "_scene_kernel_arrays"):
        raise TypeError("scene must be a SceneArrays, an array dict, or an acoustic_agent RoomRayScene")
    return steam_rt._scene_kernel_arrays(scene)


def trace_energy_field(scene: Any, source: np.ndarray, listener: np.ndarray, config: Any,
                       source_model: str | Mapping[str, Any] | None = None, *, render_ambisonics: bool = True,
                       rng: str | None = None) -> dict[str, Any]:
    """Trace the six-band energy field on the GPU; same contract as the reference entry point."""
    emitter = source_directivity(source_model)
    precision = normalize_precision(config.rt_precision)
    device_id = int(getattr(config, "rt_cuda_device", 0))
    device = runtime.require_cuda(device_id)
    arrays = _scene_arrays(scene)
    names = tuple(arrays["names"])
    intersection_backend = resolve_intersection_backend(config.intersection_backend, len(names),
                                                        config.bvh_min_surfaces)
    num_rays = max(1, int(config.rt_num_rays))
    num_bounces = int(config.rt_num_bounces)
    bin_dur = float(config.rt_bin_duration_s)
    duration = max(float(config.rt_duration_s), float(config.duration_s))
    num_bins = max(1, int(math.ceil(duration / bin_dur)))
    src = np.asarray(source, dtype=float)
    lst = np.asarray(listener, dtype=float)
    direct_delay = float(np.linalg.norm(src - lst)) / float(config.c)
    collect_visual = bool(getattr(config, "collect_visual_paths", False))
    visual_limit, visual_stride = runtime.visual_candidate_layout(
        num_rays, collect_visual, getattr(config, "rt_visual_num_rays", None), retain_limit=_VISUAL_RETAIN_LIMIT)
    mode = rng or _DEFAULT_RNG
    spec = runtime.TraceSpec(
        source=src, listener=lst, source_forward=source_forward(emitter), num_rays=num_rays,
        num_bounces=num_bounces, num_bins=num_bins, bin_duration=bin_dur, speed_of_sound=float(config.c),
        max_path_length=duration * float(config.c), direct_delay=direct_delay,
        listener_radius=float(config.rt_listener_radius), source_radius=float(config.rt_source_radius),
        irradiance_min_distance=float(config.rt_irradiance_min_distance),
        specular_exponent=float(config.rt_specular_exponent), dipole_weight=float(emitter["dipole_weight"]),
        dipole_power=float(emitter["dipole_power"]), use_bvh=intersection_backend == "bvh",
        render_ambisonics=bool(render_ambisonics), precision=precision, rng=mode, seed=int(config.seed),
        stream_key=0, visual_limit=visual_limit, visual_stride=visual_stride,
    )
    transfer_started = time.perf_counter()
    hits_before, misses_before = runtime.STREAMS.hits, runtime.STREAMS.misses
    device_scene, scene_hit = SCENES.acquire(arrays, device_id)
    try:
        stream = torch.cuda.current_stream(device)
        buffers = runtime.TraceBuffers.allocate(device_scene.num_surfaces, num_bins, device,
                                                ambisonics=bool(render_ambisonics),
                                                visual=(visual_limit, num_bounces, spec.dtype) if visual_limit
                                                else None)
        if mode == "reference":
            runtime.reference_stream(spec, device)
        runtime.diffuse_bank(spec.dtype, device)
        stream.synchronize()
        upload_time = time.perf_counter() - transfer_started
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        runtime.trace(device_scene, spec, buffers, stream=stream)
        stop.record(stream)
    finally:
        SCENES.release(device_scene)
    stop.synchronize()
    kernel_time = start.elapsed_time(stop) / 1000.0
    download_started = time.perf_counter()
    field = runtime.host_field(buffers, names, spec)
    transfer_time = upload_time + (time.perf_counter() - download_started)
    cache_stats = {"hits": runtime.STREAMS.hits - hits_before + (1 if scene_hit else 0),
                   "misses": runtime.STREAMS.misses - misses_before + (0 if scene_hit else 1)}
    return {
        "echogram": field["echogram"],
        "ambisonic_echogram": field["ambisonic_echogram"] if render_ambisonics else None,
        "num_bins": num_bins,
        "bin_duration_s": bin_dur,
        "direct_delay_s": direct_delay,
        "actual_bounces": field["actual_bounces"],
        "active_ray_count": field["active_ray_count"],
        "last_energy_time_s": field["last_energy_time_s"],
        "surface_hit_count": field["surface_hit_count"],
        "surface_contribution_count": field["surface_contribution_count"],
        "surface_energy": field["surface_energy"],
        "visual_candidates": field.get("visual_candidates") if collect_visual else None,
        "accelerator": ACCELERATOR_NAME,
        "precision": precision,
        "cuda": {k: v for k, v in runtime.device_info(device_id).items() if k != "sm_count"},
        "device_input_cache": cache_stats,
        "kernel_time_s": float(kernel_time),
        "transfer_time_s": float(transfer_time),
        "intersection_backend": intersection_backend,
        "source_directivity": dict(emitter),
    }


class Installation:
    """Handle returned by install(); ``uninstall()`` restores the reference's functions."""

    def __init__(self, module: Any, originals: dict[str, Any]) -> None:
        self.module = module
        self.originals = originals

    def uninstall(self) -> None:
        for name, fn in self.originals.items():
            setattr(self.module, name, fn)


def install(steam_rt_module: Any = None, *, route_cuda: bool = False,
            gpu_bvh_min_surfaces: int | None = None) -> Installation:
    """Route Acoustic Agent's reflection trace to this backend.

    After ``install()``, ``rt_accelerator="b200"`` selects the GPU tracer here; with
    ``route_cuda=True`` the reference's ``"cuda"`` setting is routed here too.  Other
    settings keep the reference's own dispatch (steam_rt.py:1757-1811).  The same
    setting routes the FDN late tail (``_render_parametric_fdn_late_reverb``,
    steam_rt.py:2500, called by the renderer at :1029) to ``late_reverb`` and the
    direct path (``simulate_direct``, :1315, called at :942) to ``direct``.

    ``gpu_bvh_min_surfaces=N`` also routes the scene BVH build (``build_bvh``,
    called by ``_scene_kernel_arrays`` at steam_rt.py:881 with no accelerator
    setting in reach) to the GPU build in ``bvh`` for scenes of N surfaces or
    more; the tree is the reference's, array for array.
    """
    if steam_rt_module is None:
        import acoustic_agent.steam_rt as steam_rt_module  # type: ignore[import-not-found]
    original_trace = steam_rt_module.trace_energy_field
    original_normalize = steam_rt_module._normalize_rt_accelerator
    handled = {ACCELERATOR_NAME} | ({"cuda"} if route_cuda else set())

    def normalize(value: str) -> str:
        accelerator = str(value).strip().lower()
        if accelerator in handled:
            return accelerator
        return original_normalize(value)

    def routed_trace(scene, source, listener, config, source_model=None, *, render_ambisonics=True):
        accelerator = normalize(config.rt_accelerator)
        if accelerator in handled:
            return trace_energy_field(scene, source, listener, config, source_model,
                                      render_ambisonics=render_ambisonics)
        return original_trace(scene, source, listener, config, source_model, render_ambisonics=render_ambisonics)

    originals = {"trace_energy_field": original_trace, "_normalize_rt_accelerator": original_normalize}
    steam_rt_module.trace_energy_field = routed_trace
    steam_rt_module._normalize_rt_accelerator = normalize
    original_late = getattr(steam_rt_module, "_render_parametric_fdn_late_reverb", None)
    if original_late is not None:

        def routed_late(traced_band_irs, field, rt60_bands, config, *, decay_profiles=None):
            if normalize(config.rt_accelerator) in handled:
                from acoustic_agent_b200 import late_reverb
                return late_reverb.render_parametric_fdn_late_reverb(traced_band_irs, field, rt60_bands, config,
                                                                     decay_profiles=decay_profiles)
            return original_late(traced_band_irs, field, rt60_bands, config, decay_profiles=decay_profiles)

        steam_rt_module._render_parametric_fdn_late_reverb = routed_late
        originals["_render_parametric_fdn_late_reverb"] = original_late
    original_direct = getattr(steam_rt_module, "simulate_direct", None)
    if original_direct is not None:

        def routed_direct(scene, source, listener, config, source_model=None):
            if normalize(config.rt_accelerator) in handled:
                from acoustic_agent_b200 import direct
                return direct.simulate_direct(scene, source, listener, config, source_model)
            return original_direct(scene, source, listener, config, source_model)

        steam_rt_module.simulate_direct = routed_direct
        originals["simulate_direct"] = original_direct
    original_bvh = getattr(steam_rt_module, "build_bvh", None)
    if gpu_bvh_min_surfaces is not None and original_bvh is not None:
        threshold = max(1, int(gpu_bvh_min_surfaces))

        def routed_bvh(bounds_min, bounds_max, *, leaf_size: int = 4):
            if len(bounds_min) >= threshold:
                from acoustic_agent_b200 import bvh
                return bvh.build_bvh(bounds_min, bounds_max, leaf_size=leaf_size)
            return original_bvh(bounds_min, bounds_max, leaf_size=leaf_size)

        steam_rt_module.build_bvh = routed_bvh
        originals["build_bvh"] = original_bvh
    return Installation(steam_rt_module, originals)
