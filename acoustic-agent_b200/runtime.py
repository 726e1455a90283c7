"""Device runtime: resident scenes, trace launches, band synthesis.

PyTorch supplies device memory and streams; every computation runs in
libacoustic_rt.so.  Nothing here falls back to the CPU: without a CUDA device
the calls raise.
"""
from __future__ import annotations

import ctypes
import math
from collections import OrderedDict
from dataclasses import dataclass, field
from threading import Lock
from typing import Any, Mapping, Sequence

import numpy as np
import torch

from acoustic_agent_b200 import _lib, bands, rng
from acoustic_agent_b200.scene import SceneArrays

NUM_BANDS = 6
NUM_BANK = 128


def require_cuda(device: int = 0) -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("the B200 reflection backend needs a CUDA device; it has no CPU fallback")
    if not 0 <= int(device) < torch.cuda.device_count():
        raise RuntimeError(f"CUDA device {device} is not available")
    return torch.device("cuda", int(device))


def _f64(a: Any) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _i64(a: Any) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int64)


def _dp(a: np.ndarray):
    return a.ctypes.data_as(_lib.c_double_p)


def _ip(a: np.ndarray):
    return a.ctypes.data_as(_lib.c_int64_p)


def _stream_ptr(stream: torch.cuda.Stream | None) -> ctypes.c_void_p:
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


MAX_STACK_ENTRIES = 32   # traversal stack entries per lane at most (the library's kBvhStack)


class DeviceScene:
    """A scene uploaded with ac_scene_create; owns its device memory."""

    TRAVERSALS = {"auto": 0, "scan": 1, "bvh": 2, "hybrid": 3}

    def __init__(self, arrays: SceneArrays | Mapping[str, Any], device: int = 0, *, cluster_size: int = 0,
                 traversal: str = "auto", bvh_leaf: int = 0, bvh_width: int = 0, stack_entries: int = 0) -> None:
        if traversal not in self.TRAVERSALS:
            raise ValueError(f"traversal must be one of {sorted(self.TRAVERSALS)}")
        require_cuda(device)
        a = arrays.arrays if isinstance(arrays, SceneArrays) else dict(arrays)
        self.names: tuple[str, ...] = tuple(a["names"])
        keep = {
            "kinds": _i64(a["kinds"]), "wall_a": _f64(a["wall_a"]), "wall_delta": _f64(a["wall_delta"]),
            "wall_z": _f64(a["wall_z"]), "z_values": _f64(a["z_values"]), "box_center": _f64(a["box_center"]),
            "box_axis_u": _f64(a["box_axis_u"]), "box_axis_v": _f64(a["box_axis_v"]),
            "box_half": _f64(a["box_half"]), "box_z": _f64(a["box_z"]), "normals": _f64(a["normals"]),
            "reflection": _f64(a["reflection"]), "scattering": _f64(a["scattering"]),
            "corners": _f64(np.asarray(a["corners"])[:, :2]), "bvh_bounds_min": _f64(a["bvh_bounds_min"]),
            "bvh_bounds_max": _f64(a["bvh_bounds_max"]), "bvh_start": _i64(a["bvh_start"]),
            "bvh_count": _i64(a["bvh_count"]), "bvh_escape": _i64(a["bvh_escape"]),
            "bvh_primitives": _i64(a["bvh_primitives"]),
        }
        S = keep["kinds"].shape[0]
        desc = _lib.ACSceneDesc()
        desc.num_surfaces = S
        desc.kinds = _ip(keep["kinds"])
        for name in ("wall_a", "wall_delta", "wall_z", "z_values", "box_center", "box_axis_u", "box_axis_v",
                     "box_half", "box_z", "normals", "reflection", "scattering", "corners"):
            setattr(desc, name, _dp(keep[name]))
        desc.num_corners = keep["corners"].shape[0]
        desc.bvh_node_count = keep["bvh_start"].shape[0]
        desc.bvh_bounds_min = _dp(keep["bvh_bounds_min"])
        desc.bvh_bounds_max = _dp(keep["bvh_bounds_max"])
        desc.bvh_start = _ip(keep["bvh_start"])
        desc.bvh_count = _ip(keep["bvh_count"])
        desc.bvh_escape = _ip(keep["bvh_escape"])
        desc.bvh_primitives = _ip(keep["bvh_primitives"])
        desc.device = int(device)
        desc.cluster_size = int(cluster_size)
        desc.traversal = self.TRAVERSALS[traversal]
        desc.bvh_leaf = int(bvh_leaf)
        desc.bvh_width = int(bvh_width)
        if "surface_bounds_min" in a and "surface_bounds_max" in a:
            keep["surface_bounds_min"] = _f64(a["surface_bounds_min"])
            keep["surface_bounds_max"] = _f64(a["surface_bounds_max"])
            desc.surface_bounds_min = _dp(keep["surface_bounds_min"])
            desc.surface_bounds_max = _dp(keep["surface_bounds_max"])
        handle = ctypes.c_void_p()
        _lib.check(_lib.load().ac_scene_create(ctypes.byref(desc), ctypes.byref(handle)), "ac_scene_create")
        self.handle = handle
        self.device = int(device)
        self.num_surfaces = S
        info = _lib.ACSceneInfo()
        _lib.check(_lib.load().ac_scene_get_info(handle, ctypes.byref(info)), "ac_scene_get_info")
        self.device_bytes = int(info.device_bytes)
        self.node_count = int(info.node_count)
        self.num_clusters = int(info.num_clusters)
        self.traversal = {1: "scan", 2: "bvh", 3: "hybrid"}.get(int(info.traversal), "scan")
        self.bvh_depth = int(info.bvh_depth)
        self.bvh_nodes = int(info.bvh_nodes)
        self.bvh_width = int(info.bvh_width)
        self.bvh_stack_need = int(info.bvh_stack_need)
        # traversal stack entries per lane that launches over this scene use unless told otherwise (a tuned
        # schedule knob; 0: the library's maximum)
        self.stack_entries = int(stack_entries) if self.bvh_nodes > 0 else 0
        self.max_reflection = float(np.max(keep["reflection"])) if S else 0.0
        # events recorded after CUDA-graph replays that read this scene (the library tracks eager launches
        # itself, not work captured into a graph); close() waits for them
        self.graph_guards: list[torch.cuda.Event] = []
        if self.stack_entries and not self.bvh_stack_need <= self.stack_entries <= MAX_STACK_ENTRIES:
            self.close()
            raise ValueError(f"stack_entries must lie in {self.bvh_stack_need}..{MAX_STACK_ENTRIES} for this scene")

    def close(self) -> None:
        if getattr(self, "handle", None) is not None and self.handle.value:
            for event in getattr(self, "graph_guards", ()):
                event.synchronize()
            _lib.load().ac_scene_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self) -> None:  # pragma: no cover - interpreter teardown order varies
        try:
            self.close()
        except Exception:
            pass


@dataclass
class TraceSpec:
    """Host-side description of one trace (the fields of ac_trace_params)."""

    source: Sequence[float]
    listener: Sequence[float]
    num_rays: int
    num_bounces: int
    num_bins: int
    bin_duration: float
    speed_of_sound: float
    max_path_length: float
    direct_delay: float
    source_forward: Sequence[float] = (1.0, 0.0, 0.0)
    listener_radius: float = 0.1
    source_radius: float = 0.1
    irradiance_min_distance: float = 1.0
    specular_exponent: float = 100.0
    dipole_weight: float = 0.0
    dipole_power: float = 1.0
    use_bvh: bool = False
    render_ambisonics: bool = False
    precision: str = "float32"
    rng: str = "philox"
    seed: int = 1729
    stream_key: int = 0
    energy_scale: float = 0.0
    block_size: int = 0
    grid_blocks: int = 0
    stack_entries: int = 0     # traversal stack entries per lane (0: the scene's choice, else the library's)
    visual_limit: int = 0      # visual-path candidate slots (0: none)
    visual_stride: int = 1

    @property
    def dtype(self) -> torch.dtype:
        return torch.float64 if self.precision == "float64" else torch.float32


class _StreamCache:
    """Device copies of reference-stream workspaces (cf. steam_rt_cuda.py:229-261), LRU by bytes."""

    def __init__(self, limit_bytes: int = 512 * 1024 * 1024) -> None:
        self.limit = limit_bytes
        self.entries: OrderedDict[tuple, tuple[torch.Tensor, ...]] = OrderedDict()
        self.bytes = 0
        self.hits = 0
        self.misses = 0
        self.lock = Lock()

    def get(self, key: tuple, build) -> tuple[torch.Tensor, ...]:
        with self.lock:
            hit = self.entries.get(key)
            if hit is not None:
                self.entries.move_to_end(key)
                self.hits += 1
                return hit
        value = build()
        size = sum(t.numel() * t.element_size() for t in value)
        with self.lock:
            self.misses += 1
            if size <= self.limit:   # an entry that can never fit is returned uncached, evicting nothing
                while self.entries and self.bytes + size > self.limit:
                    _, old = self.entries.popitem(last=False)
                    self.bytes -= sum(t.numel() * t.element_size() for t in old)
                self.entries[key] = value
                self.bytes += size
        return value


STREAMS = _StreamCache()


def diffuse_bank(dtype: torch.dtype, device: torch.device) -> torch.Tensor:
    key = ("bank", NUM_BANK, dtype, device.index)
    return STREAMS.get(key, lambda: (torch.as_tensor(rng.diffuse_sample_bank(NUM_BANK), dtype=dtype, device=device),))[0]


def reference_stream(spec: TraceSpec, device: torch.device) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    key = ("stream", int(spec.num_rays), int(spec.num_bounces), NUM_BANK, int(spec.seed), spec.dtype, device.index)

    def build():
        # directions (cos/sin of the host's libm, 24 bytes per ray) are drawn on the host; the per-bounce
        # uniforms and bank indices (12 bytes per ray-bounce) on the device, the same draws bit for bit
        directions = torch.as_tensor(np.array(rng.sphere_samples(spec.num_rays, spec.seed), copy=True),
                                     dtype=spec.dtype, device=device)
        drawn = rng.device_diffuse_random_sequence(spec.num_rays, spec.num_bounces, NUM_BANK, spec.seed,
                                                   dtype=spec.dtype, device=device)
        if drawn is None:
            random_values, indices = rng.diffuse_random_sequence(spec.num_rays, spec.num_bounces, NUM_BANK,
                                                                 spec.seed)
            drawn = (torch.as_tensor(np.array(random_values, copy=True), dtype=spec.dtype, device=device),
                     torch.as_tensor(np.array(indices, copy=True), dtype=torch.int32, device=device))
        # the cached tensors may be read from any stream next: finish drawing them first
        torch.cuda.current_stream(device).synchronize()
        return (directions, *drawn)

    return STREAMS.get(key, build)


@dataclass
class TraceBuffers:
    """Device outputs of one trace."""

    echogram_fx: torch.Tensor
    hit_counts: torch.Tensor
    contrib_counts: torch.Tensor
    surface_energy_fx: torch.Tensor
    counters: torch.Tensor
    echogram: torch.Tensor
    surface_energy: torch.Tensor
    ambisonic_fx: torch.Tensor | None = None
    ambisonic: torch.Tensor | None = None
    ray_surfaces: torch.Tensor | None = None
    scale: ctypes.c_double = field(default_factory=lambda: ctypes.c_double(0.0))
    visual: dict[str, torch.Tensor] | None = None   # visual-path candidate arrays (allocate(visual=...))

    @classmethod
    def allocate(cls, num_surfaces: int, num_bins: int, device: torch.device, *, ambisonics: bool = False,
                 record_rays: tuple[int, int] | None = None, echogram: bool = True,
                 visual: tuple[int, int, torch.dtype] | None = None) -> "TraceBuffers":
        """Zeroed device outputs; echogram=False leaves `echogram` for the caller to point at its own storage.

        visual=(limit, bounces, dtype) adds the visual-candidate arrays (the trace initialises them).
        """
        z64 = lambda *shape: torch.zeros(*shape, dtype=torch.int64, device=device)
        vis = None
        if visual is not None and visual[0] > 0:
            limit, bounces, dtype = visual
            e = lambda *shape, dt: torch.empty(*shape, dtype=dt, device=device)  # noqa: E731
            vis = {"hit_points": e(limit, max(1, bounces), 3, dt=dtype),
                   "surface_indices": e(limit, max(1, bounces), dt=torch.int32),
                   "ray_indices": e(limit, dt=torch.int32), "orders": e(limit, dt=torch.int32),
                   "distances": e(limit, dt=dtype), "gains": e(limit, dt=dtype)}
        return cls(visual=vis, **dict(
            echogram_fx=z64(NUM_BANDS, num_bins, 2), hit_counts=z64(num_surfaces), contrib_counts=z64(num_surfaces),
            surface_energy_fx=z64(num_surfaces, 2), counters=z64(8),
            echogram=(torch.zeros(NUM_BANDS, num_bins, dtype=torch.float32, device=device) if echogram
                      else torch.empty(0, dtype=torch.float32, device=device)),
            surface_energy=torch.zeros(num_surfaces, dtype=torch.float32, device=device),
            ambisonic_fx=z64(NUM_BANDS, 4, num_bins, 2) if ambisonics else None,
            ambisonic=torch.zeros(NUM_BANDS, 4, num_bins, dtype=torch.float32, device=device) if ambisonics else None,
            ray_surfaces=(torch.empty(record_rays[0], record_rays[1], dtype=torch.int32, device=device)
                          if record_rays else None),
        ))

    def outputs_struct(self) -> _lib.ACTraceOutputs:
        o = _lib.ACTraceOutputs()
        o.echogram_fx = self.echogram_fx.data_ptr()
        o.ambisonic_fx = self.ambisonic_fx.data_ptr() if self.ambisonic_fx is not None else None
        o.hit_counts = self.hit_counts.data_ptr()
        o.contrib_counts = self.contrib_counts.data_ptr()
        o.surface_energy_fx = self.surface_energy_fx.data_ptr()
        o.counters = self.counters.data_ptr()
        o.echogram = self.echogram.data_ptr()
        o.ambisonic = self.ambisonic.data_ptr() if self.ambisonic is not None else None
        o.surface_energy = self.surface_energy.data_ptr()
        o.ray_surfaces = self.ray_surfaces.data_ptr() if self.ray_surfaces is not None else None
        o.scale_out = ctypes.pointer(self.scale)
        if self.visual is not None:
            o.visual_hit_points = self.visual["hit_points"].data_ptr()
            o.visual_surfaces = self.visual["surface_indices"].data_ptr()
            o.visual_rays = self.visual["ray_indices"].data_ptr()
            o.visual_orders = self.visual["orders"].data_ptr()
            o.visual_distances = self.visual["distances"].data_ptr()
            o.visual_gains = self.visual["gains"].data_ptr()
        return o


def params_struct(spec: TraceSpec, device: torch.device, keepalive: list[Any] | None = None,
                  workspace: tuple[torch.Tensor, torch.Tensor, torch.Tensor] | None = None) -> _lib.ACTraceParams:
    """ac_trace_params for `spec`.  In reference-stream mode the random workspace is the reference's own
    (generated from the seed and cached), or `workspace` = (directions [R,3], uniforms [B,R], bank indices
    [B,R]) already on the device in the trace's precision (int32 indices)."""
    p = _lib.ACTraceParams()
    p.source[:] = [float(v) for v in spec.source]
    p.listener[:] = [float(v) for v in spec.listener]
    p.source_forward[:] = [float(v) for v in spec.source_forward]
    p.num_rays = int(spec.num_rays)
    p.num_bounces = int(spec.num_bounces)
    p.num_bins = int(spec.num_bins)
    p.bin_duration = float(spec.bin_duration)
    p.speed_of_sound = float(spec.speed_of_sound)
    p.max_path_length = float(spec.max_path_length)
    p.direct_delay = float(spec.direct_delay)
    p.listener_radius = float(spec.listener_radius)
    p.source_radius = float(spec.source_radius)
    p.irradiance_min_distance = float(spec.irradiance_min_distance)
    p.specular_exponent = float(spec.specular_exponent)
    p.dipole_weight = float(spec.dipole_weight)
    p.dipole_power = float(spec.dipole_power)
    p.use_bvh = 1 if spec.use_bvh else 0
    p.render_ambisonics = 1 if spec.render_ambisonics else 0
    if spec.precision not in ("float32", "float64"):
        raise ValueError("rt_precision must be float32 or float64")
    p.precision = _lib.AC_PRECISION_FP64 if spec.precision == "float64" else _lib.AC_PRECISION_FP32
    if spec.rng not in ("reference", "philox"):
        raise ValueError("rng must be 'reference' or 'philox'")
    p.rng_mode = _lib.AC_RNG_REFERENCE if spec.rng == "reference" else _lib.AC_RNG_PHILOX
    p.seed = int(spec.seed) & 0xFFFFFFFFFFFFFFFF
    p.stream_key = int(spec.stream_key) & 0xFFFFFFFFFFFFFFFF
    bank = diffuse_bank(spec.dtype, device)
    p.diffuse_bank = bank.data_ptr()
    p.num_bank = NUM_BANK
    if spec.rng == "reference":
        if workspace is not None:
            directions, random_values, indices = workspace
            R, B = int(spec.num_rays), int(spec.num_bounces)
            if (tuple(directions.shape) != (R, 3) or tuple(random_values.shape) != (B, R)
                    or tuple(indices.shape) != (B, R) or directions.dtype != spec.dtype
                    or random_values.dtype != spec.dtype or indices.dtype != torch.int32
                    or not all(t.is_cuda and t.is_contiguous() for t in workspace)):
                raise ValueError("workspace must be contiguous device tensors: directions [R,3] and uniforms "
                                 "[B,R] in the trace's precision, bank indices [B,R] int32")
        else:
            directions, random_values, indices = reference_stream(spec, device)
        p.directions = directions.data_ptr()
        p.diffuse_random = random_values.data_ptr()
        p.diffuse_indices = indices.data_ptr()
        if keepalive is not None:
            keepalive.extend([directions, random_values, indices])
    if keepalive is not None:
        keepalive.append(bank)
    p.energy_scale = float(spec.energy_scale)
    p.block_size = int(spec.block_size)
    p.grid_blocks = int(spec.grid_blocks)
    p.stack_entries = int(spec.stack_entries)
    p.visual_limit = int(spec.visual_limit)
    p.visual_stride = int(spec.visual_stride)
    return p


def trace(scene: DeviceScene, spec: TraceSpec, buffers: TraceBuffers | None = None, *,
          stream: torch.cuda.Stream | None = None, record_rays: bool = False,
          workspace: tuple[torch.Tensor, torch.Tensor, torch.Tensor] | None = None) -> TraceBuffers:
    """Launch one trace asynchronously on `stream` and return its device buffers (`workspace`: see
    params_struct)."""
    device = require_cuda(scene.device)
    if buffers is None:
        buffers = TraceBuffers.allocate(scene.num_surfaces, int(spec.num_bins), device,
                                        ambisonics=spec.render_ambisonics,
                                        record_rays=(int(spec.num_rays), int(spec.num_bounces)) if record_rays else None)
    keep: list[Any] = []
    params = params_struct(spec, device, keep, workspace)
    if not params.stack_entries:
        params.stack_entries = scene.stack_entries
    outputs = buffers.outputs_struct()
    _lib.check(_lib.load().ac_trace(scene.handle, ctypes.byref(params), ctypes.byref(outputs), _stream_ptr(stream)),
               "ac_trace")
    buffers._keepalive = keep  # type: ignore[attr-defined]
    return buffers


class _StagedWorkspace:
    """Device workspace + pinned staging of a batched entry point.

    The entry point writes its job table into the pinned staging on the host
    and copies it to the device asynchronously, so the staging may be
    rewritten only after that copy has run: `ensure` waits for the event
    recorded after the previous launch.  (Inside a stream capture no event is
    needed: the graph owns the staging until it is released.)
    """

    SIZE_FN = ""

    def __init__(self, device: torch.device) -> None:
        self.device = device
        self.device_buffer: torch.Tensor | None = None
        self.host_buffer: torch.Tensor | None = None
        self._copied: torch.cuda.Event | None = None

    def ensure(self, jobs, num_jobs: int, cfg=None) -> tuple[int, int, int]:
        size = ctypes.c_size_t()
        args = (jobs, num_jobs) + ((ctypes.byref(cfg),) if cfg is not None else ()) + (ctypes.byref(size),)
        _lib.check(getattr(_lib.load(), self.SIZE_FN)(*args), self.SIZE_FN)
        need = max(int(size.value), 256)
        if self._copied is not None and not torch.cuda.is_current_stream_capturing():
            self._copied.synchronize()   # host waits are not allowed inside a capture (nor needed there)
            self._copied = None
        if self.device_buffer is None or self.device_buffer.numel() < need:
            cap = max(need, 2 * (self.device_buffer.numel() if self.device_buffer is not None else 0), 1 << 16)
            self.device_buffer = torch.empty(cap, dtype=torch.uint8, device=self.device)
            self.host_buffer = torch.empty(cap, dtype=torch.uint8, pin_memory=True)
        assert self.device_buffer is not None and self.host_buffer is not None
        return self.device_buffer.data_ptr(), self.device_buffer.numel(), self.host_buffer.data_ptr()

    def idle(self) -> bool:
        """True when the staging may be rewritten without waiting (its last launch has run)."""
        return self._copied is None or self._copied.query()

    def launched(self, stream: torch.cuda.Stream | None) -> None:
        if torch.cuda.is_current_stream_capturing():
            return
        ev = torch.cuda.Event()
        ev.record(stream if stream is not None else torch.cuda.current_stream(self.device))
        self._copied = ev


class BatchWorkspace(_StagedWorkspace):
    """Reusable device workspace + pinned staging for ac_trace_batch."""

    SIZE_FN = "ac_batch_workspace_size"


def launch_stack_entries(scenes: Sequence[DeviceScene]) -> int:
    """Stack entries of one launch over `scenes`: the largest of the BVH scenes' choices, or 0 (the library's
    maximum) when one of them has none."""
    prefs = [s.stack_entries for s in scenes if s.bvh_nodes > 0]
    return max(prefs) if prefs and all(prefs) else 0


def trace_batch(jobs: Sequence[tuple[DeviceScene, TraceSpec, TraceBuffers]], workspace: BatchWorkspace, *,
                block_size: int = 0, grid_blocks: int = 0, chunk_rays: int = 0, stack_entries: int | None = None,
                stream: torch.cuda.Stream | None = None) -> None:
    """All jobs in one persistent launch (ac_trace_batch); `stack_entries` None: launch_stack_entries."""
    if not jobs:
        return
    device = require_cuda(jobs[0][0].device)
    arr = (_lib.ACJob * len(jobs))()
    keep: list[Any] = []
    for k, (scene, spec, buffers) in enumerate(jobs):
        arr[k].scene = scene.handle.value
        arr[k].params = params_struct(spec, device, keep)
        arr[k].outputs = buffers.outputs_struct()
    if stack_entries is None:
        stack_entries = launch_stack_entries([scene for scene, _, _ in jobs])
    cfg = _lib.ACBatchConfig(int(block_size), int(chunk_rays), int(grid_blocks), int(stack_entries))
    ws, ws_bytes, host = workspace.ensure(arr, len(jobs), cfg)
    _lib.check(_lib.load().ac_trace_batch(arr, len(jobs), ctypes.byref(cfg), ctypes.c_void_p(ws), ws_bytes,
                                          ctypes.c_void_p(host), _stream_ptr(stream)), "ac_trace_batch")
    workspace.launched(stream)
    workspace._keepalive = keep  # type: ignore[attr-defined]


class TraceService:
    """Continuous batching on one GPU (ac_service_*): one persistent trace launch fed while it runs.

    ``submit`` appends (scene, spec, buffers) jobs -- float32, Philox stream -- and returns their sequence
    numbers; ``poll`` returns the sequence numbers whose outputs are complete (never blocks).  Jobs submitted
    while others are on the GPU join the running launch.  The service keeps each job's parameter tables and
    buffers alive until it is reported done.
    """

    def __init__(self, device: int = 0, *, capacity: int = 4096, blocks_per_sm: int = 2, block_size: int = 0,
                 chunk_rays: int = 0, stack_entries: int = 0, idle_timeout_s: float = 0.02,
                 reserve_blocks: int = 0) -> None:
        self.device = require_cuda(device)
        cfg = _lib.ACServiceConfig(int(device), int(capacity), int(blocks_per_sm), int(block_size), int(chunk_rays),
                                   int(stack_entries), int(idle_timeout_s * 1e9), int(reserve_blocks), 0)
        handle = ctypes.c_void_p()
        _lib.check(_lib.load().ac_service_create(ctypes.byref(cfg), ctypes.byref(handle)), "ac_service_create")
        self.handle = handle
        self._keep: dict[int, Any] = {}
        self._done = (ctypes.c_int64 * 4096)()

    def submit(self, jobs: Sequence[tuple[DeviceScene, TraceSpec, TraceBuffers]], *,
               stream: torch.cuda.Stream | None = None) -> list[int]:
        """Append jobs; raises BackendError(AC_ERR_CAPACITY) when the ring cannot take them yet.

        The jobs are traced only after the work queued on `stream` (default: the current stream) before the
        call, such as the zero fill of freshly allocated output buffers."""
        if not jobs:
            return []
        arr = (_lib.ACJob * len(jobs))()
        keep: list[Any] = []
        for k, (scene, spec, buffers) in enumerate(jobs):
            if spec.rng != "philox" or spec.precision != "float32":
                raise ValueError("the trace service runs float32 jobs on the Philox stream")
            arr[k].scene = scene.handle.value
            arr[k].params = params_struct(spec, self.device, keep)
            arr[k].outputs = buffers.outputs_struct()
            keep.append((scene, buffers))
        first = ctypes.c_int64()
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        _lib.check(_lib.load().ac_service_submit(self.handle, arr, len(jobs), ctypes.byref(first),
                                                 _stream_ptr(stream)), "ac_service_submit")
        seqs = list(range(first.value, first.value + len(jobs)))
        for seq in seqs:
            self._keep[seq] = keep
        return seqs

    def poll(self) -> list[int]:
        out: list[int] = []
        while True:
            n = ctypes.c_int32()
            _lib.check(_lib.load().ac_service_poll(self.handle, self._done, len(self._done), ctypes.byref(n)),
                       "ac_service_poll")
            out.extend(self._done[k] for k in range(n.value))
            if n.value < len(self._done):
                break
        for seq in out:
            self._keep.pop(seq, None)
        return out

    def job_state(self, seq: int) -> dict[str, int]:
        """Progress of one of the last `capacity` submitted jobs (ac_service_inspect)."""
        st = _lib.ACServiceJobState()
        _lib.check(_lib.load().ac_service_inspect(self.handle, int(seq), ctypes.byref(st)), "ac_service_inspect")
        return {k: int(getattr(st, k)) for k, _ in st._fields_ if k != "reserved"}

    def info(self) -> dict[str, int]:
        st = _lib.ACServiceStats()
        _lib.check(_lib.load().ac_service_info(self.handle, ctypes.byref(st)), "ac_service_info")
        return {k: int(getattr(st, k)) for k, _ in st._fields_}

    def close(self) -> None:
        if getattr(self, "handle", None) is not None and self.handle.value:
            _lib.check(_lib.load().ac_service_destroy(self.handle), "ac_service_destroy")
            self.handle = ctypes.c_void_p()
            self._keep.clear()

    def __del__(self) -> None:  # pragma: no cover - interpreter teardown order varies
        try:
            self.close()
        except Exception:
            pass


class BatchTicket:
    """Completion ticket of ac_batch_submit: ``done()`` polls, ``wait()`` blocks, ``release()`` frees it."""

    def __init__(self, handle: ctypes.c_void_p, keep: list[Any]) -> None:
        self.handle = handle
        self._keep = keep   # the job table's parameter tables stay alive until the batch is done

    def done(self) -> bool:
        flag = ctypes.c_int32()
        _lib.check(_lib.load().ac_batch_poll(self.handle, ctypes.byref(flag)), "ac_batch_poll")
        return bool(flag.value)

    def wait(self) -> None:
        _lib.check(_lib.load().ac_batch_wait(self.handle), "ac_batch_wait")

    def release(self) -> None:
        if self.handle:
            _lib.check(_lib.load().ac_batch_release(self.handle), "ac_batch_release")
            self.handle = ctypes.c_void_p()
            self._keep = []

    def __del__(self) -> None:
        try:
            self.release()
        except Exception:
            pass


def submit_batch(jobs: Sequence[tuple[DeviceScene, TraceSpec, TraceBuffers]], workspace: BatchWorkspace, *,
                 block_size: int = 0, grid_blocks: int = 0, chunk_rays: int = 0, stack_entries: int | None = None,
                 stream: torch.cuda.Stream | None = None) -> BatchTicket:
    """trace_batch through the queue entry points: the launch plus a ticket to poll (ac_batch_submit)."""
    if not jobs:
        raise ValueError("submit_batch needs at least one job")
    device = require_cuda(jobs[0][0].device)
    arr = (_lib.ACJob * len(jobs))()
    keep: list[Any] = []
    for k, (scene, spec, buffers) in enumerate(jobs):
        arr[k].scene = scene.handle.value
        arr[k].params = params_struct(spec, device, keep)
        arr[k].outputs = buffers.outputs_struct()
    if stack_entries is None:
        stack_entries = launch_stack_entries([scene for scene, _, _ in jobs])
    cfg = _lib.ACBatchConfig(int(block_size), int(chunk_rays), int(grid_blocks), int(stack_entries))
    ws, ws_bytes, host = workspace.ensure(arr, len(jobs), cfg)
    handle = ctypes.c_void_p()
    _lib.check(_lib.load().ac_batch_submit(arr, len(jobs), ctypes.byref(cfg), ctypes.c_void_p(ws), ws_bytes,
                                           ctypes.c_void_p(host), _stream_ptr(stream), ctypes.byref(handle)),
               "ac_batch_submit")
    workspace.launched(stream)
    return BatchTicket(handle, keep)


def fixed_to_float64(fixed: torch.Tensor, scale: float) -> np.ndarray:
    """Fixed-point word pairs [..., 2] -> float64 values: (word1 * 2^32 + word0) / scale."""
    words = fixed.cpu().numpy()
    low = words[..., 0].view(np.uint64).astype(np.float64)
    high = words[..., 1].astype(np.float64)
    return (high * 4294967296.0 + low) / float(scale)


def host_field(buffers: TraceBuffers, names: Sequence[str], spec: TraceSpec) -> dict[str, Any]:
    """Copy one trace's outputs to the host in the reference's result layout (steam_rt.py:1892-1923)."""
    echogram = buffers.echogram.cpu().numpy()
    hits = buffers.hit_counts.cpu().numpy()
    contrib = buffers.contrib_counts.cpu().numpy()
    energy = buffers.surface_energy.cpu().numpy()
    counters = buffers.counters.cpu().numpy()
    total_energy = np.sum(echogram, axis=0)
    nonzero = np.flatnonzero(total_energy > 0.0)
    out = {
        "echogram": echogram,
        "ambisonic_echogram": buffers.ambisonic.cpu().numpy() if buffers.ambisonic is not None else None,
        "num_bins": int(spec.num_bins),
        "bin_duration_s": float(spec.bin_duration),
        "direct_delay_s": float(spec.direct_delay),
        "actual_bounces": int(counters[0]),
        "active_ray_count": int(counters[1]),
        "last_energy_time_s": float(nonzero[-1] * spec.bin_duration) if nonzero.size else 0.0,
        "surface_hit_count": {names[i]: int(hits[i]) for i in range(len(names)) if int(hits[i]) > 0},
        "surface_contribution_count": {names[i]: int(contrib[i]) for i in range(len(names)) if int(contrib[i]) > 0},
        "surface_energy": {names[i]: float(energy[i]) for i in range(len(names)) if float(energy[i]) > 0.0},
        "ray_bounces": int(counters[2]),
        "shadow_rays": int(counters[3]),
        "energy_scale": float(buffers.scale.value),
    }
    if buffers.ray_surfaces is not None:
        out["ray_surfaces"] = buffers.ray_surfaces.cpu().numpy()
    if buffers.visual is not None and spec.visual_limit > 0:
        vis = {k: v.cpu().numpy() for k, v in buffers.visual.items()}
        if spec.num_bounces < 1:   # [L, 0, ...] like the reference when there are no bounces
            vis["hit_points"] = vis["hit_points"][:, :0]
            vis["surface_indices"] = vis["surface_indices"][:, :0]
        vis.update({"surface_names": tuple(names), "candidate_limit": int(spec.visual_limit),
                    "stride": int(spec.visual_stride)})
        out["visual_candidates"] = vis
    return out


def visual_candidate_layout(num_rays: int, collect: bool, visual_num_rays: int | None = None,
                            retain_limit: int = 512) -> tuple[int, int]:
    """(limit, stride) of the visual-candidate slots, as steam_rt.py:1853-1860 sets them."""
    default = int(retain_limit * 4)
    requested = default if visual_num_rays is None else max(1, min(int(visual_num_rays), default))
    limit = min(int(num_rays), requested) if collect else 0
    stride = max(1, int(num_rays) // max(limit, 1))
    return limit, stride


# ---------------------------------------------------------------------------
# Band synthesis


class SynthWorkspace:
    def __init__(self, device: torch.device) -> None:
        self.device = device
        self.buffer: torch.Tensor | None = None

    def ensure(self, nbytes: int) -> torch.Tensor:
        if self.buffer is None or self.buffer.numel() < nbytes:
            self.buffer = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=self.device)
        return self.buffer


def synth_params(num_rirs: int, num_bins: int, bin_duration: float, fs: int, speed_of_sound: float, *,
                 rng_mode: str, seed: int, white: torch.Tensor | None = None, white_shared: bool = True,
                 direct_delays: torch.Tensor | None = None, air: torch.Tensor | None = None) -> _lib.ACSynthParams:
    p = _lib.ACSynthParams()
    p.num_rirs = int(num_rirs)
    p.num_bins = int(num_bins)
    p.samples_per_bin = bands.samples_per_bin(bin_duration, fs)
    p.sample_rate = int(fs)
    p.rng_mode = _lib.AC_RNG_PHILOX if rng_mode == "philox" else _lib.AC_RNG_REFERENCE
    p.white_shared = 1 if white_shared else 0
    p.white = white.data_ptr() if white is not None else None
    p.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    p.air = air.data_ptr() if air is not None else None
    p.direct_delays = direct_delays.data_ptr() if direct_delays is not None else None
    p.air_coefficients[:] = list(bands.AIR_ABSORPTION_NP_PER_M)
    p.speed_of_sound = float(speed_of_sound)
    p.crossover[:] = [float(v) for v in bands.crossover_table(fs).reshape(-1)]
    return p


def synthesize(echograms: torch.Tensor, params: _lib.ACSynthParams, workspace: SynthWorkspace,
               out: torch.Tensor | None = None, *, stream: torch.cuda.Stream | None = None) -> torch.Tensor:
    """[J,6,bins] float32 echograms -> [J,6,N] float32 band IRs (ac_synthesize)."""
    if echograms.dtype != torch.float32 or not echograms.is_cuda or not echograms.is_contiguous():
        raise ValueError("echograms must be a contiguous float32 CUDA tensor")
    J = int(params.num_rirs)
    N = int(params.num_bins) * int(params.samples_per_bin)
    if out is None:
        out = torch.empty(J, NUM_BANDS, N, dtype=torch.float32, device=echograms.device)
    size = ctypes.c_size_t()
    _lib.check(_lib.load().ac_synth_workspace_size(ctypes.byref(params), ctypes.byref(size)), "ac_synth_workspace_size")
    ws = workspace.ensure(int(size.value))
    _lib.check(_lib.load().ac_synthesize(ctypes.c_void_p(echograms.data_ptr()), ctypes.byref(params),
                                         ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(ws.data_ptr()),
                                         ws.numel(), _stream_ptr(stream)), "ac_synthesize")
    return out


@dataclass
class SynthJob:
    """One RIR of a ragged synthesis batch (the fields of ac_synth_job)."""

    echogram: torch.Tensor            # [6, bins] float32 CUDA
    out: torch.Tensor                 # [6, bins * spb] float32 CUDA
    fs: int
    bin_duration: float
    seed: int                         # Philox noise key (reconstruct_band_irs draws with config.seed + 7)
    direct_delay: float
    speed_of_sound: float = 343.0
    rng: str = "philox"
    white: torch.Tensor | None = None  # reference mode: [bins * spb] float64 CUDA noise
    air: torch.Tensor | None = None    # optional [6, bins] float64 CUDA air gains


def synth_batch_config(rates: Sequence[int]) -> _lib.ACSynthBatchConfig:
    rates = list(dict.fromkeys(int(r) for r in rates))
    if not 1 <= len(rates) <= _lib.AC_SYNTH_MAX_RATES:
        raise ValueError(f"a synthesis batch takes 1..{_lib.AC_SYNTH_MAX_RATES} sample rates, got {len(rates)}")
    cfg = _lib.ACSynthBatchConfig()
    cfg.num_rates = len(rates)
    for k, fs in enumerate(rates):
        cfg.sample_rates[k] = fs
        cfg.crossover[k][:] = [float(v) for v in bands.crossover_table(fs).reshape(-1)]
    cfg.air_coefficients[:] = list(bands.AIR_ABSORPTION_NP_PER_M)
    return cfg


def synth_job_array(jobs: Sequence[SynthJob], config: _lib.ACSynthBatchConfig) -> ctypes.Array:
    rate_index = {int(config.sample_rates[k]): k for k in range(config.num_rates)}
    arr = (_lib.ACSynthJob * max(1, len(jobs)))()
    for k, j in enumerate(jobs):
        spb = bands.samples_per_bin(j.bin_duration, j.fs)
        bins = int(j.echogram.shape[-1])
        if j.echogram.dtype != torch.float32 or not j.echogram.is_contiguous() or tuple(j.echogram.shape) != (NUM_BANDS, bins):
            raise ValueError("echogram must be a contiguous [6, bins] float32 tensor")
        if j.out.dtype != torch.float32 or not j.out.is_contiguous() or tuple(j.out.shape) != (NUM_BANDS, bins * spb):
            raise ValueError(f"band IR output must be a contiguous [6, {bins * spb}] float32 tensor")
        if j.rng not in ("philox", "reference"):
            raise ValueError("rng must be 'reference' or 'philox'")
        a = arr[k]
        a.echogram = j.echogram.data_ptr()
        a.band_irs = j.out.data_ptr()
        a.white = j.white.data_ptr() if j.white is not None else None
        a.air = j.air.data_ptr() if j.air is not None else None
        a.seed = int(j.seed) & 0xFFFFFFFFFFFFFFFF
        a.direct_delay = float(j.direct_delay)
        a.speed_of_sound = float(j.speed_of_sound)
        a.num_bins = bins
        a.samples_per_bin = spb
        a.rate_index = rate_index[int(j.fs)]
        a.rng_mode = _lib.AC_RNG_PHILOX if j.rng == "philox" else _lib.AC_RNG_REFERENCE
    return arr


class SynthBatchWorkspace(_StagedWorkspace):
    """Reusable device workspace + pinned staging for ac_synthesize_batch."""

    SIZE_FN = "ac_synth_batch_workspace_size"


def synthesize_batch(jobs: Sequence[SynthJob] | tuple[ctypes.Array, int, _lib.ACSynthBatchConfig],
                     workspace: SynthBatchWorkspace, *, stream: torch.cuda.Stream | None = None,
                     phase: str = "all") -> None:
    """Band IRs of every job in three launches (ac_synthesize_batch); outputs land in each job's `out`.

    phase="raw" then phase="filter" (same jobs and workspace, the second
    ordered after the first, possibly on another stream) split the work at
    the crossover recursion (ac_synthesize_batch_raw / _filter).
    """
    if phase not in ("all", "raw", "filter"):
        raise ValueError("phase must be 'all', 'raw' or 'filter'")
    if isinstance(jobs, tuple):
        arr, n, cfg = jobs
    else:
        if not jobs:
            return
        cfg = synth_batch_config([j.fs for j in jobs])
        arr, n = synth_job_array(jobs, cfg), len(jobs)
    if n == 0:
        return
    lib = _lib.load()
    if phase == "filter":
        if workspace.device_buffer is None:
            raise RuntimeError("the filter phase needs the workspace of a preceding raw phase")
        _lib.check(lib.ac_synthesize_batch_filter(arr, n, ctypes.byref(cfg),
                                                  ctypes.c_void_p(workspace.device_buffer.data_ptr()),
                                                  workspace.device_buffer.numel(), _stream_ptr(stream)),
                   "ac_synthesize_batch_filter")
        return
    ws, ws_bytes, host = workspace.ensure(arr, n, cfg)
    fn = lib.ac_synthesize_batch if phase == "all" else lib.ac_synthesize_batch_raw
    _lib.check(fn(arr, n, ctypes.byref(cfg), ctypes.c_void_p(ws), ws_bytes, ctypes.c_void_p(host),
                  _stream_ptr(stream)), "ac_synthesize_batch")
    workspace.launched(stream)


# ---------------------------------------------------------------------------
# Late reverberation (FDN impulse + hybrid tail)


class FdnWorkspace(_StagedWorkspace):
    """Reusable device workspace + pinned staging for ac_fdn_impulse."""

    SIZE_FN = "ac_fdn_workspace_size"


class LateTailWorkspace(_StagedWorkspace):
    """Reusable device workspace + pinned staging for ac_late_tail."""

    SIZE_FN = "ac_late_tail_workspace_size"


def fdn_impulse(jobs: ctypes.Array, num_jobs: int, workspace: FdnWorkspace, *,
                stream: torch.cuda.Stream | None = None) -> None:
    """Every job's FDN impulse response into its `out` (ac_fdn_impulse), one launch."""
    if num_jobs == 0:
        return
    ws, ws_bytes, host = workspace.ensure(jobs, num_jobs)
    _lib.check(_lib.load().ac_fdn_impulse(jobs, num_jobs, ctypes.c_void_p(ws), ws_bytes, ctypes.c_void_p(host),
                                          _stream_ptr(stream)), "ac_fdn_impulse")
    workspace.launched(stream)


def late_tail(jobs: ctypes.Array, num_jobs: int, config: _lib.ACSynthBatchConfig, workspace: LateTailWorkspace, *,
              stream: torch.cuda.Stream | None = None) -> None:
    """Band-limit, scale and crossfade every job's FDN into its traced band signals (ac_late_tail)."""
    if num_jobs == 0:
        return
    ws, ws_bytes, host = workspace.ensure(jobs, num_jobs, config)
    _lib.check(_lib.load().ac_late_tail(jobs, num_jobs, ctypes.byref(config), ctypes.c_void_p(ws), ws_bytes,
                                        ctypes.c_void_p(host), _stream_ptr(stream)), "ac_late_tail")
    workspace.launched(stream)


def fp64_rate_tops(device: torch.device, *, iterations: int = 8192, launches: int = 5) -> float:
    """Measured float64 add/multiply issue rate of the whole GPU in 10^12 operations/s (ac_fp64_rate_probe)."""
    sink = torch.zeros(1, dtype=torch.int64, device=device)
    stream = torch.cuda.current_stream(device)
    lib = _lib.load()
    ops = ctypes.c_int64()

    def launch():
        _lib.check(lib.ac_fp64_rate_probe(int(iterations), ctypes.c_void_p(sink.data_ptr()), ctypes.byref(ops),
                                          _stream_ptr(stream)), "ac_fp64_rate_probe")

    launch()
    best = 0.0
    for _ in range(launches):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        launch()
        e1.record(stream)
        e1.synchronize()
        best = max(best, ops.value / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    return best


def read_bandwidth_gbs(device: torch.device, nbytes: int, *, repeats: int = 10, launches: int = 20) -> float:
    """Measured read bandwidth (GB/s) over a buffer of `nbytes`: L2 when it fits, HBM otherwise."""
    buf = torch.ones(nbytes // 4, dtype=torch.float32, device=device)
    sink = torch.zeros(1, dtype=torch.int64, device=device)
    stream = torch.cuda.current_stream(device)
    lib = _lib.load()

    def launch():
        _lib.check(lib.ac_read_bandwidth_probe(ctypes.c_void_p(buf.data_ptr()), buf.numel() * 4, int(repeats),
                                               ctypes.c_void_p(sink.data_ptr()), _stream_ptr(stream)),
                   "ac_read_bandwidth_probe")

    for _ in range(3):
        launch()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(launches):
        launch()
    stop.record(stream)
    stop.synchronize()
    return (buf.numel() // 4) * 16 * repeats * launches / (start.elapsed_time(stop) / 1000.0) / 1e9


def device_info(device: int = 0) -> dict[str, Any]:
    name = ctypes.create_string_buffer(256)
    major, minor, sms = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
    _lib.check(_lib.load().ac_device_info(int(device), name, 256, ctypes.byref(major), ctypes.byref(minor),
                                          ctypes.byref(sms)), "ac_device_info")
    return {"id": int(device), "name": name.value.decode(), "compute_capability": f"{major.value}.{minor.value}",
            "sm_count": int(sms.value)}


def ray_bounce_count(buffers: TraceBuffers) -> int:
    return int(buffers.counters[2].item())


def num_bins_for(duration_s: float, rt_duration_s: float, bin_duration_s: float) -> int:
    return max(1, int(math.ceil(max(float(rt_duration_s), float(duration_s)) / float(bin_duration_s))))
