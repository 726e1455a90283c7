"""Direct sound with GPU occlusion and transmission queries.

Drop-in for Acoustic Agent's ``simulate_direct`` (acoustic_agent/steam_rt.py:
1315-1350).  Distance, directivity, air absorption, delay and the band gains
are host arithmetic with the reference's formulas; the ray casting -- the
surface blocking the direct path, the volumetric visibility of the source
(``_volumetric_occlusion``, :4215-4240) and the transmission through the
surfaces crossed (``_transmission``, :3437-3462) -- runs in one float64 GPU
launch (``ac_direct``), for one pair or a whole batch of them.  The sample
sphere (``_sphere_volume_samples``, :4233-4240) is built here with numpy, as
the reference builds it.  There is no CPU path: the calls raise without the
library or a CUDA device.
"""
from __future__ import annotations

import ctypes
import math
from threading import Lock
from typing import Any, Mapping, Sequence

import numpy as np
import torch

from acoustic_agent_b200 import _lib, bands, runtime
from acoustic_agent_b200.directivity import source_directivity, source_forward


def sphere_volume_samples(count: int) -> np.ndarray:
    """[count, 3] points filling the unit ball: golden-angle longitudes, uniform cos(theta), radius by the
    cube root of the index (steam_rt.py:4233-4240)."""
    k = np.arange(count, dtype=float) + 0.5
    phi = 2.0 * math.pi * np.mod(k * 0.6180339887498949, 1.0)
    cz = 1.0 - 2.0 * k / count
    sz = np.sqrt(np.clip(1.0 - cz * cz, 0.0, 1.0))
    r = np.power(k / count, 1.0 / 3.0)
    return np.stack([r * sz * np.cos(phi), r * sz * np.sin(phi), r * cz], axis=1)


def directivity_gain(direction: Sequence[float], model: Mapping[str, Any]) -> float:
    """Weighted-dipole gain toward `direction` (acoustic_agent/directivity.py:70-78)."""
    v = np.asarray(direction, dtype=np.float64)
    n = float(np.linalg.norm(v))
    if n <= 1e-12:
        return 1.0
    c = float(np.clip(np.dot(source_forward(model), v / n), -1.0, 1.0))
    w = float(model.get("dipole_weight", 0.0))
    p = float(model.get("dipole_power", 1.0))
    return float(abs((1.0 - w) + w * c) ** p)


def surface_groups(names: Sequence[str]) -> np.ndarray:
    """Surfaces that share a name share a group: the transmission walk counts each name once."""
    ids: dict[str, int] = {}
    return np.asarray([ids.setdefault(str(n), len(ids)) for n in names], dtype=np.int32)


class DirectTables:
    """Device tables of one scene: per-surface band transmission and name groups, and the sample sphere."""

    def __init__(self, names: Sequence[str], transmission: np.ndarray, device: torch.device) -> None:
        t = np.ascontiguousarray(np.asarray(transmission, dtype=np.float64).reshape(len(names), 6))
        self.names = tuple(str(n) for n in names)
        self.transmission = torch.from_numpy(t).to(device)
        self.groups = torch.from_numpy(surface_groups(self.names)).to(device)
        self.device = device
        self._samples: dict[int, torch.Tensor] = {}

    def samples(self, count: int) -> torch.Tensor:
        if count not in self._samples:
            self._samples[count] = torch.from_numpy(np.ascontiguousarray(sphere_volume_samples(count))).to(self.device)
        return self._samples[count]


def run_queries(scene: runtime.DeviceScene, tables: DirectTables, queries: ctypes.Array, count: int, *,
                samples: int, stream: torch.cuda.Stream | None = None) -> np.ndarray:
    """ac_direct over `count` queries; returns the ac_direct_result records as a numpy structured array."""
    results = torch.empty(max(count, 1) * ctypes.sizeof(_lib.ACDirectResult), dtype=torch.uint8,
                          device=tables.device)
    t = _lib.ACDirectTables()
    sample_table = tables.samples(max(1, int(samples)))
    t.unit_samples = sample_table.data_ptr()
    t.num_samples = max(1, int(samples))
    t.transmission = tables.transmission.data_ptr()
    t.surface_group = tables.groups.data_ptr()
    lib = _lib.load()
    size = ctypes.c_size_t()
    _lib.check(lib.ac_direct_workspace_size(count, ctypes.byref(size)), "ac_direct_workspace_size")
    ws = torch.empty(max(int(size.value), 256), dtype=torch.uint8, device=tables.device)
    staging = torch.empty(max(int(size.value), 256), dtype=torch.uint8, pin_memory=True)
    stream = stream if stream is not None else torch.cuda.current_stream(tables.device)
    _lib.check(lib.ac_direct(scene.handle, queries, count, ctypes.byref(t), ctypes.c_void_p(results.data_ptr()),
                             ctypes.c_void_p(ws.data_ptr()), ws.numel(), ctypes.c_void_p(staging.data_ptr()),
                             ctypes.c_void_p(stream.cuda_stream)), "ac_direct")
    host = results.to("cpu", non_blocking=True)
    stream.synchronize()
    dtype = np.dtype([("occlusion", "<f8"), ("transmission", "<f8", (6,)), ("occlusion_surface", "<i4"),
                      ("reserved", "<i4")])
    return np.frombuffer(host.numpy().tobytes(), dtype=dtype)[:count].copy()


def make_query(source: np.ndarray, listener: np.ndarray, config: Any) -> _lib.ACDirectQuery:
    q = _lib.ACDirectQuery()
    q.source[:] = [float(v) for v in source]
    q.listener[:] = [float(v) for v in listener]
    q.radius = max(1e-4, float(config.direct_occlusion_radius_m))
    q.occlusion = 1 if config.direct_occlusion else 0
    q.volumetric = 1 if str(config.direct_occlusion_mode) == "volumetric" else 0
    q.transmission = 1 if config.direct_transmission else 0
    q.max_layers = max(1, int(config.num_transmission_rays))
    if q.max_layers > _lib.AC_DIRECT_MAX_LAYERS:
        raise ValueError(f"num_transmission_rays above {_lib.AC_DIRECT_MAX_LAYERS} is not supported")
    return q


_TABLES: dict[tuple[int, int], tuple[Any, DirectTables]] = {}
_TABLES_LOCK = Lock()


def scene_surfaces(scene: Any) -> tuple[list[str], np.ndarray]:
    """Names and [S, 6] transmission of a reference RoomRayScene's surfaces (in the kernel arrays' order)."""
    surfaces = getattr(scene, "surfaces", None)
    if surfaces is None:
        raise TypeError("the direct path needs an acoustic_agent RoomRayScene (surface transmission and names)")
    return [str(s.name) for s in surfaces], np.stack([np.asarray(s.transmission, dtype=float) for s in surfaces])


def _device_scene_and_tables(scene: Any, device_id: int) -> tuple[runtime.DeviceScene, DirectTables]:
    from acoustic_agent_b200 import backend
    arrays = backend._scene_arrays(scene)
    device_scene, _ = backend.SCENES.acquire(arrays, device_id)
    key = (id(scene), device_id)
    with _TABLES_LOCK:
        hit = _TABLES.get(key)
        if hit is not None and hit[0] is scene:
            return device_scene, hit[1]
    names, transmission = scene_surfaces(scene)
    tables = DirectTables(names, transmission, torch.device("cuda", device_id))
    with _TABLES_LOCK:
        _TABLES[key] = (scene, tables)
        while len(_TABLES) > 32:
            _TABLES.pop(next(iter(_TABLES)))
    return device_scene, tables


def simulate_direct_batch(scene: Any, pairs: Sequence[tuple[Sequence[float], Sequence[float]]], config: Any,
                          source_model: str | Mapping[str, Any] | None = None) -> list[dict[str, Any]]:
    """simulate_direct for many (source, listener) pairs of one scene, with one GPU launch for all of them."""
    device_id = int(getattr(config, "rt_cuda_device", 0))
    runtime.require_cuda(device_id)
    from acoustic_agent_b200 import backend
    with torch.cuda.device(device_id):
        device_scene, tables = _device_scene_and_tables(scene, device_id)
        try:
            return direct_results(device_scene, tables, pairs, config, source_model)
        finally:
            backend.SCENES.release(device_scene)


def direct_results(device_scene: runtime.DeviceScene, tables: DirectTables,
                   pairs: Sequence[tuple[Sequence[float], Sequence[float]]], config: Any,
                   source_model: str | Mapping[str, Any] | None = None) -> list[dict[str, Any]]:
    """The simulate_direct result dicts for `pairs` of a resident scene and its tables."""
    emitter = source_directivity(source_model)
    out: list[dict[str, Any]] = []
    queries = (_lib.ACDirectQuery * max(1, len(pairs)))()
    traced: list[int] = []
    geometry = []
    for source, listener in pairs:
        src = np.asarray(source, dtype=float)
        lst = np.asarray(listener, dtype=float)
        delta = src - lst
        distance = float(np.linalg.norm(delta))
        geometry.append((src, lst, distance))
        if config.direct_occlusion and distance > 1e-6:
            queries[len(traced)] = make_query(src, lst, config)
            traced.append(len(geometry) - 1)
    records = None
    names = tables.names
    if traced:
        records = run_queries(device_scene, tables, queries, len(traced),
                              samples=max(1, int(config.direct_occlusion_samples)))
    slot = {g: k for k, g in enumerate(traced)}
    for g, (src, lst, distance) in enumerate(geometry):
        gain = directivity_gain(lst - src, emitter)
        attenuation = 1.0 / max(distance, config.min_distance_m)
        air = np.asarray([math.exp(-bands.AIR_ABSORPTION_NP_PER_M[b] * distance) for b in range(6)], dtype=float)
        occlusion = 1.0
        transmission = np.ones(6, dtype=float)
        surface = None
        if g in slot:
            rec = records[slot[g]]
            occlusion = float(rec["occlusion"])
            surface = names[int(rec["occlusion_surface"])] if int(rec["occlusion_surface"]) >= 0 else None
            if occlusion < 1.0:
                transmission = np.asarray(rec["transmission"], dtype=float)
        band_gains = {band: float(gain * attenuation * air[i] * (occlusion + (1.0 - occlusion) * transmission[i]))
                      for i, band in enumerate(bands.FREQUENCY_BANDS)}
        out.append({
            "distance_m": distance,
            "delay_s": distance / config.c,
            "distance_attenuation": attenuation,
            "air_absorption": air,
            "occlusion": occlusion,
            "transmission": transmission,
            "occlusion_surface": surface,
            "source_directivity_gain": gain,
            "band_gains": band_gains,
        })
    return out


def simulate_direct(scene: Any, source: np.ndarray, listener: np.ndarray, config: Any,
                    source_model: str | Mapping[str, Any] | None = None) -> dict[str, Any]:
    """Same arguments and result dict as steam_rt.py:1315 ``simulate_direct``."""
    return simulate_direct_batch(scene, [(source, listener)], config, source_model)[0]
