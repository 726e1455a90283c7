"""Autotuner for the tracer's schedule: per-scene traversal and per-launch shape.

Every knob here changes only how the work is scheduled, never a result: the
closest surface is the minimum distance with ties to the lower index whatever
the visiting order, echogram bins are exact fixed-point sums, and rays are
keyed by (seed, stream key, ray index).  The GPU tests check bit-identical
outputs across traversal modes, leaf sizes, block sizes and chunk sizes, so
the tuner may choose by measured time alone.

Knobs
-----
per scene (``tune_scene``)
    ``traversal`` -- "scan" (kind-separated clusters in warp lockstep), "bvh"
    (per-lane descent of a surface-area-heuristic BVH with a short stack) or
    "hybrid" (walls in lockstep, a BVH over the boxes);
    ``bvh_leaf`` -- surfaces per BVH leaf (1, 2, 4): smaller leaves mean a
    deeper tree and a deeper traversal stack, fewer surface tests per leaf;
    ``stack_entries`` -- each lane's traversal stack (shared memory, 1 KiB
    per entry per 256-thread block), timed on the fastest traversal from the
    tree's own need up to 32: a shorter stack leaves more of the SM's on-chip
    memory to the L1 that holds the scene.  A launch over several scenes
    takes the largest of their choices unless it is tuned itself.
per launch (``tune_launch``)
    ``block_size`` -- rays per block (one ray per lane: 128 or 256 threads);
    ``chunk_rays`` -- queue granularity: rays a warp takes from the shared
    work counter at once (16 .. 128);
    ``stack_entries`` -- the stack depth again, for the launch as a whole,
    from the largest need among its BVH scenes, at the chosen shape.

Choices are cached by a fingerprint of the scene's surface arrays
(``TuneCache``), so a scene resident in a serving loop is tuned once.
"""
from __future__ import annotations

import hashlib
import json
import threading
from dataclasses import asdict, dataclass, replace
from pathlib import Path
from typing import Any, Sequence

import numpy as np
import torch

from acoustic_agent_b200 import runtime
from acoustic_agent_b200.scene import SceneArrays

SCENE_CANDIDATES: tuple[dict[str, Any], ...] = (
    {"traversal": "scan", "bvh_leaf": 0, "bvh_width": 0},
    {"traversal": "bvh", "bvh_leaf": 1, "bvh_width": 2},
    {"traversal": "bvh", "bvh_leaf": 2, "bvh_width": 2},
    {"traversal": "bvh", "bvh_leaf": 4, "bvh_width": 2},
    {"traversal": "hybrid", "bvh_leaf": 1, "bvh_width": 2},
)
# Four-wide BVHs (bvh_width=4) trace the same rays but measured 6-18 % slower than binary ones on the
# furnished U room and the 8-room apartment, so they are not timed by default; pass them in `candidates`.
WIDE_CANDIDATES: tuple[dict[str, Any], ...] = (
    {"traversal": "bvh", "bvh_leaf": 1, "bvh_width": 4},
    {"traversal": "hybrid", "bvh_leaf": 1, "bvh_width": 4},
)
LAUNCH_CANDIDATES: tuple[dict[str, int], ...] = tuple(
    {"block_size": b, "chunk_rays": c} for b in (256, 128) for c in (16, 32, 64, 128))


STACK_CANDIDATES: tuple[int, ...] = (8, 12, 16, 24, 32)


def stack_candidates(need: int) -> list[int]:
    """Stack depths to time for a tree that needs `need` entries: the need itself and the fixed steps above."""
    if need <= 0:
        return [0]
    return sorted({need} | {n for n in STACK_CANDIDATES if n >= need})


@dataclass(frozen=True)
class SceneChoice:
    traversal: str
    bvh_leaf: int
    ms: float
    bvh_width: int = 0
    stack_entries: int = 0              # 0: scan mode (no stack) or not tuned (the library's maximum)
    stack_ms: tuple[tuple[int, float], ...] = ()   # (entries, ms) of every depth timed

    def options(self) -> dict[str, Any]:
        return {"traversal": self.traversal, "bvh_leaf": self.bvh_leaf, "bvh_width": self.bvh_width,
                "stack_entries": self.stack_entries}


@dataclass(frozen=True)
class LaunchChoice:
    block_size: int
    chunk_rays: int
    ms: float
    stack_entries: int = 0              # 0: the launch needs no stack (scan scenes only) or was not tuned
    stack_ms: tuple[tuple[int, float], ...] = ()


def fingerprint(arrays: SceneArrays | dict[str, Any]) -> str:
    """Stable hash of the surface arrays the tracer reads."""
    a = arrays.arrays if isinstance(arrays, SceneArrays) else arrays
    h = hashlib.sha1()
    for key in ("kinds", "wall_a", "wall_delta", "wall_z", "z_values", "box_center", "box_axis_u", "box_axis_v",
                "box_half", "box_z", "corners"):
        v = np.ascontiguousarray(np.asarray(a[key], dtype=np.float64))
        h.update(key.encode())
        h.update(str(v.shape).encode())
        h.update(v.tobytes())
    return h.hexdigest()


class TuneCache:
    """Scene choices by fingerprint; optionally persisted as JSON."""

    def __init__(self, path: str | Path | None = None) -> None:
        self.path = Path(path) if path else None
        self.entries: dict[str, SceneChoice] = {}
        self._lock = threading.Lock()
        if self.path and self.path.exists():
            for key, value in json.loads(self.path.read_text()).items():
                value["stack_ms"] = tuple(tuple(x) for x in value.get("stack_ms", ()))
                self.entries[key] = SceneChoice(**value)

    def get(self, key: str) -> SceneChoice | None:
        with self._lock:
            return self.entries.get(key)

    def put(self, key: str, choice: SceneChoice) -> None:
        with self._lock:
            self.entries[key] = choice
            if self.path:
                self.path.write_text(json.dumps({k: asdict(v) for k, v in self.entries.items()}, indent=1))


def _time_ms(fn, reps: int, stream: torch.cuda.Stream) -> float:
    fn()  # warm-up (also sizes workspaces)
    times = []
    for _ in range(reps):
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        fn()
        stop.record(stream)
        stop.synchronize()
        times.append(start.elapsed_time(stop))
    return float(np.median(times))


def tune_scene(arrays: SceneArrays, spec: runtime.TraceSpec, *, device: int = 0, sample_rays: int = 16384,
               reps: int = 3, candidates: Sequence[dict[str, Any]] = SCENE_CANDIDATES,
               cache: TuneCache | None = None, tune_stack: bool = True) -> SceneChoice:
    """Fastest traversal for one scene, then the fastest stack depth for it, timed on a sample of `spec`'s
    rays (float32, Philox)."""
    key = fingerprint(arrays)
    if cache is not None:
        hit = cache.get(key)
        if hit is not None:
            return hit
    dev = runtime.require_cuda(device)
    stream = torch.cuda.current_stream(dev)
    sample = replace(spec, num_rays=max(1, min(int(spec.num_rays), int(sample_rays))), precision="float32",
                     rng="philox", render_ambisonics=False, stack_entries=0)
    best: SceneChoice | None = None
    best_need = 0
    for cand in candidates:
        scene = runtime.DeviceScene(arrays, device=dev.index, **cand)
        try:
            if scene.traversal != cand["traversal"]:
                continue   # nothing for a BVH to hold (no boxes, or only horizontal surfaces)
            if scene.traversal != "scan" and scene.bvh_width != int(cand.get("bvh_width", 2) or 2):
                continue   # a four-wide tree that would need too deep a stack stays binary
            buffers = runtime.TraceBuffers.allocate(scene.num_surfaces, int(sample.num_bins), dev)
            ms = _time_ms(lambda: runtime.trace(scene, sample, buffers, stream=stream), reps, stream)
            need = scene.bvh_stack_need if scene.bvh_nodes > 0 else 0
        finally:
            scene.close()
        if best is None or ms < best.ms:
            best = SceneChoice(cand["traversal"], int(cand.get("bvh_leaf", 0)), ms, int(cand.get("bvh_width", 0)))
            best_need = need
    assert best is not None
    if tune_stack and best_need > 0:
        scene = runtime.DeviceScene(arrays, device=dev.index, **best.options())
        try:
            buffers = runtime.TraceBuffers.allocate(scene.num_surfaces, int(sample.num_bins), dev)
            timed = []
            for entries in stack_candidates(scene.bvh_stack_need):
                run = replace(sample, stack_entries=entries)
                timed.append((entries, _time_ms(lambda: runtime.trace(scene, run, buffers, stream=stream), reps,
                                                stream)))
        finally:
            scene.close()
        entries, ms = min(timed, key=lambda t: (t[1], t[0]))
        best = replace(best, ms=ms, stack_entries=entries, stack_ms=tuple(timed))
    if cache is not None:
        cache.put(key, best)
    return best


def tune_launch(jobs: Sequence[tuple[runtime.DeviceScene, runtime.TraceSpec]], *, device: int = 0,
                ray_fraction: float = 1.0 / 16.0, reps: int = 2,
                candidates: Sequence[dict[str, int]] = LAUNCH_CANDIDATES, tune_stack: bool = True) -> LaunchChoice:
    """Fastest (block_size, chunk_rays), then stack depth, for one persistent launch over `jobs`.

    Timed on the same jobs with their ray budgets scaled by `ray_fraction`, so
    the mix of scenes, bounce limits and relative job sizes is the real one.
    """
    dev = runtime.require_cuda(device)
    stream = torch.cuda.current_stream(dev)
    scaled = [(scene, replace(spec, num_rays=max(1, int(round(spec.num_rays * ray_fraction)))),
               runtime.TraceBuffers.allocate(scene.num_surfaces, int(spec.num_bins), dev)) for scene, spec in jobs]
    workspace = runtime.BatchWorkspace(dev)
    best: LaunchChoice | None = None
    for cand in candidates:
        ms = _time_ms(lambda: runtime.trace_batch(scaled, workspace, block_size=cand["block_size"],
                                                  chunk_rays=cand["chunk_rays"], stream=stream), reps, stream)
        if best is None or ms < best.ms:
            best = LaunchChoice(cand["block_size"], cand["chunk_rays"], ms)
    assert best is not None
    need = max((scene.bvh_stack_need for scene, _ in jobs if scene.bvh_nodes > 0), default=0)
    if tune_stack and need > 0:
        shape = best
        timed = []
        for entries in stack_candidates(need):
            timed.append((entries, _time_ms(lambda: runtime.trace_batch(
                scaled, workspace, block_size=shape.block_size, chunk_rays=shape.chunk_rays, stack_entries=entries,
                stream=stream), reps, stream)))
        entries, ms = min(timed, key=lambda t: (t[1], t[0]))
        best = replace(shape, ms=ms, stack_entries=entries, stack_ms=tuple(timed))
    return best
