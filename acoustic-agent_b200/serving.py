"""Continuous-batching RIR server on one GPU.

The reference answers one request at a time: ``AcousticAgent.run`` and the
batch helpers (api.py:477-639, batch.py:139-185, engine.py:64-73) trace each
(source, channel) job to completion before the next starts.  This loop keeps
the GPU fed while requests arrive:

* **admission by free HBM** -- a request is admitted when its footprint (its
  scene, unless already resident, plus the trace outputs, echograms, band IRs
  and synthesis workspace of its jobs) fits the device budget that the
  in-flight batches leave, and a launch slot is free; a request that cannot
  fit even on an idle device is rejected (its result carries the reason) and
  the others are served;
* **continuous batching** -- every admitted request that waits is folded into
  the next batch: ONE persistent tracer launch over all their jobs (any mix of
  scene sizes, ray budgets and lengths) plus one ragged synthesis and the
  copy of the band IRs to pinned host memory.  Up to ``max_inflight`` batches
  run on their own CUDA streams at once, so a batch formed from requests that
  arrived while others were on the GPU starts as soon as a slot frees, and its
  blocks fill the SMs the previous launch's tail leaves idle;
* **resident scenes** -- scenes (BVH, surface records, material table) stay on
  the device in an LRU cache keyed by their surface arrays and are reused by
  later requests and by every keyframe of a moving source; only idle scenes
  are evicted, and only when an admission needs their memory.

Every job's result is independent of the batch it ran in: rays are keyed by
(seed, stream key, ray index) with the stream key derived from the request
identity, echogram bins are exact fixed-point sums, and synthesis noise is
keyed by the job's own seed.  ``tests/test_gpu_serving.py`` checks that each
served result equals the same request rendered alone.
"""
from __future__ import annotations

import math
import time
from collections import OrderedDict, deque
from dataclasses import dataclass, field
from typing import Any, Sequence

import numpy as np
import torch

from acoustic_agent_b200 import _lib, autotune, bands, rng, runtime
from acoustic_agent_b200.batching import NUM_BANDS
from acoustic_agent_b200.directivity import source_directivity, source_forward
from acoustic_agent_b200.scene import SceneArrays, compile_scene
from acoustic_agent_b200.workloads import Workload


@dataclass
class Request:
    """One RIR solve: a scene, one source (or keyframes of a moving source) and its receiver channels."""

    id: int
    workload: Workload
    sources: list[tuple[float, float, float]]
    arrival_s: float = 0.0
    moving: bool = False

    @property
    def num_rirs(self) -> int:
        return len(self.sources) * len(self.workload.listeners)


@dataclass
class Result:
    request: Request
    band_irs: list[np.ndarray]          # [6, N] float32 per (keyframe, channel), keyframe-major
    ray_bounces: int
    admitted_s: float
    done_s: float
    error: str | None = None            # set when the request was rejected (its band_irs are empty)
    traced_s: float | None = None       # when its last job's trace was complete (continuous server)

    @property
    def latency_s(self) -> float:
        return self.done_s - self.request.arrival_s


@dataclass
class Report:
    results: list[Result]
    makespan_s: float
    rirs: int
    ray_bounces: int
    batches: int
    max_inflight_seen: int
    scene_hits: int
    scene_misses: int
    evictions: int
    peak_bytes: int = 0                 # device bytes held by resident scenes and in-flight batches, at most

    @property
    def rejected(self) -> list[Result]:
        return [r for r in self.results if r.error is not None]

    def latency_ms(self, q: float) -> float:
        lat = np.array([r.latency_s for r in self.results if r.error is None]) * 1e3
        return float(np.percentile(lat, q)) if lat.size else float("nan")

    def phase_ms(self, q: float) -> dict[str, float]:
        """Percentile `q` of arrival -> admitted, admitted -> traced and traced -> band IRs on the host."""
        served = [r for r in self.results if r.error is None and r.traced_s is not None]
        if not served:
            return {}
        parts = {"queued": [r.admitted_s - r.request.arrival_s for r in served],
                 "traced": [r.traced_s - r.admitted_s for r in served],
                 "synthesized": [r.done_s - r.traced_s for r in served]}
        return {k: float(np.percentile(np.array(v) * 1e3, q)) for k, v in parts.items()}

    def summary(self) -> dict[str, Any]:
        return {
            "requests": len(self.results), "rejected": len(self.rejected), "rirs": self.rirs,
            "makespan_s": self.makespan_s, "peak_device_bytes": self.peak_bytes,
            "rirs_per_s": self.rirs / self.makespan_s if self.makespan_s > 0 else float("nan"),
            "ray_bounces_per_s": self.ray_bounces / self.makespan_s if self.makespan_s > 0 else float("nan"),
            "p50_ms": self.latency_ms(50), "p99_ms": self.latency_ms(99), "batches": self.batches,
            "max_inflight": self.max_inflight_seen, "scene_cache": {"hits": self.scene_hits,
                                                                    "misses": self.scene_misses,
                                                                    "evictions": self.evictions},
        }


def request_jobs(req: Request, precision: str = "float32") -> list[runtime.TraceSpec]:
    """TraceSpecs of a request, keyframe-major then channel; keyed by the request's identity."""
    w = req.workload
    cfg = w.config
    emitter = source_directivity(w.source_model)
    forward = source_forward(emitter)
    specs = []
    for k, src in enumerate(req.sources):
        key = rng.stream_key(w.name, req.id, k)
        for lst in w.listeners:
            src_a = np.asarray(src, dtype=float)
            lst_a = np.asarray(lst, dtype=float)
            specs.append(runtime.TraceSpec(
                source=src_a, listener=lst_a, source_forward=forward, num_rays=max(1, cfg.rt_num_rays),
                num_bounces=cfg.rt_num_bounces, num_bins=cfg.num_bins, bin_duration=cfg.rt_bin_duration_s,
                speed_of_sound=cfg.c, max_path_length=cfg.max_path_length,
                direct_delay=float(np.linalg.norm(src_a - lst_a)) / cfg.c,
                listener_radius=cfg.rt_listener_radius, source_radius=cfg.rt_source_radius,
                irradiance_min_distance=cfg.rt_irradiance_min_distance,
                specular_exponent=cfg.rt_specular_exponent, dipole_weight=float(emitter["dipole_weight"]),
                dipole_power=float(emitter["dipole_power"]), use_bvh=cfg.intersection_backend == "bvh",
                render_ambisonics=False, precision=precision, rng="philox", seed=cfg.seed, stream_key=key))
    return specs


def job_bytes(spec: runtime.TraceSpec, fs: int, num_surfaces: int, *, late_tail: bool = False) -> int:
    """Device bytes one job holds while in flight (outputs, echogram, band IRs, synthesis rows, and with
    `late_tail` the float64 copy, hybrid outputs, FDN impulse, band split and delay lines)."""
    bins = int(spec.num_bins)
    n = bins * bands.samples_per_bin(spec.bin_duration, fs)
    trace_out = 8 * (NUM_BANDS * bins * 2 + 4 * num_surfaces + 8) + 4 * (NUM_BANDS * bins + num_surfaces)
    synth = 8 * (2 * NUM_BANDS * bins + NUM_BANDS * n)
    tail = (8 + 4 + 4 + 4) * NUM_BANDS * n + 8 * n + (1 << 20) if late_tail else 0
    return trace_out + 4 * NUM_BANDS * n + synth + tail + 1024


class SceneCache:
    """Resident device scenes keyed by surface-array fingerprint, LRU over idle entries."""

    def __init__(self, device: int, *, tune: bool = True, tune_cache: autotune.TuneCache | None = None) -> None:
        self.device = device
        self.tune = tune
        self.tune_cache = tune_cache or autotune.TuneCache()
        self.entries: OrderedDict[str, runtime.DeviceScene] = OrderedDict()
        self.refs: dict[str, int] = {}
        # compiled arrays by the identity of the workload's spec dict; the spec is kept with its
        # entry, so an id reused by a later object can never alias an earlier scene.  Entries go
        # when their scene is evicted, and the map keeps at most `max_arrays` (least recent out).
        self.arrays: OrderedDict[int, tuple[Any, str, SceneArrays]] = OrderedDict()
        self.max_arrays = 1024
        self.hits = self.misses = self.evictions = 0

    def resident_bytes(self) -> int:
        return sum(s.device_bytes for s in self.entries.values())

    def key_of(self, w: Workload) -> tuple[str, SceneArrays]:
        entry = self.arrays.get(id(w.spec))
        if entry is None or entry[0] is not w.spec:
            arrays = compile_scene(w.spec)
            entry = (w.spec, autotune.fingerprint(arrays), arrays)
            self.arrays[id(w.spec)] = entry
            while len(self.arrays) > self.max_arrays:
                self.arrays.popitem(last=False)
        else:
            self.arrays.move_to_end(id(w.spec))
        return entry[1], entry[2]

    def is_resident(self, w: Workload) -> bool:
        return self.key_of(w)[0] in self.entries

    def acquire(self, w: Workload, sample: runtime.TraceSpec) -> runtime.DeviceScene:
        key, arrays = self.key_of(w)
        scene = self.entries.get(key)
        if scene is None:
            self.misses += 1
            options: dict[str, Any] = {}
            if self.tune:
                options = autotune.tune_scene(arrays, sample, device=self.device, cache=self.tune_cache).options()
            scene = runtime.DeviceScene(arrays, device=self.device, **options)
            self.entries[key] = scene
        else:
            self.hits += 1
            self.entries.move_to_end(key)
        self.refs[key] = self.refs.get(key, 0) + 1
        return scene

    def release(self, w: Workload) -> None:
        key = self.key_of(w)[0]
        self.refs[key] -= 1

    def evict_idle(self, need: int) -> int:
        """Free idle scenes, least recently used first, until `need` bytes are freed; returns bytes freed."""
        freed = 0
        for key in list(self.entries):
            if freed >= need:
                break
            if self.refs.get(key, 0) > 0:
                continue
            scene = self.entries.pop(key)
            freed += scene.device_bytes
            scene.close()
            self.evictions += 1
            for spec_id in [i for i, e in self.arrays.items() if e[1] == key]:
                del self.arrays[spec_id]
        return freed

    def close(self) -> None:
        for scene in self.entries.values():
            scene.close()
        self.entries.clear()


@dataclass
class _Batch:
    requests: list[Request]
    specs: list[list[runtime.TraceSpec]]
    stream: torch.cuda.Stream
    done: torch.cuda.Event
    host: torch.Tensor
    lengths: list[list[int]]
    buffers: list[runtime.TraceBuffers]
    bytes: int
    admitted_s: float
    keep: list[Any] = field(default_factory=list)
    # late tails: the band IRs and host echograms wait for the tail phase, which replaces `done`
    ir_store: torch.Tensor | None = None
    echograms: list[torch.Tensor] | None = None
    tails_pending: bool = False


class Server:
    """Continuous batching over one GPU (see the module docstring)."""

    POLICIES = ("small_first", "fifo")

    def __init__(self, device: int = 0, *, max_inflight: int = 3, hbm_budget: int | None = None,
                 max_batch_rays: int = 400_000_000, tune: bool = True, block_size: int = 0,
                 chunk_rays: int = 0, policy: str = "small_first", starve_s: float = 1.0,
                 late_tail: bool = False, transition_s: float = 1.0, overlap_fraction: float = 0.25,
                 trace_blocks_per_sm: int = 2) -> None:
        """`policy` orders the waiting requests when a batch is formed: "fifo" by arrival, or
        "small_first" by ray count, except that requests waiting longer than `starve_s` go first
        (in arrival order), so a stream of small requests cannot hold a large one back for ever.
        With `late_tail`, every served RIR is crossfaded into its FDN late tail as the reference's
        renderer does with late_tail=True (late_reverb.batch_late_tails, one launch pair per batch).
        `trace_blocks_per_sm` > 0 caps each batch's persistent trace grid at that many blocks per SM
        (0: the library's choice, three).  Two leave room for other batches' synthesis recursion beside a
        trace, whose one-warp blocks do not fit next to three trace blocks' registers."""
        if policy not in self.POLICIES:
            raise ValueError(f"policy must be one of {self.POLICIES}")
        self.policy = policy
        self.starve_s = float(starve_s)
        self.dev = runtime.require_cuda(device)
        self.max_inflight = max(1, int(max_inflight))
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info(self.dev)
            hbm_budget = int(free * 0.8)
        self.budget = int(hbm_budget)
        self.max_batch_rays = int(max_batch_rays)
        self.scenes = SceneCache(self.dev.index, tune=tune)
        self.block_size = block_size
        self.chunk_rays = chunk_rays
        self.streams = [torch.cuda.Stream(self.dev) for _ in range(self.max_inflight)]
        self.in_use = 0     # bytes held by in-flight batches
        self.late_tail = bool(late_tail)
        self.transition_s = float(transition_s)
        self.overlap_fraction = float(overlap_fraction)
        self._late: dict[int, Any] = {}
        sms = torch.cuda.get_device_properties(self.dev).multi_processor_count
        self.trace_grid = max(0, int(trace_blocks_per_sm)) * sms

    # ---- footprint and admission
    def footprint(self, req: Request, specs: Sequence[runtime.TraceSpec]) -> int:
        scene = 0 if self.scenes.is_resident(req.workload) else self._scene_estimate(req.workload)
        surfaces = self.scenes.key_of(req.workload)[1].num_surfaces
        return scene + sum(job_bytes(s, req.workload.config.fs, surfaces, late_tail=self.late_tail) for s in specs)

    def _scene_estimate(self, w: Workload) -> int:
        arrays = self.scenes.key_of(w)[1]
        return 4096 + 512 * arrays.num_surfaces + 64 * len(arrays.arrays["corners"])

    def _fits(self, need: int) -> bool:
        if self.scenes.resident_bytes() + self.in_use + need <= self.budget:
            return True
        over = self.scenes.resident_bytes() + self.in_use + need - self.budget
        self.scenes.evict_idle(over)
        return self.scenes.resident_bytes() + self.in_use + need <= self.budget

    # ---- one batch: trace + synthesis + copy to pinned host memory, all on the batch's stream
    def _launch(self, reqs: list[Request], specs: list[list[runtime.TraceSpec]], nbytes: int, now: float,
                stream: torch.cuda.Stream) -> _Batch:
        jobs, synth, lengths, keep = [], [], [], []
        buffers: list[runtime.TraceBuffers] = []
        total = sum(4 * NUM_BANDS * s.num_bins * bands.samples_per_bin(s.bin_duration, r.workload.config.fs)
                    for r, ss in zip(reqs, specs) for s in ss) // 4
        with torch.cuda.stream(stream):
            ir_store = torch.empty(max(1, total), dtype=torch.float32, device=self.dev)
            off = 0
            for r, ss in zip(reqs, specs):
                scene = self.scenes.acquire(r.workload, ss[0])
                fs = r.workload.config.fs
                row = []
                for s in ss:
                    b = runtime.TraceBuffers.allocate(scene.num_surfaces, s.num_bins, self.dev)
                    n = s.num_bins * bands.samples_per_bin(s.bin_duration, fs)
                    out = ir_store[off:off + NUM_BANDS * n].view(NUM_BANDS, n)
                    off += NUM_BANDS * n
                    jobs.append((scene, s, b))
                    buffers.append(b)
                    synth.append(runtime.SynthJob(b.echogram, out, fs, s.bin_duration, seed=int(s.seed) + 7,
                                                  direct_delay=max(0.0, float(s.direct_delay)),
                                                  speed_of_sound=s.speed_of_sound))
                    row.append(n)
                lengths.append(row)
            trace_ws = runtime.BatchWorkspace(self.dev)
            synth_ws = runtime.SynthBatchWorkspace(self.dev)
            runtime.trace_batch(jobs, trace_ws, block_size=self.block_size, chunk_rays=self.chunk_rays,
                                grid_blocks=self.trace_grid, stream=stream)
            runtime.synthesize_batch(synth, synth_ws, stream=stream)
            host = torch.empty(ir_store.shape, dtype=torch.float32, pin_memory=True)
            echograms = None
            if self.late_tail:   # the tails need the echograms on the host first
                echograms = []
                for b in buffers:
                    e = torch.empty(b.echogram.shape, dtype=torch.float32, pin_memory=True)
                    e.copy_(b.echogram, non_blocking=True)
                    echograms.append(e)
            else:
                host.copy_(ir_store, non_blocking=True)
            done = torch.cuda.Event()
            done.record(stream)
        keep.extend([ir_store, trace_ws, synth_ws, synth])
        return _Batch(reqs, specs, stream, done, host, lengths, buffers, nbytes, now, keep, ir_store=ir_store,
                      echograms=echograms, tails_pending=self.late_tail)

    def _start_tails(self, batch: _Batch) -> None:
        """Second phase of a late-tail batch: RT60s from the echograms, the FDN tails of every job in one
        launch pair on the batch's stream, and the hybrid band IRs to pinned host memory."""
        from acoustic_agent_b200 import late_reverb
        # one renderer (and so one device workspace) per stream: batches in flight on other streams
        # must not share delay lines or band-split scratch with this one
        key = id(batch.stream)
        if key not in self._late:
            self._late[key] = late_reverb.LateReverbRenderer(self.dev)
        irs, fs, seeds, bins, speeds = [], [], [], [], []
        off = 0
        for req, ss, row in zip(batch.requests, batch.specs, batch.lengths):
            for s, n in zip(ss, row):
                irs.append(batch.ir_store[off:off + NUM_BANDS * n].view(NUM_BANDS, n))
                off += NUM_BANDS * n
                fs.append(req.workload.config.fs)
                seeds.append(int(s.seed))
                bins.append(s.bin_duration)
                speeds.append(s.speed_of_sound)
        tails = late_reverb.batch_late_tails(self._late[key], irs, [e.numpy() for e in batch.echograms], fs, seeds,
                                             bins, speeds, transition_s=self.transition_s,
                                             overlap_fraction=self.overlap_fraction, stream=batch.stream)
        with torch.cuda.stream(batch.stream):
            batch.host.copy_(tails.out, non_blocking=True)
            done = torch.cuda.Event()
            done.record(batch.stream)
        batch.keep.append(tails)
        batch.done = done
        batch.tails_pending = False

    def _finish(self, batch: _Batch, now: float) -> list[Result]:
        host = batch.host.numpy()
        out, off, k = [], 0, 0
        for req, row in zip(batch.requests, batch.lengths):
            irs = []
            rb = 0
            for n in row:
                irs.append(host[off:off + NUM_BANDS * n].reshape(NUM_BANDS, n).copy())
                off += NUM_BANDS * n
                rb += int(batch.buffers[k].counters[2].item())
                k += 1
            out.append(Result(req, irs, rb, batch.admitted_s, now))
            self.scenes.release(req.workload)
        self.in_use -= batch.bytes
        return out

    def _order(self, waiting, now: float) -> list[tuple[Request, list[runtime.TraceSpec]]]:
        if self.policy == "fifo":
            return list(waiting)

        def key(entry):
            req, ss = entry
            if now - req.arrival_s > self.starve_s:
                return (0, req.arrival_s)
            return (1, sum(s.num_rays for s in ss), req.arrival_s)

        return sorted(waiting, key=key)

    def serve(self, requests: Sequence[Request], *, realtime: bool = True, idle_sleep_s: float = 2e-4) -> Report:
        """Run every request to completion; arrivals follow `arrival_s` (wall clock) when `realtime`."""
        pending = deque(sorted(requests, key=lambda r: r.arrival_s))
        waiting: deque[tuple[Request, list[runtime.TraceSpec]]] = deque()
        inflight: list[_Batch] = []
        results: list[Result] = []
        batches = max_seen = peak = 0
        free_streams = list(self.streams)
        t0 = time.perf_counter()
        clock = (lambda: time.perf_counter() - t0) if realtime else (lambda: float("inf"))
        while pending or waiting or inflight:
            now = clock()
            while pending and pending[0].arrival_s <= now:
                req = pending.popleft()
                waiting.append((req, request_jobs(req)))
            # completions first: they return slots and memory
            for batch in list(inflight):
                if batch.done.query() and batch.tails_pending:
                    self._start_tails(batch)
                    continue
                if batch.done.query():
                    done_at = time.perf_counter() - t0
                    results.extend(self._finish(batch, done_at))
                    inflight.remove(batch)
                    free_streams.append(batch.stream)
            # admit what fits into one new batch while a slot is free
            if waiting and free_streams:
                reqs, specs, need_total, rays = [], [], 0, 0
                for entry in self._order(waiting, time.perf_counter() - t0 if realtime else 0.0):
                    req, ss = entry
                    need = self.footprint(req, ss)
                    req_rays = sum(s.num_rays for s in ss)
                    if reqs and rays + req_rays > self.max_batch_rays:
                        break
                    if not self._fits(need_total + need):
                        if not reqs and not inflight and self.scenes.resident_bytes() + need > self.budget:
                            # cannot fit even on an idle device: reject it, keep serving the others
                            waiting.remove(entry)
                            t = time.perf_counter() - t0
                            results.append(Result(req, [], 0, t, t, error=f"needs {need} bytes of device memory; "
                                                                              f"the budget is {self.budget}"))
                            continue
                        break
                    waiting.remove(entry)
                    reqs.append(req)
                    specs.append(ss)
                    need_total += need
                    rays += req_rays
                if reqs:
                    self.in_use += need_total
                    peak = max(peak, self.in_use + self.scenes.resident_bytes())
                    stream = free_streams.pop()
                    inflight.append(self._launch(reqs, specs, need_total, time.perf_counter() - t0, stream))
                    batches += 1
                    max_seen = max(max_seen, len(inflight))
                    continue
            if not realtime and not inflight and not waiting and pending:
                continue
            if inflight or (pending and realtime):
                time.sleep(idle_sleep_s)
        served = [r for r in results if r.error is None]
        makespan = max((r.done_s for r in served), default=0.0) - min((r.request.arrival_s for r in served),
                                                                      default=0.0)
        return Report(results=sorted(results, key=lambda r: r.request.id), makespan_s=makespan,
                      rirs=sum(r.request.num_rirs for r in served),
                      ray_bounces=sum(r.ray_bounces for r in served), batches=batches, max_inflight_seen=max_seen,
                      scene_hits=self.scenes.hits, scene_misses=self.scenes.misses,
                      evictions=self.scenes.evictions, peak_bytes=peak)

    def close(self) -> None:
        self.scenes.close()


@dataclass
class _Live:
    """An admitted request of the continuous server: its jobs on the trace service, then its synthesis."""

    request: Request
    specs: list[runtime.TraceSpec]
    scene: runtime.DeviceScene
    buffers: list[runtime.TraceBuffers]
    seqs: list[int]
    remaining: set[int]
    bytes: int
    admitted_s: float
    est_ray_bounces: float
    predicted_s: float = 0.0            # admission to traced, as predicted when it was admitted
    traced_s: float | None = None       # when its last job's trace was complete
    ray_bounces: int = 0
    irs: list[torch.Tensor] = field(default_factory=list)
    keep: torch.Tensor | None = None    # the device store of its band IRs until the host copy is done
    host: torch.Tensor | None = None
    done: torch.cuda.Event | None = None


class ContinuousServer:
    """Continuous batching at kernel level on one GPU.

    One persistent trace launch (runtime.TraceService, ac_service_*) runs while requests arrive: an admitted
    request's jobs are appended to the launch's job ring at once, and its warps pick them up as they run out
    of older work, so a request never waits for a batch to form or for another batch's launch to end.  When a
    request's last job is done, its band synthesis (one ragged launch for every request that completed in the
    same poll) and the copy to pinned host memory run on a second stream beside the persistent launch, whose
    grid leaves room for them: three blocks per SM less `reserve_blocks` (16) by default, so that a few SMs
    hold two trace blocks and the synthesis warps' registers (measured: 20 % more served than two blocks on
    every SM; three on every SM starves the synthesis).

    Admission: a request is admitted when its device footprint fits the HBM budget (resident scenes plus the
    outputs of requests in flight); one that could never fit is rejected.  With `slo_s`, a request is also
    rejected at arrival when the traced work already admitted or waiting ahead of it, plus its own, would take
    longer than `slo_s` at the service's throughput (never while nothing is ahead of it); work is estimated
    from each scene's measured ray-bounces per ray, and the prediction is scaled by the running ratio of
    measured to predicted times from admission to traced: overload is shed instead of queueing without
    bound.  The throughput
    is `capacity_rb_per_s` ray-bounces/s (about the served rate under overload) until the
    server has run saturated -- at least a quarter second of work ahead -- for a second; from then on, the
    rate measured while saturated (a rate measured while the device idles between requests would understate
    it and shed work the device could take).  Requests that wait for memory are admitted in arrival order.
    Each result is the same as the request rendered alone (rays keyed by request identity, exact fixed-point
    sums, synthesis noise keyed by the job's seed).
    """

    def __init__(self, device: int = 0, *, hbm_budget: int | None = None, tune: bool = True,
                 slo_s: float | None = None, capacity_rb_per_s: float = 2.6e9, blocks_per_sm: int = 3,
                 capacity: int = 16384, idle_timeout_s: float = 0.02, chunk_rays: int = 0,
                 reserve_blocks: int = 16) -> None:
        self.dev = runtime.require_cuda(device)
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info(self.dev)
            hbm_budget = int(free * 0.8)
        self.budget = int(hbm_budget)
        self.scenes = SceneCache(self.dev.index, tune=tune)
        self.service = runtime.TraceService(self.dev.index, capacity=capacity, blocks_per_sm=blocks_per_sm,
                                            chunk_rays=chunk_rays, idle_timeout_s=idle_timeout_s,
                                            reserve_blocks=reserve_blocks)
        self.synth_stream = torch.cuda.Stream(self.dev)
        # synthesis workspaces in rotation: a workspace's staging is free once its last batch has run, and
        # waiting for that on the host would stop admission and polling while synthesis queues for SM room
        self.synth_pool: list[runtime.SynthBatchWorkspace] = []
        self.slo_s = slo_s
        self.capacity_rb_per_s = float(capacity_rb_per_s)
        self.in_use = 0
        self.bounces_per_ray = 40.0      # running estimate of ray-bounces per ray, from finished jobs
        self.scene_bounces: dict[str, float] = {}   # the same per scene (by workload name) once one finished
        # measured / predicted time from admission to traced (running mean over requests whose prediction was
        # at least a quarter second): corrects the work-over-rate prediction for what it leaves out (the
        # sharing of the device with the synthesis, the order in which warps take jobs)
        self.latency_scale = 1.0
        self._sizer = Server.__new__(Server)   # footprint arithmetic shared with the batch server
        self._sizer.scenes, self._sizer.late_tail = self.scenes, False

    def footprint(self, req: Request, specs: Sequence[runtime.TraceSpec]) -> int:
        return Server.footprint(self._sizer, req, specs)

    def _fits(self, need: int) -> bool:
        if self.scenes.resident_bytes() + self.in_use + need <= self.budget:
            return True
        if self.service.info()["running_launches"] == 0:
            # a running launch may still hold an evicted scene's lines in L1: evict only between launches
            self.scenes.evict_idle(self.scenes.resident_bytes() + self.in_use + need - self.budget)
        return self.scenes.resident_bytes() + self.in_use + need <= self.budget

    def _est_rb(self, specs: Sequence[runtime.TraceSpec], scene: str | None = None) -> float:
        per_ray = self.scene_bounces.get(scene, self.bounces_per_ray) if scene is not None else self.bounces_per_ray
        return sum(min(float(s.num_bounces), per_ray) * s.num_rays for s in specs)

    def _admit(self, req: Request, specs: list[runtime.TraceSpec], need: int, now: float) -> _Live:
        scene = self.scenes.acquire(req.workload, specs[0])
        try:
            buffers = [runtime.TraceBuffers.allocate(scene.num_surfaces, s.num_bins, self.dev) for s in specs]
            seqs = self.service.submit([(scene, s, b) for s, b in zip(specs, buffers)])
        except Exception:
            self.scenes.release(req.workload)
            raise
        self.in_use += need
        return _Live(req, specs, scene, buffers, seqs, set(seqs), need, now,
                     self._est_rb(specs, req.workload.name))

    def _synth_workspace(self, limit: int = 16) -> runtime.SynthBatchWorkspace:
        for ws in self.synth_pool:
            if ws.idle():
                return ws
        if len(self.synth_pool) < limit:
            self.synth_pool.append(runtime.SynthBatchWorkspace(self.dev))
            return self.synth_pool[-1]
        return self.synth_pool[0]   # all busy: this one waits for its last batch

    def _synthesize(self, lives: list[_Live]) -> None:
        """Band IRs of requests whose traces are done: one ragged synthesis and one host copy per request."""
        synth = []
        with torch.cuda.stream(self.synth_stream):
            for live in lives:
                fs = live.request.workload.config.fs
                lengths = [s.num_bins * bands.samples_per_bin(s.bin_duration, fs) for s in live.specs]
                store = torch.empty(NUM_BANDS * sum(lengths), dtype=torch.float32, device=self.dev)
                off = 0
                for s, b, n in zip(live.specs, live.buffers, lengths):
                    out = store[off:off + NUM_BANDS * n].view(NUM_BANDS, n)
                    off += NUM_BANDS * n
                    live.irs.append(out)
                    synth.append(runtime.SynthJob(b.echogram, out, fs, s.bin_duration, seed=int(s.seed) + 7,
                                                  direct_delay=max(0.0, float(s.direct_delay)),
                                                  speed_of_sound=s.speed_of_sound))
                live.host = torch.empty(store.shape, dtype=torch.float32, pin_memory=True)
                live.keep = store
            runtime.synthesize_batch(synth, self._synth_workspace(), stream=self.synth_stream)
            for live in lives:
                live.host.copy_(live.keep, non_blocking=True)
                live.done = torch.cuda.Event()
                live.done.record(self.synth_stream)

    def serve(self, requests: Sequence[Request], *, realtime: bool = True, idle_sleep_s: float = 2e-4) -> Report:
        """Run every request to completion (or rejection); arrivals follow `arrival_s` when `realtime`."""
        pending = deque(sorted(requests, key=lambda r: r.arrival_s))
        waiting: deque[tuple[Request, list[runtime.TraceSpec], int]] = deque()
        tracing: dict[int, _Live] = {}      # sequence number -> its request
        synthesizing: list[_Live] = []
        results: list[Result] = []
        outstanding_rb = 0.0               # estimated ray-bounces admitted and not yet traced
        sat_rb = 0.0                       # ray-bounces finished, and seconds spent, while saturated
        sat_s = 0.0
        peak = 0
        t0 = time.perf_counter()
        tick = t0
        clock = (lambda: time.perf_counter() - t0) if realtime else (lambda: float("inf"))
        max_live = live_now = 0            # requests on the GPU (tracing or synthesizing), most at once
        while pending or waiting or tracing or synthesizing:
            now = clock()
            saturated = outstanding_rb >= 0.25 * self.capacity_rb_per_s
            rate = sat_rb / sat_s if sat_s >= 1.0 and sat_rb > 0 else self.capacity_rb_per_s
            # arrivals: reject what can never fit, or what the admitted work would make miss its SLO
            while pending and pending[0].arrival_s <= now:
                req = pending.popleft()
                specs = request_jobs(req)
                need = self.footprint(req, specs)
                t = time.perf_counter() - t0
                if need > self.budget:   # could not fit even on an idle device
                    results.append(Result(req, [], 0, t, t, error=f"needs {need} bytes of device memory; "
                                                                   f"the budget is {self.budget}"))
                    continue
                if self.slo_s is not None:
                    # its latency is about the work ahead plus its own (the ring is served roughly in order),
                    # scaled by the measured / predicted ratio; a request is never shed while nothing is ahead
                    ahead = outstanding_rb + sum(self._est_rb(w[1], w[0].workload.name) for w in waiting)
                    own = self._est_rb(specs, req.workload.name)
                    wait = self.latency_scale * (ahead + own) / rate if ahead > 0 else 0.0
                    if wait > self.slo_s:
                        results.append(Result(req, [], 0, t, t, error=f"overloaded: about {wait:.2f} s of traced work "
                                                                       f"(ahead of it and its own) exceeds the "
                                                                       f"{self.slo_s:g} s limit"))
                        continue
                waiting.append((req, specs, need))
            # admission in arrival order while memory allows; the ring may ask us to come back later
            while waiting:
                req, specs, need = waiting[0]
                if not self._fits(need):
                    break
                try:
                    live = self._admit(req, specs, need, time.perf_counter() - t0)
                except _lib.BackendError as exc:
                    if exc.code != _lib.AC_ERR_CAPACITY:
                        raise
                    break   # the job ring is full: admit it after the next completions
                waiting.popleft()
                for seq in live.seqs:
                    tracing[seq] = live
                live.predicted_s = (outstanding_rb + live.est_ray_bounces) / rate
                outstanding_rb += live.est_ray_bounces
                live_now += 1
                peak = max(peak, self.in_use + self.scenes.resident_bytes())
            # traces that finished: their requests go to synthesis once all their jobs are done
            finished = []
            for seq in self.service.poll():
                live = tracing.pop(seq)
                live.remaining.discard(seq)
                if not live.remaining:
                    finished.append(live)
            if finished:
                for live in finished:
                    rb = int(torch.stack([b.counters[2] for b in live.buffers]).sum().item())   # one host read
                    rays = sum(s.num_rays for s in live.specs)
                    self.bounces_per_ray = 0.8 * self.bounces_per_ray + 0.2 * rb / max(rays, 1)
                    name = live.request.workload.name
                    seen = self.scene_bounces.get(name)
                    self.scene_bounces[name] = rb / max(rays, 1) if seen is None else 0.7 * seen + 0.3 * rb / max(rays, 1)
                    if saturated:
                        sat_rb += rb
                    live.traced_s = time.perf_counter() - t0
                    if live.predicted_s >= 0.25:
                        measured = live.traced_s - live.admitted_s
                        sample = min(4.0, max(0.5, measured / live.predicted_s))
                        self.latency_scale = 0.9 * self.latency_scale + 0.1 * sample
                    outstanding_rb -= live.est_ray_bounces
                    live.ray_bounces = rb
                self._synthesize(finished)
                synthesizing.extend(finished)
            for live in list(synthesizing):
                if live.done is not None and live.done.query():
                    synthesizing.remove(live)
                    host = live.host.numpy()
                    irs, off = [], 0
                    for ir in live.irs:
                        irs.append(host[off:off + ir.numel()].reshape(ir.shape).copy())
                        off += ir.numel()
                    results.append(Result(live.request, irs, live.ray_bounces, live.admitted_s,
                                          time.perf_counter() - t0, traced_s=live.traced_s))
                    self.scenes.release(live.request.workload)
                    self.in_use -= live.bytes
                    live_now -= 1
            max_live = max(max_live, live_now)
            nowp = time.perf_counter()
            if saturated:
                sat_s += nowp - tick
            tick = nowp
            if not realtime and not tracing and not waiting and not synthesizing and pending:
                continue
            if tracing or synthesizing or (pending and realtime):
                time.sleep(idle_sleep_s)
        served = [r for r in results if r.error is None]
        makespan = max((r.done_s for r in served), default=0.0) - min((r.request.arrival_s for r in served),
                                                                      default=0.0)
        info = self.service.info()
        return Report(results=sorted(results, key=lambda r: r.request.id), makespan_s=makespan,
                      rirs=sum(r.request.num_rirs for r in served), ray_bounces=sum(r.ray_bounces for r in served),
                      batches=int(info["launches"]), max_inflight_seen=max_live, scene_hits=self.scenes.hits,
                      scene_misses=self.scenes.misses, evictions=self.scenes.evictions, peak_bytes=peak)

    def close(self) -> None:
        self.service.close()
        self.scenes.close()


def requests_from_stream(stream: Sequence[dict[str, Any]]) -> list[Request]:
    """Requests from workloads.request_stream entries."""
    return [Request(k, e["workload"], list(e["sources"]), float(e["arrival_s"]), bool(e.get("moving", False)))
            for k, e in enumerate(stream)]


def render_alone(req: Request, device: int = 0, *, late_tail: bool = False) -> list[np.ndarray]:
    """The same request rendered by itself (one batch, nothing else on the GPU)."""
    server = Server(device, max_inflight=1, tune=False, late_tail=late_tail)
    try:
        report = server.serve([Request(req.id, req.workload, req.sources, 0.0, req.moving)], realtime=False)
    finally:
        server.close()
    return report.results[0].band_irs
