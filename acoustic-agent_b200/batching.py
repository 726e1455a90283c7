"""Batched RIR rendering: many (scene, source, channel) jobs per launch.

Replaces the per-job loops of Acoustic Agent (engine.py:64-73 channel loop,
api.py:477-639 run_batch / run_sources / run_many, batch.py:139-185
simulate_batch), which run one full trace per job, by:

1. one persistent tracer launch over every job (``ac_trace_batch``): lanes
   pull (job, ray) work items from a shared counter, so jobs of any size
   share the GPU without per-job launch or tail costs;
2. one ragged synthesis over every job (``ac_synthesize_batch``: three
   launches whatever the mix of lengths and sample rates);
3. optionally, both captured once as a CUDA graph and replayed.

Per-job results are identical to running each job alone (integer echogram
bins), which the tests check.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Any, Iterable, Sequence

import numpy as np
import torch

from acoustic_agent_b200 import bands, rng, runtime
from acoustic_agent_b200.directivity import source_directivity, source_forward
from acoustic_agent_b200.scene import SceneArrays, compile_scene
from acoustic_agent_b200.workloads import TraceConfig, Workload

NUM_BANDS = 6


@dataclass
class Job:
    scene_index: int
    spec: runtime.TraceSpec
    fs: int
    workload: int
    source: int
    channel: int


@dataclass
class Plan:
    """Device state for a fixed set of jobs, reusable across steps."""

    jobs: list[Job]
    scenes: list[runtime.DeviceScene]
    buffers: list[runtime.TraceBuffers]
    echo_store: torch.Tensor            # every job's float32 [6, bins] echogram, back to back
    ir_store: torch.Tensor              # every job's float32 [6, N] band IRs, back to back
    irs: list[torch.Tensor]             # per job: its [6, N] view of ir_store
    synth_jobs: Any                     # ac_synth_job array over all jobs
    synth_config: Any                   # ac_synth_batch_config (sample rates + crossover tables)
    workspace: runtime.BatchWorkspace
    synth_workspace: runtime.SynthBatchWorkspace
    graph: torch.cuda.CUDAGraph | None = None
    # capture(split=True): `graph` holds the trace alone and `synth_graph` the synthesis, replayed back to
    # back on one stream, so that events recorded between the two replays time the trace live
    synth_graph: torch.cuda.CUDAGraph | None = None
    keepalive: list[Any] = field(default_factory=list)
    # pipelined steps (launch_pipelined): a copy of the previous step's echograms and its synthesis jobs
    echo_prev: torch.Tensor | None = None
    synth_jobs_prev: Any = None
    pipe_graph: torch.cuda.CUDAGraph | None = None
    # recorded after every replay of either graph; the plan's scenes wait for it before they are destroyed
    replayed: torch.cuda.Event | None = None

    @property
    def num_rirs(self) -> int:
        return len(self.jobs)


def workload_jobs(workloads: Sequence[Workload], *, precision: str = "float32", rng_mode: str = "philox"
                  ) -> tuple[list[dict[str, Any]], list[Job]]:
    """Expand workloads into one job per (source, channel); returns (scene specs, jobs)."""
    specs: list[dict[str, Any]] = []
    jobs: list[Job] = []
    for w_index, w in enumerate(workloads):
        specs.append(w.spec)
        cfg: TraceConfig = w.config
        emitter = source_directivity(w.source_model)
        forward = source_forward(emitter)
        key = rng.stream_key(w.name, w_index)
        for s_index, src in enumerate(w.sources):
            for c_index, lst in enumerate(w.listeners):
                src_a = np.asarray(src, dtype=float)
                lst_a = np.asarray(lst, dtype=float)
                spec = runtime.TraceSpec(
                    source=src_a, listener=lst_a, source_forward=forward, num_rays=max(1, cfg.rt_num_rays),
                    num_bounces=cfg.rt_num_bounces, num_bins=cfg.num_bins, bin_duration=cfg.rt_bin_duration_s,
                    speed_of_sound=cfg.c, max_path_length=cfg.max_path_length,
                    direct_delay=float(np.linalg.norm(src_a - lst_a)) / cfg.c,
                    listener_radius=cfg.rt_listener_radius, source_radius=cfg.rt_source_radius,
                    irradiance_min_distance=cfg.rt_irradiance_min_distance,
                    specular_exponent=cfg.rt_specular_exponent, dipole_weight=float(emitter["dipole_weight"]),
                    dipole_power=float(emitter["dipole_power"]), use_bvh=cfg.intersection_backend == "bvh",
                    render_ambisonics=False, precision=precision, rng=rng_mode, seed=cfg.seed,
                    stream_key=key)
                jobs.append(Job(w_index, spec, cfg.fs, w_index, s_index, c_index))
    return specs, jobs


class RIRRenderer:
    """Batched tracer + synthesis on one GPU."""

    def __init__(self, device: int = 0, *, block_size: int = 0, grid_blocks: int = 0, chunk_rays: int = 0,
                 stack_entries: int | None = None) -> None:
        self.device = runtime.require_cuda(device)
        self.block_size = block_size
        self.grid_blocks = grid_blocks
        self.chunk_rays = chunk_rays
        self.stack_entries = stack_entries   # None: the largest of the plan's scenes' choices
        # eager plans share one pair of staged workspaces; a captured plan gets its own
        self._trace_ws = runtime.BatchWorkspace(self.device)
        self._synth_ws = runtime.SynthBatchWorkspace(self.device)

    def plan(self, scenes: Sequence[SceneArrays | dict[str, Any] | runtime.DeviceScene], jobs: Sequence[Job], *,
             scene_options: Sequence[dict[str, Any]] | None = None) -> Plan:
        """Upload scenes (unless already resident) and lay out every job's outputs.

        `scene_options` (one dict per scene, e.g. from autotune.tune_scene)
        chooses each uploaded scene's traversal; results do not depend on it.
        """
        opts = list(scene_options) if scene_options is not None else [{}] * len(scenes)
        device_scenes = [s if isinstance(s, runtime.DeviceScene) else
                         runtime.DeviceScene(s if isinstance(s, SceneArrays) else compile_scene(s),
                                             device=self.device.index, **o)
                         for s, o in zip(scenes, opts)]
        buffers = [runtime.TraceBuffers.allocate(device_scenes[j.scene_index].num_surfaces, j.spec.num_bins,
                                                 self.device, echogram=False) for j in jobs]
        bins = [int(j.spec.num_bins) for j in jobs]
        lengths = [b * bands.samples_per_bin(j.spec.bin_duration, j.fs) for b, j in zip(bins, jobs)]
        echo_store = torch.zeros(NUM_BANDS * sum(bins), dtype=torch.float32, device=self.device)
        ir_store = torch.empty(NUM_BANDS * sum(lengths), dtype=torch.float32, device=self.device)
        irs, synth = [], []
        e_off = i_off = 0
        for k, j in enumerate(jobs):
            # each job's float32 echogram is written by the tracer straight into the synthesis input
            buffers[k].echogram = echo_store[e_off:e_off + NUM_BANDS * bins[k]].view(NUM_BANDS, bins[k])
            irs.append(ir_store[i_off:i_off + NUM_BANDS * lengths[k]].view(NUM_BANDS, lengths[k]))
            e_off += NUM_BANDS * bins[k]
            i_off += NUM_BANDS * lengths[k]
            synth.append(runtime.SynthJob(buffers[k].echogram, irs[k], j.fs, j.spec.bin_duration,
                                          seed=int(j.spec.seed) + 7, direct_delay=max(0.0, float(j.spec.direct_delay)),
                                          speed_of_sound=j.spec.speed_of_sound))
        config = runtime.synth_batch_config([j.fs for j in jobs] or [16000])
        synth_jobs = runtime.synth_job_array(synth, config)
        return Plan(list(jobs), device_scenes, buffers, echo_store, ir_store, irs, synth_jobs, config,
                    self._trace_ws, self._synth_ws)

    def launch(self, plan: Plan, stream: torch.cuda.Stream | None = None,
               trace_events: tuple[torch.cuda.Event, torch.cuda.Event] | None = None) -> None:
        """Enqueue trace + synthesis of every job (asynchronous).

        `trace_events` (a pair of timing events) are recorded around the trace
        alone; with a captured plan that needs ``capture(plan, split=True)``.
        """
        if plan.graph is not None:
            current = torch.cuda.current_stream(self.device)
            if trace_events is not None and plan.synth_graph is None:
                raise ValueError("timing the trace of a captured plan needs capture(plan, split=True)")
            if trace_events is not None:
                trace_events[0].record(current)
            plan.graph.replay()
            if trace_events is not None:
                trace_events[1].record(current)
            if plan.synth_graph is not None:
                plan.synth_graph.replay()
            plan.replayed.record(current)
            return
        self._enqueue(plan, stream, trace_events)

    def _enqueue(self, plan: Plan, stream: torch.cuda.Stream | None,
                 trace_events: tuple[torch.cuda.Event, torch.cuda.Event] | None = None, *,
                 trace: bool = True, synth: bool = True) -> None:
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        if trace:
            if trace_events is not None:
                trace_events[0].record(s)
            runtime.trace_batch([(plan.scenes[j.scene_index], j.spec, b) for j, b in zip(plan.jobs, plan.buffers)],
                                plan.workspace, block_size=self.block_size, grid_blocks=self.grid_blocks,
                                chunk_rays=self.chunk_rays, stack_entries=self.stack_entries, stream=stream)
            if trace_events is not None:
                trace_events[1].record(s)
        if synth:
            runtime.synthesize_batch((plan.synth_jobs, len(plan.jobs), plan.synth_config), plan.synth_workspace,
                                     stream=stream)

    def capture(self, plan: Plan, *, split: bool = False) -> None:
        """Record the launch sequence once as a CUDA graph (the job table is staged in pinned memory).

        With `split`, the trace and the synthesis are two graphs replayed back to back.
        """
        plan.workspace = runtime.BatchWorkspace(self.device)
        plan.synth_workspace = runtime.SynthBatchWorkspace(self.device)
        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(side):
            self._enqueue(plan, side)   # warm-up: sizes workspaces, fills caches
        side.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=side):
            self._enqueue(plan, side, synth=not split)
        synth_graph = None
        if split:
            synth_graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(synth_graph, stream=side):
                self._enqueue(plan, side, trace=False)
        torch.cuda.current_stream(self.device).wait_stream(side)
        plan.graph = graph
        plan.synth_graph = synth_graph
        _guard_scenes(plan)

    # ---- pipelined steps: the trace of step k runs beside the synthesis of step k-1
    def _pipe_setup(self, plan: Plan) -> None:
        if plan.echo_prev is not None:
            return
        plan.echo_prev = torch.zeros_like(plan.echo_store)
        synth, off = [], 0
        for k, j in enumerate(plan.jobs):
            bins = int(j.spec.num_bins)
            view = plan.echo_prev[off:off + NUM_BANDS * bins].view(NUM_BANDS, bins)
            off += NUM_BANDS * bins
            synth.append(runtime.SynthJob(view, plan.irs[k], j.fs, j.spec.bin_duration, seed=int(j.spec.seed) + 7,
                                          direct_delay=max(0.0, float(j.spec.direct_delay)),
                                          speed_of_sound=j.spec.speed_of_sound))
        plan.synth_jobs_prev = runtime.synth_job_array(synth, plan.synth_config)
        plan.keepalive.append(synth)
        plan.pipe_side = torch.cuda.Stream(self.device)  # type: ignore[attr-defined]
        # private staged workspaces: the synthesis and the trace now run on different streams
        plan.workspace = runtime.BatchWorkspace(self.device)
        plan.synth_workspace = runtime.SynthBatchWorkspace(self.device)

    def _enqueue_pipelined(self, plan: Plan, main: torch.cuda.Stream) -> None:
        side: torch.cuda.Stream = plan.pipe_side  # type: ignore[attr-defined]
        side.wait_stream(main)
        raw_done = torch.cuda.Event()
        synth = (plan.synth_jobs_prev, len(plan.jobs), plan.synth_config)
        with torch.cuda.stream(side):
            # the previous step's echograms, then their raw band signals -- before the trace takes every SM
            plan.echo_prev.copy_(plan.echo_store)
            runtime.synthesize_batch(synth, plan.synth_workspace, stream=side, phase="raw")
            raw_done.record(side)
        main.wait_event(raw_done)
        with torch.cuda.stream(main):
            runtime.trace_batch([(plan.scenes[j.scene_index], j.spec, b) for j, b in zip(plan.jobs, plan.buffers)],
                                plan.workspace, block_size=self.block_size, grid_blocks=self.grid_blocks,
                                chunk_rays=self.chunk_rays, stack_entries=self.stack_entries, stream=main)
        with torch.cuda.stream(side):
            # the recursion runs as one-warp blocks beside the persistent trace blocks
            runtime.synthesize_batch(synth, plan.synth_workspace, stream=side, phase="filter")
        main.wait_stream(side)

    def launch_pipelined(self, plan: Plan) -> None:
        """One pipelined step: trace every job while synthesising the echograms the previous step traced.

        Every step does the full trace and the full synthesis; the band IRs in
        `plan.irs` after a step belong to the echograms of the step before it
        (after `launch`, or a first pipelined step, to that launch's trace).
        """
        self._pipe_setup(plan)
        if plan.pipe_graph is not None:
            plan.pipe_graph.replay()
            plan.replayed.record(torch.cuda.current_stream(self.device))
            return
        self._enqueue_pipelined(plan, torch.cuda.current_stream(self.device))

    def capture_pipelined(self, plan: Plan) -> None:
        """Record one pipelined step as a CUDA graph (two streams forked and joined inside the graph)."""
        self._pipe_setup(plan)
        main = torch.cuda.Stream(self.device)
        main.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(main):
            self._enqueue_pipelined(plan, main)   # warm-up: sizes workspaces
        main.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=main):
            self._enqueue_pipelined(plan, main)
        torch.cuda.current_stream(self.device).wait_stream(main)
        plan.pipe_graph = graph
        _guard_scenes(plan)

    def late_tails(self, plan: Plan, *, transition_s: float = 1.0, overlap_fraction: float = 0.25,
                   stream: torch.cuda.Stream | None = None):
        """Hybrid FDN late tails of every job of `plan` (see plan_late_tails)."""
        return plan_late_tails(self, plan, transition_s=transition_s, overlap_fraction=overlap_fraction,
                               stream=stream)

    def ray_bounces(self, plan: Plan) -> int:
        return int(sum(int(b.counters[2].item()) for b in plan.buffers))

    def results(self, plan: Plan) -> list[np.ndarray]:
        """Band IRs per job, [6, N] float32 host arrays, in job order (one device-to-host copy)."""
        host = plan.ir_store.cpu().numpy()
        out, off = [], 0
        for t in plan.irs:
            out.append(host[off:off + t.numel()].reshape(t.shape))
            off += t.numel()
        return out


def _guard_scenes(plan: Plan) -> None:
    """Make each of the plan's scenes wait, before it is destroyed, for the plan's last graph replay."""
    if plan.replayed is None:
        plan.replayed = torch.cuda.Event()
    for scene in plan.scenes:
        if not any(g is plan.replayed for g in scene.graph_guards):
            scene.graph_guards.append(plan.replayed)


def plan_late_tails(renderer: "RIRRenderer", plan: Plan, *, transition_s: float = 1.0,
                    overlap_fraction: float = 0.25, stream: torch.cuda.Stream | None = None):
    """Late tails for every job of a plan whose trace and synthesis have been enqueued on `stream`
    (late_reverb.batch_late_tails over the plan's band IRs and echograms); returns its BatchTails."""
    from acoustic_agent_b200 import late_reverb
    stream = stream if stream is not None else torch.cuda.current_stream(renderer.device)
    with torch.cuda.stream(stream):
        echo_host = plan.echo_store.to("cpu", non_blocking=True)
    stream.synchronize()
    echo = echo_host.numpy()
    echograms, off = [], 0
    for j in plan.jobs:
        bins = int(j.spec.num_bins)
        echograms.append(echo[off:off + NUM_BANDS * bins].reshape(NUM_BANDS, bins))
        off += NUM_BANDS * bins
    if getattr(renderer, "_late", None) is None:
        renderer._late = late_reverb.LateReverbRenderer(renderer.device)
    return late_reverb.batch_late_tails(
        renderer._late, plan.irs, echograms, [j.fs for j in plan.jobs], [int(j.spec.seed) for j in plan.jobs],
        [j.spec.bin_duration for j in plan.jobs], [j.spec.speed_of_sound for j in plan.jobs],
        transition_s=transition_s, overlap_fraction=overlap_fraction, stream=stream)


def render(workloads: Sequence[Workload], *, device: int = 0, precision: str = "float32",
           rng_mode: str = "philox") -> list[np.ndarray]:
    """End-to-end: host scene specs in, host band IRs out (one [6, N] array per source x channel)."""
    renderer = RIRRenderer(device)
    specs, jobs = workload_jobs(workloads, precision=precision, rng_mode=rng_mode)
    plan = renderer.plan([compile_scene(s) for s in specs], jobs)
    renderer.launch(plan)
    torch.cuda.synchronize(renderer.device)
    results = renderer.results(plan)
    for s in plan.scenes:
        s.close()
    return results
