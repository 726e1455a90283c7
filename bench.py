"""Benchmark: RIRs/s (and ray-bounces/s) of the B200 reflection backend.

Default workload (one step = one pass over one batch): the batching
configuration -- 256 seeded scenes whose sizes run from a single furnished
room to an 8-room apartment, 1-4 sources x 1-8 receiver channels each, ray
budgets log-uniform in 1e4-1e6, 50-200 bounces, fs 16 kHz, 1-2 s, per-scene
six-band materials (2,863 RIRs per step).  A step is one graph-captured
persistent trace launch over every job followed by one ragged band synthesis
of every job; scenes are resident in HBM and L2 is flushed between timed
steps.  Beside it the line reports the plain per-job loop over the same jobs,
the drop-in ``trace_energy_field`` per job inside the reference, the
reference's own Numba-CUDA float32 backend per job on this GPU, the
reference's float64 Numba path (``cpu_baseline``), the parity of the GPU
echograms against that float64 path, and the single-scene U-room figures
(``config1_u_room``; ``--workload u_room_20_boxes`` gives that workload a
line of its own).

``--impl reference`` times the reference's own CPU implementation of the path
instead: the unmodified reference package installed under baseline/_ref,
``steam_rt.trace_energy_field`` on its float64 Numba path over all host
threads plus ``reconstruct_band_irs``, one uniformly drawn job of the same
batch per step.  Under torchrun each rank runs an independent replica
(replicas only: jobs are independent, no collective on the data path); rank 0
prints one JSON line.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import sys
import threading
import time
import types
from datetime import timedelta
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))

METRIC = "RIRs/s"
L2_FLUSH_BYTES = 256 * 1024 * 1024
LAUNCHES_PER_STEP = 6  # zero-outputs, trace, finalize, synth prepare, synth raw, synth filter


def _peaks() -> dict:
    path = REPO / "MEASURED_PEAKS.json"
    if path.exists():
        data = json.loads(path.read_text())
        return {"hbm_gbs": float(data["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def _workload(name: str):
    from acoustic_agent_b200 import workloads
    if name == "u_room_20_boxes":
        return [workloads.u_furnished(1729)]
    if name == "shoebox":
        return [workloads.shoebox(1729)]
    if name == "apartment":
        return [workloads.apartment(1729)]
    raise SystemExit(f"unknown workload {name}")


class ClockSampler:
    """NVML clock / throttle-reason sampling during the timed region (read-only)."""

    REASONS = {
        0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
        0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown",
        0x100: "display_clock_setting",
    }

    def __init__(self, index: int) -> None:
        self.samples: list[int] = []
        self.reasons: set[str] = set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._thread = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = pynvml
            self.handle = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = int(pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM))
        except Exception:
            self.nvml = None

    def _run(self) -> None:
        while not self._stop.is_set():
            try:
                self.samples.append(int(self.nvml.nvmlDeviceGetClockInfo(self.handle, self.nvml.NVML_CLOCK_SM)))
                mask = int(self.nvml.nvmlDeviceGetCurrentClocksEventReasons(self.handle))
                self.reasons |= {name for bit, name in self.REASONS.items() if mask & bit and name != "gpu_idle"}
            except Exception:
                pass
            self._stop.wait(0.1)

    def __enter__(self):
        if self.nvml is not None:
            self._thread = threading.Thread(target=self._run, daemon=True)
            self._thread.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._thread is not None:
            self._thread.join()

    def median_mhz(self) -> int | None:
        return int(statistics.median(self.samples)) if self.samples else None

    def summary(self) -> dict:
        return {"sm_mhz": int(statistics.median(self.samples)) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons), "samples": len(self.samples)}


def replica_throughput(ms_per_step: float, rirs_per_step: int, dist=None, device=None) -> tuple[float, float]:
    """Whole-job throughput of independent replicas: every rank ran the same step count on its own
    jobs; the job took as long as the slowest rank (MAX over ranks), and the RIRs of all ranks count."""
    world = 1
    if dist is not None and dist.is_initialized():
        import torch
        world = dist.get_world_size()
        t = torch.tensor([ms_per_step], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_per_step = float(t.item())
    return ms_per_step, world * rirs_per_step / (ms_per_step / 1000.0)


def _dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


REFERENCE_TARGET = REPO / "baseline" / "_ref"


class _Stub(types.ModuleType):
    """Stand-in for a module the reference imports at top level but the tracer never calls."""

    def __getattr__(self, item):
        if item.startswith("__"):
            raise AttributeError(item)
        return type(item, (), {})


def import_reference_package():
    """The unmodified reference installed with pip --target under baseline/_ref: (steam_rt, models) or a reason.

    shapely and h5py are imported at module level by the reference but unused
    on the reflection path, and are absent here; empty stand-ins take their place.
    """
    if not (REFERENCE_TARGET / "acoustic_agent" / "steam_rt.py").exists():
        return None, "reference package not installed under baseline/_ref"
    for name in ("shapely", "shapely.geometry", "shapely.geometry.base", "shapely.ops", "h5py"):
        try:
            __import__(name)
        except Exception:
            sys.modules[name] = _Stub(name)
    if isinstance(sys.modules.get("shapely"), _Stub):
        sys.modules["shapely"].affinity = _Stub("shapely.affinity")
    try:
        import networkx  # noqa: F401
    except Exception:
        sys.modules.setdefault("networkx", _Stub("networkx"))
    if str(REFERENCE_TARGET) not in sys.path:
        sys.path.insert(0, str(REFERENCE_TARGET))
    try:
        from acoustic_agent import models, steam_rt
    except Exception as exc:  # pragma: no cover - depends on the box
        return None, f"reference import failed: {type(exc).__name__}: {exc}"
    return (steam_rt, models), None


def reference_scene(steam_rt, models, spec: dict):
    """The reference's own RoomRayScene for a workload spec (models.Room + per-surface materials)."""
    band_names = models.FREQUENCY_BANDS

    def material(kind, data):
        absorption = data.get("absorption", [0.1] * 6)
        scattering = data.get("scattering", [0.1] * 6)
        return models.Material(id=f"bench_{kind}", name=kind, semantic=kind,
                               absorption={b: float(v) for b, v in zip(band_names, absorption)},
                               scattering={b: float(v) for b, v in zip(band_names, scattering)})

    metadata = {}
    if spec.get("surface_segments") is not None:
        metadata["surface_segments"] = [dict(s) for s in spec["surface_segments"]]
    if spec.get("objects") is not None:
        metadata["objects"] = [dict(o) for o in spec["objects"]]
    room = models.Room(id="bench", name="bench", corners=tuple((float(x), float(y)) for x, y in spec["corners"]),
                       height_m=float(spec["height"]),
                       materials={k: material(k, v) for k, v in spec.get("materials", {}).items()},
                       metadata=metadata)
    steam_rt._clear_static_caches()
    scene = steam_rt.RoomRayScene(room)
    if spec.get("surface_absorption") is not None:
        for surface, row in zip(scene.surfaces, spec["surface_absorption"]):
            surface.absorption = np.asarray(row, dtype=float)
    if spec.get("surface_scattering") is not None:
        for surface, value in zip(scene.surfaces, spec["surface_scattering"]):
            surface.scattering = np.full(6, float(value))
    return scene


def reference_rirs(workload, steps: int, warmup: int, *, accelerator: str, precision: str,
                   channel: int = 0, rays: int | None = None) -> dict:
    """One RIR per step through the reference's public reflection call on one channel of the workload.

    ``steam_rt.trace_energy_field`` (steam_rt.py:1757-1804; "numba" = the
    float64 Numba CPU path over all host threads, "cuda" = its Numba-CUDA
    float32 kernel) followed by ``reconstruct_band_irs`` (steam_rt.py:2205-2232).
    """
    ref, reason = import_reference_package()
    if ref is None:
        return {"unavailable": reason}
    steam_rt, models = ref
    cfg = workload.config
    if accelerator == "cuda":
        from acoustic_agent.steam_rt_cuda import cuda_available
        if not cuda_available(0):
            return {"unavailable": "the reference's Numba-CUDA backend reports no usable CUDA device"}
    scene = reference_scene(steam_rt, models, workload.spec)
    R = int(rays or cfg.rt_num_rays)
    sim = models.SimConfig(fs=cfg.fs, c=cfg.c, duration_s=cfg.duration_s, rt_duration_s=cfg.rt_duration_s,
                           rt_num_rays=R, rt_num_bounces=cfg.rt_num_bounces,
                           rt_bin_duration_s=cfg.rt_bin_duration_s, rt_specular_exponent=cfg.rt_specular_exponent,
                           rt_irradiance_min_distance=cfg.rt_irradiance_min_distance,
                           rt_source_radius=cfg.rt_source_radius, rt_listener_radius=cfg.rt_listener_radius,
                           intersection_backend=cfg.intersection_backend, seed=cfg.seed,
                           rt_accelerator=accelerator, rt_precision=precision, collect_visual_paths=False,
                           render_ambisonics=False)
    src = np.asarray(workload.sources[0], dtype=float)
    lst = np.asarray(workload.listeners[channel], dtype=float)
    times, trace_times = [], []
    field = None
    for k in range(warmup + steps):
        t0 = time.perf_counter()
        field = steam_rt.trace_energy_field(scene, src, lst, sim, workload.source_model, render_ambisonics=False)
        t1 = time.perf_counter()
        steam_rt.reconstruct_band_irs(field, sim)
        if k >= warmup:
            times.append(time.perf_counter() - t0)
            trace_times.append(t1 - t0)
    per_rir = float(np.mean(times))
    threads = None
    if accelerator == "numba":
        import numba
        threads = int(numba.get_num_threads())
    return {"value": 1.0 / per_rir, "seconds_per_rir": per_rir, "trace_seconds": float(np.mean(trace_times)),
            "threads": threads, "rays": R,
            "accelerator": field.get("accelerator") if isinstance(field, dict) else accelerator,
            "sample": (f"channel {channel} of {len(workload.listeners)}: {R} rays x {cfg.rt_num_bounces} bounces, "
                       f"trace_energy_field(rt_accelerator={accelerator!r}, rt_precision={precision!r}) + "
                       f"reconstruct_band_irs, mean of {steps} after {warmup} warm-up")}


def cpu_reference(workload, steps: int, warmup: int, *, channel: int = 0, rays: int | None = None) -> dict:
    """The reference algorithm on the host: float64 trace + band synthesis of one RIR per step (all cores)."""
    from oracle import oracle
    from acoustic_agent_b200 import scene as scene_mod, rng as rng_mod
    from acoustic_agent_b200.directivity import source_directivity, source_forward
    cfg = workload.config
    arrays = scene_mod.compile_scene(workload.spec)
    R = int(rays or cfg.rt_num_rays)
    B = cfg.rt_num_bounces
    key = rng_mod.stream_key(workload.name, 0)
    directions, rnd, idx = oracle.philox_workspace(R, B, cfg.seed, key)
    _, bank, _, _ = oracle.workspace(1, 0, 0)
    emitter = source_directivity(workload.source_model)
    src = np.asarray(workload.sources[0], dtype=float)
    lst = np.asarray(workload.listeners[channel], dtype=float)
    delay = float(np.linalg.norm(src - lst)) / cfg.c
    spb = max(1, int(math.ceil(cfg.rt_bin_duration_s * cfg.fs)))
    white = np.random.default_rng(cfg.seed + 7).uniform(-1.0, 1.0, size=cfg.num_bins * spb)
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    times = []
    stats = None
    for k in range(warmup + steps):
        t0 = time.perf_counter()
        res = oracle.trace(arrays, source=src, listener=lst, directions=directions, diffuse_bank=bank,
                           diffuse_random=rnd, diffuse_indices=idx, num_bins=cfg.num_bins,
                           bin_dur=cfg.rt_bin_duration_s, c=cfg.c, max_path_len=cfg.max_path_length,
                           direct_delay=delay, source_forward=source_forward(emitter),
                           dipole_weight=float(emitter["dipole_weight"]), dipole_power=float(emitter["dipole_power"]),
                           use_bvh=cfg.intersection_backend == "bvh", threads=cores)
        oracle.synthesize(res["echogram"].astype(np.float32), fs=cfg.fs, bin_dur=cfg.rt_bin_duration_s,
                          direct_delay=delay, c=cfg.c, white=white)
        if k >= warmup:
            times.append(time.perf_counter() - t0)
        stats = res
    per_rir = float(np.mean(times))
    # Algorithmic bytes per ray-bounce in the reference's traversal order:
    # nodes 32 B, walls 32 B, polygons 16 B + 8 B per edge, boxes 48 B, one 32 B material row per bounce.
    q = stats["closest_queries"]
    walls, polys, boxes = stats["prims_tested"]
    bytes_total = (stats["nodes_visited"] * 32 + walls * 32 + polys * 16 + stats["polygon_edges"] * 8 + boxes * 48
                   + q * 32)
    return {
        "value": 1.0 / per_rir, "seconds_per_rir": per_rir, "cores": cores, "ray_bounces": q,
        "ray_bounces_per_s": q / per_rir, "bytes_per_ray_bounce": bytes_total / max(q, 1),
        "sample": (f"channel {channel} of {len(workload.listeners)}: {R} rays x {B} bounces, float64 trace + "
                   f"band synthesis, {cores} threads, mean of {steps} after {warmup} warm-up"),
    }


def run_reference_arm(args, workload_name: str) -> None:
    """The reference's own CPU implementation of the path, one RIR per step, all host threads.

    The unmodified reference package under baseline/_ref runs its float64
    Numba path (``rt_accelerator="numba"``); when that package cannot be
    imported, the float64 C restatement of the same algorithm runs instead.
    """
    world, rank, _ = _dist_setup()
    if rank != 0:
        return
    workload = _workload(workload_name)[0]
    ref = reference_rirs(workload, args.steps, args.warmup, accelerator="numba", precision="float64")
    if "unavailable" not in ref:
        kind, cores, note = "reference", ref["threads"], ("the reference package (baseline/_ref), "
                                                           "steam_rt.trace_energy_field float64 Numba path")
    else:
        reason = ref["unavailable"]
        ref = cpu_reference(workload, args.steps, args.warmup)
        kind, cores, note = "port", ref["cores"], f"{reason}; float64 C restatement of the reference algorithm"
    line = {
        "impl": "reference", "metric": METRIC, "value": ref["value"], "unit": "RIRs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ref["seconds_per_rir"] * 1000.0,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload.name, "rays": workload.config.rt_num_rays,
                   "bounces": workload.config.rt_num_bounces, "channels_per_step": 1, "note": note},
        "cpu_baseline": {"value": ref["value"], "unit": "RIRs/s", "cores": cores, "kind": kind,
                         "sample": ref["sample"]},
        "e2e": {"value": ref["value"], "unit": "RIRs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_reference_mixed(args) -> None:
    """The reference's own CPU path on the headline mix: one job of the 256-scene batch per step.

    Jobs are drawn uniformly (seeded) from the same batch as the default arm, so the mean time per step
    estimates the reference's mean time per RIR over the batch; each step runs the unmodified reference's
    ``trace_energy_field`` on its float64 Numba path over all host threads plus ``reconstruct_band_irs``.
    Under torchrun only rank 0 runs.
    """
    world, rank, _ = _dist_setup()
    if rank != 0:
        return
    from acoustic_agent_b200 import batching, workloads
    population = workloads.mixed_batch(1729, args.scenes)
    _, jobs = batching.workload_jobs(population)
    picks = uniform_jobs(jobs, args.warmup + args.steps, seed=11)
    ref = reference_job_loop(population, jobs, picks, accelerator="numba", precision="float64", untimed=args.warmup)
    config = {"workload": f"mixed_batch: {args.scenes} scenes of 1-8 rooms, 1-4 sources x 1-8 channels, "
                          "1e4-1e6 rays, 50-200 bounces, fs 16 kHz, 1-2 s, 10 ms bins",
              "rirs_per_step": 1, "note": "one uniformly drawn job of the batch per step"}
    if "unavailable" in ref:
        print(json.dumps({"impl": "reference", "unavailable": ref["unavailable"]}), flush=True)
        return
    value = ref["rirs_per_s"]
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "RIRs/s", "n_gpus": world,
        "steps": ref["jobs_timed"], "warmup": args.warmup, "ms_per_step": 1000.0 / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded scene generator)",
        "config": config,
        "cpu_baseline": {"value": value, "unit": "RIRs/s", "cores": ref["threads"], "kind": "reference",
                         "sample": ref["sample"]},
        "e2e": {"value": value, "unit": "RIRs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)


def main() -> int:
    parser = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=10)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", choices=("ours", "reference"), default="ours")
    parser.add_argument("--workload", default="mixed_batch",
                        choices=("u_room_20_boxes", "shoebox", "apartment", "mixed_batch", "serving", "late_reverb",
                                 "direct", "bvh_build"))
    parser.add_argument("--no-graph", action="store_true", help="launch eagerly instead of replaying a CUDA graph")
    parser.add_argument("--no-pipeline", action="store_true",
                        help="run each step's synthesis after its own trace instead of beside the next trace")
    parser.add_argument("--no-cpu-baseline", action="store_true")
    parser.add_argument("--e2e-slots", type=int, default=3, help="end-to-end steps kept in flight (streams)")
    parser.add_argument("--block", type=int, default=0)
    parser.add_argument("--scenes", type=int, default=256, help="mixed_batch: scenes in the batch")
    parser.add_argument("--reference-jobs", type=int, default=16,
                        help="mixed_batch: jobs of the reference's plain per-scene CUDA path to time")
    parser.add_argument("--plain-jobs", type=int, default=0,
                        help="mixed_batch: jobs of the plain per-job loop to time (0: all)")
    parser.add_argument("--parity-jobs", type=int, default=3,
                        help="mixed_batch: uniformly drawn jobs traced by the reference's float64 path for the "
                             "parity block and the CPU baseline")
    parser.add_argument("--e2e-steps", type=int, default=2, help="mixed_batch: end-to-end steps to time")
    parser.add_argument("--profile-launch", action="store_true",
                        help="after the warm-up, run one eager step (mixed_batch) or trace launch (single-scene "
                             "workloads) between cudaProfilerStart/Stop and exit (for ncu --profile-from-start off)")
    parser.add_argument("--no-config1", dest="with_config1", action="store_false",
                        help="mixed_batch: skip the single-scene U-room figures added to the line")
    parser.add_argument("--rate", type=float, default=50.0, help="serving: Poisson arrival rate, requests/s")
    parser.add_argument("--rates", default="", help="serving: comma-separated arrival rates (overrides --rate)")
    parser.add_argument("--runs", type=int, default=1, help="serving: runs per rate")
    parser.add_argument("--server", default="continuous", choices=("continuous", "batched"),
                        help="serving: kernel-level continuous batching or batch-level server")
    parser.add_argument("--slo", type=float, default=2.0,
                        help="serving (continuous): shed requests whose admitted work ahead exceeds this, seconds")
    parser.add_argument("--capacity-rb", type=float, default=2.6e9,
                        help="serving (continuous): ray-bounces/s assumed until measured while saturated")
    parser.add_argument("--service-blocks-per-sm", type=int, default=3,
                        help="serving (continuous): persistent trace blocks per SM")
    parser.add_argument("--service-reserve-blocks", type=int, default=16,
                        help="serving (continuous): blocks left out of the persistent grid, for the synthesis")
    parser.add_argument("--duration", type=float, default=10.0, help="serving: seconds of arrivals")
    parser.add_argument("--policy", default="small_first", choices=("small_first", "fifo"),
                        help="serving: order in which waiting requests join a batch")
    parser.add_argument("--max-batch-rays", type=int, default=400_000_000, help="serving: rays per batch at most")
    parser.add_argument("--max-inflight", type=int, default=3, help="serving: batches on the GPU at once")
    parser.add_argument("--late-tail", action="store_true",
                        help="serving: crossfade every served RIR into its FDN late tail")
    parser.add_argument("--trace-blocks-per-sm", type=int, default=2,
                        help="serving: cap each batch's trace grid (0: the library's choice)")
    args = parser.parse_args()
    if args.warmup < 3:
        parser.error("--warmup must be at least 3")
    if args.impl == "reference" and args.workload == "late_reverb":
        world, rank, _ = _dist_setup()
        if rank == 0:
            ref = reference_late_tails(args.steps, args.warmup)
            print(json.dumps({
                "impl": "reference", "metric": "late tails/s", "value": ref["value"], "unit": "tails/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ref["seconds_per_tail"] * 1000.0, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded decaying noise)",
                "config": {"workload": "late_reverb: one 48 kHz x 2 s channel per step"},
                "cpu_baseline": {"value": ref["value"], "unit": "tails/s", "cores": ref["cores"], "kind": ref["kind"],
                                 "sample": ref["sample"]},
                "e2e": {"value": ref["value"], "unit": "tails/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
                flush=True)
        return 0
    if args.impl == "reference" and args.workload == "direct":
        world, rank, _ = _dist_setup()
        if rank == 0:
            from acoustic_agent_b200 import workloads
            w = workloads.u_furnished(1729)
            ref = reference_direct(w, direct_pairs(w, DIRECT_PAIRS), max(20, args.steps))
            if "unavailable" in ref:
                print(json.dumps({"impl": "reference", "unavailable": ref["unavailable"]}), flush=True)
            else:
                print(json.dumps({
                    "impl": "reference", "metric": "direct paths/s", "value": ref["value"], "unit": "paths/s",
                    "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                    "ms_per_step": ref["seconds_per_pair"] * 1000.0, "higher_is_better": True, "scaling": "weak",
                    "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded pairs)",
                    "config": {"workload": "direct: one source/listener pair per step, furnished U room"},
                    "cpu_baseline": {"value": ref["value"], "unit": "paths/s", "cores": 1, "kind": "reference",
                                     "sample": ref["sample"]},
                    "e2e": {"value": ref["value"], "unit": "paths/s", "h2d_bytes_per_step": 0,
                            "d2h_bytes_per_step": 0}}), flush=True)
        return 0
    if args.impl == "reference" and args.workload == "bvh_build":
        world, rank, _ = _dist_setup()
        if rank == 0:
            ref = reference_bvh(max(3, args.steps))
            if "unavailable" in ref:
                print(json.dumps({"impl": "reference", "unavailable": ref["unavailable"]}), flush=True)
            else:
                print(json.dumps({
                    "impl": "reference", "metric": "BVH surfaces/s", "value": ref["value"], "unit": "surfaces/s",
                    "n_gpus": world, "steps": max(3, args.steps), "warmup": args.warmup,
                    "ms_per_step": ref["seconds"] * 1000.0, "higher_is_better": True, "scaling": "weak",
                    "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded warehouse AABBs)",
                    "config": {"workload": f"bvh_build: {BVH_SAMPLE} of the {BVH_SURFACES} warehouse surfaces"},
                    "cpu_baseline": {"value": ref["value"], "unit": "surfaces/s", "cores": 1, "kind": "reference",
                                     "sample": ref["sample"]},
                    "e2e": {"value": ref["value"], "unit": "surfaces/s", "h2d_bytes_per_step": 0,
                            "d2h_bytes_per_step": 0}}), flush=True)
        return 0
    if args.impl == "reference":
        if args.workload == "serving":
            parser.error("--impl reference has no serving arm: the reference has no request loop")
        if args.workload == "mixed_batch":
            run_reference_mixed(args)
        else:
            run_reference_arm(args, args.workload)
        return 0
    if args.workload == "mixed_batch":
        return run_mixed_batch(args)
    if args.workload == "serving":
        return run_serving(args)
    if args.workload == "late_reverb":
        return run_late_reverb(args)
    if args.workload == "direct":
        return run_direct(args)
    if args.workload == "bvh_build":
        return run_bvh_build(args)

    return run_single_scene(args, args.workload)


def run_single_scene(args, workload_name: str, *, extras_only: bool = False):
    """One scene (the U room of the second configuration by default): every channel per step in one
    persistent trace launch beside the band synthesis of the previous step (pipelined, graph-replayed).

    With `extras_only` it returns the resident throughput and trace launch time as a dict (no end-to-end
    run, no baselines) for the headline line instead of printing a line of its own.
    """
    import torch
    from acoustic_agent_b200 import batching, runtime, scene as scene_mod

    world, rank, local = _dist_setup()
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    dist = None
    if world > 1 and not extras_only:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=device)

    workloads_ = _workload(workload_name)
    specs, jobs = batching.workload_jobs(workloads_, precision="float32", rng_mode="philox")
    renderer = batching.RIRRenderer(local, block_size=args.block)
    arrays = [scene_mod.compile_scene(s) for s in specs]
    plan = renderer.plan(arrays, jobs)
    pipelined = not args.no_pipeline
    if pipelined:
        renderer.launch(plan)   # the first pipelined step synthesises this trace's echograms
        if not args.no_graph:
            renderer.capture_pipelined(plan)
        step = lambda: renderer.launch_pipelined(plan)  # noqa: E731
    else:
        if not args.no_graph:
            renderer.capture(plan)
        step = lambda: renderer.launch(plan)  # noqa: E731
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=device)
    stream = torch.cuda.current_stream(device)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(device)
    ray_bounces_per_step = renderer.ray_bounces(plan)
    if args.profile_launch and not extras_only:
        # one trace launch of every channel between cudaProfilerStart/Stop (for `ncu --profile-from-start off`)
        profiled = [(plan.scenes[j.scene_index], j.spec, b) for j, b in zip(plan.jobs, plan.buffers)]
        torch.cuda.profiler.start()
        runtime.trace_batch(profiled, runtime.BatchWorkspace(device), block_size=args.block)
        torch.cuda.synchronize(device)
        torch.cuda.profiler.stop()
        print(json.dumps({"profiled": "trace launch", "ray_bounces": ray_bounces_per_step}), flush=True)
        return 0

    def barrier():
        if dist is not None:
            dist.barrier(device_ids=[local])

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    sampler = ClockSampler(local)
    barrier()
    torch.cuda.synchronize(device)
    with sampler:
        for k in range(args.steps):
            flush.fill_(float(k))  # evict L2 (256 MiB > 126 MB) outside the timed event pair
            starts[k].record(stream)
            step()
            stops[k].record(stream)
        torch.cuda.synchronize(device)
    barrier()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, stops)]
    ms_per_step = float(np.mean(step_ms))
    rirs_per_step = plan.num_rirs
    ms_per_step, value = replica_throughput(ms_per_step, rirs_per_step, dist, device)

    # Tracer kernel alone (for the roofline): eager trace_batch launches timed with events.
    trace_ms = []
    job_list = [(plan.scenes[j.scene_index], j.spec, b) for j, b in zip(plan.jobs, plan.buffers)]
    for k in range(max(3, args.steps // 2)):
        flush.fill_(float(k))
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        runtime.trace_batch(job_list, plan.workspace, block_size=args.block, stream=stream)
        e.record(stream)
        e.synchronize()
        trace_ms.append(s.elapsed_time(e))
    trace_launch_ms = float(np.median(trace_ms))
    if extras_only:
        return {"workload": f"{workloads_[0].name}: {rirs_per_step} channels x {workloads_[0].config.rt_num_rays} "
                            f"rays x {workloads_[0].config.rt_num_bounces} bounces, fs {workloads_[0].config.fs}",
                "rirs_per_s": value, "ms_per_step": ms_per_step, "trace_launch_ms": trace_launch_ms,
                "ray_bounces_per_s": ray_bounces_per_step / (ms_per_step / 1000.0), "steps": args.steps,
                "step": "pipelined trace + synthesis, graph-replayed, L2 flushed between steps"}

    # End to end through the public API: every step uploads the scene from host arrays
    # (ac_scene_create), lays out the jobs' outputs, traces and synthesises, and copies the band IRs
    # to pinned host memory.  Several steps are in flight on their own streams (one renderer each), so a
    # step's synthesis and copy overlap the next steps' upload and trace, as a streaming caller would run it.
    slots = [{"stream": torch.cuda.Stream(device), "renderer": batching.RIRRenderer(local, block_size=args.block),
              "out": torch.empty(plan.ir_store.shape, dtype=plan.ir_store.dtype, pin_memory=True), "busy": None}
             for _ in range(max(1, args.e2e_slots))]

    def e2e_drain(slot):
        if slot["busy"] is not None:
            event, scenes_prev, _ = slot["busy"]
            event.synchronize()
            for sc in scenes_prev:
                sc.close()
            slot["busy"] = None

    def e2e_step(slot):
        e2e_drain(slot)
        with torch.cuda.stream(slot["stream"]):
            scenes_k = [runtime.DeviceScene(a, device=local) for a in arrays]
            plan_k = slot["renderer"].plan(scenes_k, jobs)
            slot["renderer"].launch(plan_k, stream=slot["stream"])
            slot["out"].copy_(plan_k.ir_store, non_blocking=True)
            done = torch.cuda.Event()
            done.record(slot["stream"])
        slot["busy"] = (done, scenes_k, plan_k)
        return scenes_k, plan_k

    for k in range(args.warmup):
        e2e_step(slots[k % len(slots)])
    for slot in slots:
        e2e_drain(slot)
    e2e_steps = max(4, args.steps)
    t0 = time.perf_counter()
    for k in range(e2e_steps):
        scenes_k, plan_k = e2e_step(slots[k % len(slots)])
    for slot in slots:
        e2e_drain(slot)
    e2e_s = time.perf_counter() - t0
    h2d = sum(sc.device_bytes for sc in scenes_k) + plan_k.workspace.device_buffer.numel()
    d2h = plan_k.ir_store.numel() * plan_k.ir_store.element_size()
    e2e_value = world * rirs_per_step * e2e_steps / e2e_s

    peaks = _peaks()
    result = None
    if rank == 0:
        cpu = ref_cpu = ref_cuda = None
        if world == 1 and not args.no_cpu_baseline:
            # traversal statistics of the reference algorithm (C restatement) give the algorithmic bytes
            cpu = cpu_reference(workloads_[0], steps=1, warmup=0)
            ref_cpu = reference_rirs(workloads_[0], 1, 1, accelerator="numba", precision="float64")
            ref_cuda = reference_rirs(workloads_[0], 3, 1, accelerator="cuda", precision="float32")
        bytes_per_rb = cpu["bytes_per_ray_bounce"] if cpu else None
        achieved = (bytes_per_rb * ray_bounces_per_step / (trace_launch_ms / 1000.0) / 1e9) if bytes_per_rb else None
        result = {
            "metric": METRIC, "value": value, "unit": "RIRs/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator)",
            "config": {"workload": f"{workloads_[0].name}: U room 6x10x2.8 m, 20 boxes, 8-mic circular array"
                       if workload_name == "u_room_20_boxes" else workloads_[0].name,
                       "rirs_per_step": rirs_per_step, "rays_per_rir": workloads_[0].config.rt_num_rays,
                       "max_bounces": workloads_[0].config.rt_num_bounces, "fs": workloads_[0].config.fs,
                       "bins": workloads_[0].config.num_bins, "rng": "philox", "graph": not args.no_graph,
                       "pipelined": pipelined,
                       "step": ("one full trace of every channel beside the band synthesis of the previous "
                                "step's echograms (two streams)" if pipelined else
                                "one full trace of every channel, then its band synthesis"),
                       "parallelism": f"replicas x{world}", "l2": "flushed between timed steps (256 MiB write)"},
            "ray_bounces_per_step": ray_bounces_per_step,
            "ray_bounces_per_s": world * ray_bounces_per_step / (ms_per_step / 1000.0),
            "trace_launch_ms": trace_launch_ms,
            "e2e": {"value": e2e_value, "unit": "RIRs/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "steps": e2e_steps, "in_flight": len(slots),
                    "step": "upload the scene, plan, trace + synthesise, band IRs to pinned host memory; "
                            f"{len(slots)} steps in flight on {len(slots)} streams"},
            "gpu_launches": LAUNCHES_PER_STEP * args.steps,
            "roofline": roofline_line(achieved, bytes_per_rb, workload_name, device, ray_bounces_per_step)
            if achieved else None,
            "cpu_baseline": _cpu_baseline(cpu, ref_cpu),
            "reference_cuda": _reference_cuda_line(ref_cuda),
            "clocks": sampler.summary(),
        }
        print(json.dumps(result), flush=True)
    if dist is not None:
        dist.barrier(device_ids=[local])
        dist.destroy_process_group()
    return 0


def _device_timed(fn, steps: int, device, flush) -> list[float]:
    import torch
    stream = torch.cuda.current_stream(device)
    out = []
    for k in range(steps):
        flush.fill_(float(k))
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        fn()
        stop.record(stream)
        stop.synchronize()
        out.append(start.elapsed_time(stop))
    return out


def sim_config(models, w, *, accelerator: str, precision: str, rays: int | None = None):
    """The reference's SimConfig for one workload of the mix (the settings its job loops pass per call)."""
    cfg = w.config
    return models.SimConfig(fs=cfg.fs, c=cfg.c, duration_s=cfg.duration_s, rt_duration_s=cfg.rt_duration_s,
                            rt_num_rays=int(rays or cfg.rt_num_rays), rt_num_bounces=cfg.rt_num_bounces,
                            rt_bin_duration_s=cfg.rt_bin_duration_s, rt_specular_exponent=cfg.rt_specular_exponent,
                            rt_irradiance_min_distance=cfg.rt_irradiance_min_distance,
                            rt_source_radius=cfg.rt_source_radius, rt_listener_radius=cfg.rt_listener_radius,
                            intersection_backend=cfg.intersection_backend, seed=cfg.seed, rt_accelerator=accelerator,
                            rt_precision=precision, collect_visual_paths=False, render_ambisonics=False)


def uniform_jobs(jobs, count: int, seed: int) -> list[int]:
    """`count` job indices drawn uniformly without replacement (seeded), so their mean cost estimates the batch's."""
    rng = np.random.default_rng(seed)
    return [int(k) for k in rng.choice(len(jobs), size=min(count, len(jobs)), replace=False)]


def reference_job_loop(population, jobs, picks, *, accelerator: str, precision: str, warm: bool = True,
                       time_limit_s: float | None = None, untimed: int = 0) -> dict:
    """The reference's own per-job call on jobs of the mix, as its job loops make them (engine.py:64-73,
    batch.py:139-185): ``steam_rt.trace_energy_field`` + ``reconstruct_band_irs`` per (scene, source, channel).

    accelerator "numba" = its float64 Numba path over all host threads, "cuda" = its Numba-CUDA float32 kernel
    on this GPU, "b200" = this repository's drop-in installed into the reference.  The first call (kernel
    compilation) runs on the batch's smallest job and is not timed.  Returns RIRs/s over the timed jobs and,
    per job, its float echogram.
    """
    ref, reason = import_reference_package()
    if ref is None:
        return {"unavailable": reason}
    steam_rt, models = ref
    installation = None
    if accelerator == "cuda":
        try:
            from acoustic_agent.steam_rt_cuda import cuda_available
            if not cuda_available(0):
                return {"unavailable": "the reference's Numba-CUDA backend reports no usable CUDA device"}
        except Exception as exc:  # pragma: no cover - depends on the box
            return {"unavailable": f"reference CUDA backend import failed: {type(exc).__name__}: {exc}"}
    if accelerator == "b200":
        from acoustic_agent_b200 import backend
        installation = backend.install(steam_rt)
    scenes: dict[int, object] = {}

    def run(k):
        j = jobs[k]
        w = population[j.workload]
        if j.workload not in scenes:
            scenes[j.workload] = reference_scene(steam_rt, models, w.spec)
        sim = sim_config(models, w, accelerator=accelerator, precision=precision)
        field = steam_rt.trace_energy_field(scenes[j.workload], np.asarray(w.sources[j.source], dtype=float),
                                            np.asarray(w.listeners[j.channel], dtype=float), sim, w.source_model,
                                            render_ambisonics=False)
        steam_rt.reconstruct_band_irs(field, sim)
        return np.asarray(field["echogram"], dtype=np.float64)

    try:
        if warm:
            run(min(range(len(jobs)), key=lambda k: jobs[k].spec.num_rays))
        for k in picks[:untimed]:
            run(k)
        echograms, seconds, timed = {}, 0.0, []
        for k in picks[untimed:]:
            t0 = time.perf_counter()
            echograms[k] = run(k)
            seconds += time.perf_counter() - t0
            timed.append(k)
            if time_limit_s is not None and seconds > time_limit_s:
                break
    finally:
        if installation is not None:
            installation.uninstall()
    threads = None
    if accelerator == "numba":
        import numba
        threads = int(numba.get_num_threads())
    rays = [jobs[k].spec.num_rays for k in timed]
    return {"rirs_per_s": len(timed) / seconds, "jobs_timed": len(timed), "seconds": seconds,
            "ray_mean": float(np.mean(rays)), "threads": threads, "echograms": echograms,
            "sample": (f"{len(timed)} jobs drawn uniformly from the batch (mean {np.mean(rays):,.0f} rays against "
                       f"{np.mean([j.spec.num_rays for j in jobs]):,.0f} over the batch): trace_energy_field("
                       f"rt_accelerator={accelerator!r}, rt_precision={precision!r}) + reconstruct_band_irs per job, "
                       "after one untimed call")}


def facade_rirs(workload, runs: int = 2) -> dict:
    """The reference's public facade on one workload, its reflection trace routed to this backend:
    ``AcousticAgent.create(scene="geometry", room=Room(...), config=SimConfig(rt_accelerator="b200"),
    receiver_model=<the workload's circular array>).run()`` (api.py:172-245, :405-475; the channel loop of
    engine.py:64-73), after one untimed call.  Everything but the reflection trace is the reference's own code
    on the host (direct sound, diffraction, band synthesis, decay fits); late tail off, as in the reference's
    accelerator benchmark."""
    ref, reason = import_reference_package()
    if ref is None:
        return {"unavailable": reason}
    steam_rt, models = ref
    from acoustic_agent import api
    from acoustic_agent_b200 import backend
    cfg = workload.config
    room = reference_scene(steam_rt, models, workload.spec).room
    sim = models.SimConfig(fs=cfg.fs, duration_s=cfg.duration_s, rt_duration_s=cfg.rt_duration_s,
                           rt_num_rays=cfg.rt_num_rays, rt_num_bounces=cfg.rt_num_bounces,
                           rt_bin_duration_s=cfg.rt_bin_duration_s, intersection_backend=cfg.intersection_backend,
                           late_tail=False, adaptive_geometry_bounces=False, rt_accelerator="b200",
                           rt_precision="float32", seed=cfg.seed)
    center = np.mean(np.asarray(workload.listeners, dtype=float), axis=0)
    array = {"type": "circular", "count": len(workload.listeners), "radius_m": 0.05}
    handle = backend.install(steam_rt)
    try:
        agent = api.AcousticAgent.create(scene="geometry", room=room, config=sim, receiver_model=array,
                                         source_model=workload.source_model, source=workload.sources[0],
                                         receiver=tuple(center))
        agent.run()
        t0 = time.perf_counter()
        for _ in range(runs):
            result = agent.run()
        seconds = (time.perf_counter() - t0) / runs
    finally:
        handle.uninstall()
    refl = result.metadata["steam_audio"]["reflections"]
    channels = int(result.rir.shape[0])
    return {"rirs_per_s": channels / seconds, "seconds_per_run": seconds, "channels": channels,
            "trace_kernel_s_channel0": refl.get("kernel_time_s"), "accelerator": refl.get("accelerator"),
            "sample": f"AcousticAgent.create(...).run() over {channels} channels, mean of {runs} after 1 warm-up"}


def single_rir_latency(workload, repeats: int = 5) -> dict:
    """Latency of ONE RIR (channel 0) end to end through the drop-in: ``backend.trace_energy_field`` (scene
    resident after the first call, the reference's random stream drawn on the device, echogram back on the
    host), then the band synthesis of that echogram on the GPU (``runtime.synthesize``, band IRs back on the
    host).  Median of `repeats` after one warm-up; the synthesis share is stated."""
    import torch
    from acoustic_agent_b200 import backend, runtime, scene as scene_mod
    cfg = workload.config
    arrays = scene_mod.compile_scene(workload.spec)
    src = np.asarray(workload.sources[0], dtype=float)
    lst = np.asarray(workload.listeners[0], dtype=float)
    device = torch.device("cuda", 0)
    ws = runtime.SynthWorkspace(device)
    trace_ms, synth_ms, kernel_ms, upload_ms, hits = [], [], [], [], []
    for k in range(repeats + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        field = backend.trace_energy_field(arrays, src, lst, cfg, workload.source_model, render_ambisonics=False)
        t1 = time.perf_counter()
        if k:
            kernel_ms.append(1e3 * field["kernel_time_s"])
            upload_ms.append(1e3 * field["transfer_time_s"])
            hits.append(field["device_input_cache"])
        echo = torch.as_tensor(field["echogram"][None], device=device)
        d = torch.tensor([field["direct_delay_s"]], dtype=torch.float64, device=device)
        params = runtime.synth_params(1, int(field["num_bins"]), cfg.rt_bin_duration_s, cfg.fs, cfg.c,
                                      rng_mode="philox", seed=int(cfg.seed) + 7, direct_delays=d)
        runtime.synthesize(echo.contiguous(), params, ws).cpu()
        t2 = time.perf_counter()
        if k:
            trace_ms.append(1e3 * (t1 - t0))
            synth_ms.append(1e3 * (t2 - t1))
    tr, sy = float(np.median(trace_ms)), float(np.median(synth_ms))
    return {"trace_ms": tr, "synthesis_ms": sy, "total_ms": tr + sy, "synthesis_share": sy / (tr + sy),
            "trace_kernel_ms": float(np.median(kernel_ms)), "transfer_ms": float(np.median(upload_ms)),
            "device_input_cache": hits[-1],
            "note": "one channel: drop-in trace_energy_field (reference stream, on the device) + GPU band "
                    "synthesis, host arrays in and out, median of 5 after 1 warm-up"}


def mix_bytes_per_ray_bounce(arrays, jobs, ray_bounces_per_job, sample_rays: int = 512) -> float:
    """Algorithmic bytes per ray-bounce over the mix (roofline numerator, per-unit figure).

    For each scene, the float64 C restatement traces the first `sample_rays` rays of its first job on the same
    Philox stream as the GPU and counts the reference traversal's fetches (nodes 32 B, walls 32 B, polygons
    16 B + 8 B per edge, boxes 48 B, one 32 B material row per closest-hit query); scenes are weighted by the
    ray-bounces the GPU executed for their jobs.
    """
    from oracle import oracle
    from acoustic_agent_b200.directivity import source_directivity, source_forward
    _, bank, _, _ = oracle.workspace(1, 0, 0)
    first: dict[int, int] = {}
    weight: dict[int, float] = {}
    for k, j in enumerate(jobs):
        first.setdefault(j.scene_index, k)
        weight[j.scene_index] = weight.get(j.scene_index, 0.0) + float(ray_bounces_per_job[k])
    total_bytes = total_rb = 0.0
    for si, k in first.items():
        spec = jobs[k].spec
        R = min(int(spec.num_rays), sample_rays)
        dirs, rnd, idx = oracle.philox_workspace(R, int(spec.num_bounces), int(spec.seed), int(spec.stream_key))
        emitter = {"dipole_weight": spec.dipole_weight, "dipole_power": spec.dipole_power}
        res = oracle.trace(arrays[si], source=np.asarray(spec.source), listener=np.asarray(spec.listener),
                           directions=dirs, diffuse_bank=bank, diffuse_random=rnd, diffuse_indices=idx,
                           num_bins=int(spec.num_bins), bin_dur=spec.bin_duration, c=spec.speed_of_sound,
                           max_path_len=spec.max_path_length, direct_delay=spec.direct_delay,
                           source_forward=np.asarray(spec.source_forward, dtype=float),
                           dipole_weight=float(emitter["dipole_weight"]), dipole_power=float(emitter["dipole_power"]),
                           use_bvh=bool(spec.use_bvh), threads=1)
        q = res["closest_queries"]
        walls, polys, boxes = res["prims_tested"]
        per = (res["nodes_visited"] * 32 + walls * 32 + polys * 16 + res["polygon_edges"] * 8 + boxes * 48 + q * 32)
        total_bytes += weight[si] * per / max(q, 1)
        total_rb += weight[si]
    return total_bytes / max(total_rb, 1.0)


def run_mixed_batch(args) -> int:
    """Batched mixed-size workload (the headline): many scenes, sources and channels in one persistent launch.

    256 seeded scenes log-uniform between a single room and an 8-room apartment, 1-4 sources and 1-8 channels
    each, 1e4-1e6 rays, fs 16 kHz, 1-2 s.  One step = the graph-captured tracer over every job + the ragged
    band synthesis of every job (autotuned traversal per scene and launch shape).  Beside it: the plain
    per-job loop over the same jobs (resident ac_trace + ac_synthesize + host copy per RIR), the drop-in
    ``trace_energy_field`` per job inside the reference, the reference's own Numba-CUDA float32 backend per
    job, the reference's float64 Numba path (CPU baseline) and the parity of the GPU echograms against it.
    """
    import torch
    from acoustic_agent_b200 import autotune, batching, metrics, runtime, scene as scene_mod, workloads
    world, rank, local = _dist_setup()
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=device)
    t0 = time.perf_counter()
    population = workloads.mixed_batch(1729, args.scenes)
    specs, jobs = batching.workload_jobs(population)
    arrays = [scene_mod.compile_scene(s) for s in specs]
    t_compile = time.perf_counter() - t0
    t0 = time.perf_counter()
    cache = autotune.TuneCache()
    first_job = {}
    for j in jobs:
        first_job.setdefault(j.scene_index, j)
    options = [autotune.tune_scene(a, first_job[k].spec, device=local, cache=cache).options()
               for k, a in enumerate(arrays)]
    renderer = batching.RIRRenderer(local)
    plan = renderer.plan(arrays, jobs, scene_options=options)
    launch = autotune.tune_launch([(plan.scenes[j.scene_index], j.spec) for j in plan.jobs], device=local)
    renderer.block_size, renderer.chunk_rays = launch.block_size, launch.chunk_rays
    renderer.stack_entries = launch.stack_entries
    t_tune = time.perf_counter() - t0
    if not args.no_graph:
        renderer.capture(plan, split=True)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=device)
    stream = torch.cuda.current_stream(device)
    for _ in range(args.warmup):
        renderer.launch(plan)
    torch.cuda.synchronize(device)
    per_job_rb = [int(b.counters[2].item()) for b in plan.buffers]
    rb = int(sum(per_job_rb))
    if args.profile_launch:
        # one eager step of the batch (trace + synthesis) between cudaProfilerStart/Stop, for
        # `ncu --profile-from-start off`
        job_list = [(plan.scenes[j.scene_index], j.spec, b) for j, b in zip(plan.jobs, plan.buffers)]
        ws, sws = runtime.BatchWorkspace(device), runtime.SynthBatchWorkspace(device)
        torch.cuda.profiler.start()
        runtime.trace_batch(job_list, ws, block_size=launch.block_size, chunk_rays=launch.chunk_rays,
                            stack_entries=launch.stack_entries)
        runtime.synthesize_batch((plan.synth_jobs, len(plan.jobs), plan.synth_config), sws)
        torch.cuda.synchronize(device)
        torch.cuda.profiler.stop()
        print(json.dumps({"profiled": "one step (trace + synthesis)", "jobs": len(jobs), "ray_bounces": rb}),
              flush=True)
        return 0

    def barrier():
        if dist is not None:
            dist.barrier(device_ids=[local])

    marks = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    sampler = ClockSampler(local)
    barrier()
    torch.cuda.synchronize(device)
    with sampler:
        for k in range(args.steps):
            flush.fill_(float(k))   # evict L2 (256 MiB > 126 MB) outside the timed events
            start, t_start, t_stop, stop = marks[k]
            start.record(stream)
            renderer.launch(plan, trace_events=(t_start, t_stop))
            stop.record(stream)
        torch.cuda.synchronize(device)
    barrier()
    step_ms = [m[0].elapsed_time(m[3]) for m in marks]
    trace_ms = float(np.mean([m[1].elapsed_time(m[2]) for m in marks]))
    ms = float(np.mean(step_ms))
    ms, value = replica_throughput(ms, len(jobs), dist, device)
    if rank != 0:
        barrier()
        if dist is not None:
            dist.destroy_process_group()
        return 0

    # plain per-job loop over the same jobs: one ac_trace + one ac_synthesize + a host copy per RIR, scenes resident
    order = list(range(len(jobs)))
    if args.plain_jobs > 0:
        order = uniform_jobs(jobs, args.plain_jobs, seed=0)
    ws = runtime.SynthWorkspace(device)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    for k in order:
        j = jobs[k]
        b = runtime.trace(plan.scenes[j.scene_index], j.spec)
        d = torch.tensor([max(0.0, j.spec.direct_delay)], dtype=torch.float64, device=device)
        p = runtime.synth_params(1, j.spec.num_bins, j.spec.bin_duration, j.fs, j.spec.speed_of_sound,
                                 rng_mode="philox", seed=int(j.spec.seed) + 7, direct_delays=d)
        runtime.synthesize(b.echogram[None].contiguous(), p, ws).cpu()
    plain_s = time.perf_counter() - t0
    plain_rirs_per_s = len(order) / plain_s

    # end to end through the public API, host buffers: every step uploads the 256 scenes from host arrays,
    # lays out the jobs, traces + synthesises them (one launch each) and copies the band IRs to pinned host memory
    host_out = torch.empty(plan.ir_store.shape, dtype=plan.ir_store.dtype, pin_memory=True)
    e2e_renderer = batching.RIRRenderer(local, block_size=launch.block_size, chunk_rays=launch.chunk_rays,
                                        stack_entries=launch.stack_entries)

    def e2e_step():
        scenes_k = [runtime.DeviceScene(a, device=local, **o) for a, o in zip(arrays, options)]
        plan_k = e2e_renderer.plan(scenes_k, jobs)
        e2e_renderer.launch(plan_k)
        host_out.copy_(plan_k.ir_store, non_blocking=True)
        torch.cuda.current_stream(device).synchronize()
        for sc in scenes_k:
            sc.close()
        return scenes_k, plan_k

    e2e_step()   # warm-up (staging buffers, allocator)
    e2e_steps = max(2, args.e2e_steps)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        scenes_k, plan_k = e2e_step()
    e2e_s = time.perf_counter() - t0
    h2d = sum(sc.device_bytes for sc in scenes_k) + plan_k.workspace.device_buffer.numel()
    d2h = plan_k.ir_store.numel() * plan_k.ir_store.element_size()
    del plan_k, scenes_k

    line = {
        "metric": METRIC, "value": value, "unit": "RIRs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded scene generator: 256 scenes of 1-8 rooms, random-init materials)",
        "config": {"workload": f"mixed_batch: {args.scenes} scenes of 1-8 rooms, 1-4 sources x 1-8 channels, "
                               "1e4-1e6 rays, 50-200 bounces, fs 16 kHz, 1-2 s, 10 ms bins",
                   "rirs_per_step": len(jobs), "rays_per_step": int(sum(j.spec.num_rays for j in jobs)),
                   "step": "one graph-captured persistent trace launch over every job, then one ragged band "
                           "synthesis of every job (second graph)",
                   "graph": not args.no_graph, "rng": "philox", "parallelism": f"replicas x{world}",
                   "l2": "flushed between timed steps (256 MiB write)",
                   "traversal": {m: sum(1 for s in plan.scenes if s.traversal == m) for m in ("scan", "bvh", "hybrid")},
                   "launch": {"block_size": launch.block_size, "chunk_rays": launch.chunk_rays,
                              "stack_entries": launch.stack_entries,
                              "stack_ms": {str(n): round(t, 3) for n, t in launch.stack_ms}},
                   "stack_entries_by_scene": {str(n): sum(1 for o in options if o["stack_entries"] == n)
                                              for n in sorted({o["stack_entries"] for o in options})}},
        "ray_bounces_per_step": rb, "ray_bounces_per_s": world * rb / (ms / 1000.0),
        "trace_launch_ms": trace_ms, "synthesis_ms": ms - trace_ms,
        "plain": {"rirs_per_s": plain_rirs_per_s, "jobs_timed": len(order), "seconds": plain_s,
                  "note": "per job: ac_trace + ac_synthesize + copy to host, scenes resident, same jobs"},
        "batched_vs_plain": value / plain_rirs_per_s,
        "e2e": {"value": len(jobs) * e2e_steps / e2e_s, "unit": "RIRs/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "steps": e2e_steps,
                "step": "upload 256 scenes from host arrays, plan, trace + synthesise, band IRs to pinned host"},
        "gpu_launches": 6 * args.steps,
        "setup_s": {"compile": t_compile, "tune": t_tune},
        "clocks": sampler.summary(),
    }

    # the extras below each record an error in the line instead of losing it
    def guarded(key, fn):
        try:
            fn()
        except Exception as exc:   # pragma: no cover - depends on the box
            line.setdefault("errors", {})[key] = f"{type(exc).__name__}: {exc}"

    def roofline():
        # algorithmic bytes over the mix / the trace launch's live CUDA-event duration
        bpr = mix_bytes_per_ray_bounce(arrays, jobs, per_job_rb)
        achieved = bpr * rb / (trace_ms / 1000.0) / 1e9
        line["roofline"] = roofline_line(achieved, bpr, "mixed_batch", device, rb)

    picks = uniform_jobs(jobs, args.reference_jobs, seed=3)

    def reference_float64():
        ref64 = reference_job_loop(population, jobs, picks[:args.parity_jobs], accelerator="numba",
                                   precision="float64")
        if "unavailable" in ref64:
            line["cpu_baseline"] = {"unavailable": ref64["unavailable"]}
            return
        line["cpu_baseline"] = {"value": ref64["rirs_per_s"], "unit": "RIRs/s", "cores": ref64["threads"],
                                "kind": "reference", "sample": ref64["sample"]}
        drop = reference_job_loop(population, jobs, picks[:max(args.parity_jobs, 4)], accelerator="b200",
                                  precision="float32", time_limit_s=30.0)
        line["drop_in_plain"] = {k: v for k, v in drop.items() if k != "echograms"}
        if "rirs_per_s" in drop:
            line["batched_vs_drop_in_plain"] = value / drop["rirs_per_s"]
        echo_host = plan.echo_store.cpu().numpy()
        offsets = np.cumsum([0] + [6 * int(j.spec.num_bins) for j in jobs])
        same, philox, philox_rays = [], [], []
        from oracle import oracle
        _, bank, _, _ = oracle.workspace(1, 0, 0)
        for k, ref_echo in ref64["echograms"].items():
            spec = jobs[k].spec
            bd = spec.bin_duration
            ours_philox = echo_host[offsets[k]:offsets[k + 1]].reshape(6, -1)
            philox.append(metrics.parity(ours_philox, ref_echo, bd))
            if k in drop.get("echograms", {}):
                same.append(metrics.parity(drop["echograms"][k], ref_echo, bd))
            # the float64 restatement of the reference's tracer fed the batch's own Philox rays (its workspace
            # holds 12 bytes per ray-bounce slot: jobs up to 4e7 slots)
            if int(spec.num_rays) * int(spec.num_bounces) > 40_000_000:
                continue
            dirs, rnd, idx = oracle.philox_workspace(int(spec.num_rays), int(spec.num_bounces), int(spec.seed),
                                                     int(spec.stream_key))
            f64 = oracle.trace(arrays[jobs[k].scene_index], source=np.asarray(spec.source),
                               listener=np.asarray(spec.listener), directions=dirs, diffuse_bank=bank,
                               diffuse_random=rnd, diffuse_indices=idx, num_bins=int(spec.num_bins), bin_dur=bd,
                               c=spec.speed_of_sound, max_path_len=spec.max_path_length, direct_delay=spec.direct_delay,
                               source_forward=np.asarray(spec.source_forward, dtype=float),
                               dipole_weight=spec.dipole_weight, dipole_power=spec.dipole_power,
                               use_bvh=bool(spec.use_bvh))["echogram"]
            philox_rays.append(metrics.parity(ours_philox, f64, bd))

        def worst(rows):
            return {key: max(r[key] for r in rows) for key in rows[0]} if rows else None

        line["parity"] = {
            "jobs": len(ref64["echograms"]),
            "same_stream": worst(same),
            "philox_same_rays": worst(philox_rays),
            "philox_stream": worst(philox),
            "note": ("worst band and job.  same_stream: the drop-in (float32) on the reference's own random stream "
                     "against the reference's float64 Numba echogram of the same job (trace_energy_field, "
                     "rt_precision='float64'; identical rays).  philox_same_rays: the batch's own float32 echogram "
                     "against the float64 restatement of the reference's tracer fed the same Philox rays.  "
                     "philox_stream: the batch's echogram against the reference's float64 echogram on its own "
                     "stream (different rays: Monte-Carlo difference, large for 1e4-ray jobs)"),
        }

    def reference_cuda():
        ref_cuda = reference_job_loop(population, jobs, picks, accelerator="cuda", precision="float32")
        line["reference_cuda_plain"] = {k: v for k, v in ref_cuda.items() if k != "echograms"}
        if "rirs_per_s" in ref_cuda:
            line["batched_vs_reference_cuda_plain"] = value / ref_cuda["rirs_per_s"]

    def config1():
        line["config1_u_room"] = run_single_scene(args, "u_room_20_boxes", extras_only=True)
        if not args.no_cpu_baseline and world == 1:
            line["config1_u_room"]["single_rir_latency"] = single_rir_latency(workloads.u_furnished(1729))
            line["config1_u_room"]["facade"] = facade_rirs(workloads.u_furnished(1729))

    if not args.no_cpu_baseline:
        guarded("roofline", roofline)
    if not args.no_cpu_baseline and world == 1:
        guarded("cpu_baseline", reference_float64)
        guarded("reference_cuda_plain", reference_cuda)
    if args.with_config1:
        guarded("config1_u_room", config1)
    print(json.dumps(line), flush=True)
    barrier()
    if dist is not None:
        dist.destroy_process_group()
    return 0


def run_serving(args) -> int:
    """Serving: Poisson request streams over the mixed-size population, one line with every rate.

    Requests arrive at each rate of `--rates` (req/s) for `--duration` seconds; 20 % move their source along a
    seeded 3 m path with 8 keyframes.  Scenes are uploaded and tuned before the streams start (a warm,
    resident scene cache).  Latency = arrival to band IRs in host memory.  `--server continuous` (default)
    is the kernel-level continuous batcher (one persistent trace launch fed while it runs, overload shed at
    arrival when the admitted work would miss `--slo` seconds); `--server batched` the batch-level server.
    Each rate runs `--runs` times on fresh arrival seeds.
    """
    import torch
    from acoustic_agent_b200 import serving, workloads
    world, rank, local = _dist_setup()
    if world > 1:
        raise SystemExit("serving runs on one GPU")
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    population = workloads.mixed_batch(1730, 64)
    rates = [float(r) for r in str(args.rates).split(",")] if args.rates else [args.rate]
    if args.server == "continuous":
        server = serving.ContinuousServer(local, slo_s=args.slo, capacity_rb_per_s=args.capacity_rb,
                                          blocks_per_sm=args.service_blocks_per_sm,
                                          reserve_blocks=args.service_reserve_blocks)
    else:
        server = serving.Server(local, max_inflight=args.max_inflight, policy=args.policy,
                                max_batch_rays=args.max_batch_rays, late_tail=args.late_tail,
                                trace_blocks_per_sm=args.trace_blocks_per_sm)
    t0 = time.perf_counter()
    for w in population:   # warm the resident scene cache (upload + tune) before the clock starts
        req = serving.Request(-1, w, [w.sources[0]])
        server.scenes.acquire(w, serving.request_jobs(req)[0])
        server.scenes.release(w)
    warm_s = time.perf_counter() - t0
    warm = serving.requests_from_stream(workloads.request_stream(1, rate_hz=20.0, duration_s=0.4,
                                                                 population=population))
    server.serve(warm, realtime=False)   # kernels, allocator, pinned pool
    table = []
    sampler = ClockSampler(local)
    with sampler:
        for rate in rates:
            for run in range(args.runs):
                stream = workloads.request_stream(1729 + 97 * run, rate_hz=rate, duration_s=args.duration,
                                                  population=population)
                requests = serving.requests_from_stream(stream)
                report = server.serve(requests, realtime=True)
                s = report.summary()
                served = [r for r in report.results if r.error is None]
                table.append({
                    "rate_req_s": rate, "run": run, "requests": len(requests), "admitted": len(served),
                    "rejected": s["rejected"], "offered_rirs_per_s": sum(r.num_rirs for r in requests) / args.duration,
                    "rirs_per_s": s["rirs_per_s"], "ray_bounces_per_s": s["ray_bounces_per_s"],
                    "p50_ms": s["p50_ms"], "p99_ms": s["p99_ms"],
                    "p50_phase_ms": report.phase_ms(50), "p99_phase_ms": report.phase_ms(99),
                    "max_requests_on_gpu": s["max_inflight"], "launches_or_batches": s["batches"]})
    if hasattr(server, "close"):
        server.close()
    by_rate = {}
    for rate in rates:
        rows = [r for r in table if r["rate_req_s"] == rate]
        by_rate[f"{rate:g}"] = {k: float(np.mean([r[k] for r in rows])) for k in
                                ("rirs_per_s", "p50_ms", "p99_ms", "admitted", "rejected", "offered_rirs_per_s")}
    head = by_rate[f"{rates[0]:g}"]
    line = {
        "metric": METRIC, "value": head["rirs_per_s"], "unit": "RIRs/s", "n_gpus": 1, "steps": len(table),
        "warmup": len(warm), "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded scene generator, Poisson arrivals)",
        "config": {"workload": f"serving: Poisson arrivals at {', '.join(f'{r:g}' for r in rates)} req/s for "
                               f"{args.duration:g} s each over 64 mixed scenes, 20% moving sources x 8 keyframes",
                   "server": args.server, "slo_s": args.slo if args.server == "continuous" else None,
                   "runs_per_rate": args.runs},
        "latency_ms": {"p50": head["p50_ms"], "p99": head["p99_ms"]},
        "by_rate": by_rate, "runs": table, "warm_cache_s": warm_s,
        "e2e": {"value": head["rirs_per_s"], "unit": "RIRs/s", "note": "arrival to host band IRs"},
        "clocks": sampler.summary(),
    }
    print(json.dumps(line), flush=True)
    return 0


LATE_FS, LATE_SAMPLES, LATE_CHANNELS = 48000, 96000, 8
LATE_RT60 = (0.72, 0.68, 0.62, 0.57, 0.50, 0.41)
# float64 operations per FDN sample: 96 absorptive sections x 9, Hadamard 64, line writes 32, output mean 17,
# all-pass 16, tone sections 6 x 9 (steam_rt.py:2257-2326)
FDN_FLOPS_PER_SAMPLE = 96 * 9 + 64 + 32 + 17 + 16 + 6 * 9


def late_reverb_inputs(channels: int, seed: int = 1729):
    """Traced band IRs of the U-room RIR set (48 kHz, 2 s, 8 channels): seeded noise under per-band
    exponential decays, each channel with its own RT60 targets, as float32 [6, N] arrays."""
    rng = np.random.default_rng(seed)
    t = np.arange(LATE_SAMPLES) / LATE_FS
    out = []
    for ch in range(channels):
        rt60 = tuple(v * (1.0 + 0.01 * ch) for v in LATE_RT60)
        env = np.stack([np.exp(-3.0 * math.log(10.0) * t / r) for r in rt60])
        out.append((((rng.uniform(-1.0, 1.0, env.shape) * env) * 1e-2).astype(np.float32), rt60))
    return out


def _late_config(seed: int = 1729):
    return types.SimpleNamespace(fs=LATE_FS, seed=seed, late_tail=True, hybrid_transition_s=1.0,
                                 hybrid_overlap_fraction=0.25, rt_bin_duration_s=0.001)


def reference_late_tails(steps: int, warmup: int) -> dict:
    """The reference's _render_parametric_fdn_late_reverb (float64 Numba FDN, one host thread) on one
    channel per step; the oracle's restatement when the reference package is absent."""
    traced, rt60 = late_reverb_inputs(1)[0]
    rt60_bands = dict(zip(("125", "250", "500", "1000", "2000", "4000"), rt60))
    ref, reason = import_reference_package()
    times = []
    if ref is not None:
        steam_rt, models = ref
        cfg = models.SimConfig(fs=LATE_FS, duration_s=2.0, hybrid_transition_s=1.0, hybrid_overlap_fraction=0.25,
                               seed=1729)
        kind, what = "reference", "steam_rt._render_parametric_fdn_late_reverb (baseline/_ref, Numba float64)"
        for k in range(warmup + steps):
            t0 = time.perf_counter()
            steam_rt._render_parametric_fdn_late_reverb(traced, {"bin_duration_s": 0.001}, rt60_bands, cfg)
            if k >= warmup:
                times.append(time.perf_counter() - t0)
    else:
        from oracle import oracle
        kind, what = "port", f"{reason}; oracle restatement (C float64 FDN + numpy)"
        for k in range(warmup + steps):
            t0 = time.perf_counter()
            oracle.late_reverb(traced, 0.001, rt60_bands, fs=LATE_FS, seed=1729, transition_s=1.0,
                               overlap_fraction=0.25)
            if k >= warmup:
                times.append(time.perf_counter() - t0)
    per = float(np.mean(times))
    return {"value": 1.0 / per, "seconds_per_tail": per, "cores": 1, "kind": kind,
            "sample": f"one 48 kHz x 2 s channel per step, {what}, mean of {steps} after {warmup} warm-up"}


def run_late_reverb(args) -> int:
    """Hybrid FDN late tails of the U-room RIR set: 8 channels x 48 kHz x 2 s per step.

    value: ``LateReverbRenderer.render`` with traced band IRs resident (one FDN
    launch + one band split + one mix launch for the 8 tails; designs cached).
    e2e: the reference-facing drop-in ``render_parametric_fdn_late_reverb``
    per channel from host arrays, with a fresh design per call (RT60 changes
    every step), host<->device copies included.  A second launch of 1184 FDN
    impulses (8 per SM) gives the network's saturated throughput.
    """
    import torch
    from acoustic_agent_b200 import _lib, late_reverb, runtime
    world, rank, local = _dist_setup()
    if world > 1:
        raise SystemExit("late_reverb runs on one GPU")
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    stream = torch.cuda.current_stream(device)
    inputs = late_reverb_inputs(LATE_CHANNELS)
    r = late_reverb.LateReverbRenderer(local)
    traced = [torch.from_numpy(t.astype(np.float64)).to(device) for t, _ in inputs]
    jobs = [late_reverb.LateReverbJob(t, torch.empty(t.shape, dtype=torch.float32, device=device),
                                      torch.empty(t.shape, dtype=torch.float32, device=device), LATE_FS, 1729, rt60,
                                      0.001, 1.0, 0.25) for t, (_, rt60) in zip(traced, inputs)]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)
    for _ in range(args.warmup):
        r.render(jobs, stream=stream)
    torch.cuda.synchronize()
    fdn_ms, steps_ms = [], []
    sampler = ClockSampler(local)
    with sampler:
        for k in range(args.steps):
            flush.fill_(k & 0xFF)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            ev[0].record(stream)
            r.render(jobs, stream=stream, fdn_events=(ev[1], ev[2]))
            ev[3].record(stream)
            ev[3].synchronize()
            steps_ms.append(ev[0].elapsed_time(ev[3]))
            fdn_ms.append(ev[1].elapsed_time(ev[2]))
    step_ms = float(np.mean(steps_ms))
    fdn_kernel_ms = float(np.mean(fdn_ms))
    design = r.design(LATE_FS, 1729, inputs[0][1])
    samples_per_tail = LATE_SAMPLES + design.preroll
    fdn_flops = FDN_FLOPS_PER_SAMPLE * samples_per_tail * LATE_CHANNELS
    # saturated FDN throughput: 1184 impulses in one launch
    sat_jobs = 8 * torch.cuda.get_device_properties(device).multi_processor_count
    designs = [r.design(LATE_FS, 1729, rt60) for _, rt60 in inputs]
    sat_out = torch.empty(sat_jobs, LATE_SAMPLES, dtype=torch.float64, device=device)
    arr = (_lib.ACFdnJob * sat_jobs)()
    for k in range(sat_jobs):
        d = designs[k % len(designs)]
        arr[k].absorptive[:] = d.absorptive.reshape(-1).tolist()
        arr[k].tone[:] = d.tone.reshape(-1).tolist()
        arr[k].delays[:] = [int(v) for v in d.delays]
        arr[k].allpass_delays[:] = list(d.allpass)
        arr[k].num_samples = LATE_SAMPLES
        arr[k].preroll = d.preroll
        arr[k].out = sat_out[k].data_ptr()
    ws = runtime.FdnWorkspace(device)
    for _ in range(2):
        runtime.fdn_impulse(arr, sat_jobs, ws, stream=stream)
    torch.cuda.synchronize()
    sat_ms = []
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        runtime.fdn_impulse(arr, sat_jobs, ws, stream=stream)
        e1.record(stream)
        e1.synchronize()
        sat_ms.append(e0.elapsed_time(e1))
    sat = float(np.median(sat_ms))
    sat_flops = FDN_FLOPS_PER_SAMPLE * samples_per_tail * sat_jobs
    del sat_out
    # end to end through the drop-in, a new RT60 (so a new design) every call
    h2d = d2h = 0
    e2e_times = []
    for k in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for ch, (t, rt60) in enumerate(inputs):
            bands_rt60 = dict(zip(("125", "250", "500", "1000", "2000", "4000"), (v * (1.0 + 1e-6 * k) for v in rt60)))
            out, comp, _ = late_reverb.render_parametric_fdn_late_reverb(t, {"bin_duration_s": 0.001}, bands_rt60,
                                                                         _late_config())
            if k == 0:
                h2d += t.size * 8
                d2h += out.nbytes + comp.nbytes + 6 * _lib.AC_LATE_STATS * 8
        if k >= args.warmup:
            e2e_times.append(time.perf_counter() - t0)
    e2e_step = float(np.mean(e2e_times))
    cpu = None if args.no_cpu_baseline else reference_late_tails(2, 1)
    # the FDN's float64 adds and multiplies are separate instructions (bit-exact order), so its roof is the
    # measured float64 add/multiply issue rate, one operation each
    peak_fp64 = runtime.fp64_rate_tops(device)
    achieved = fdn_flops / (fdn_kernel_ms * 1e-3) / 1e12
    sat_achieved = sat_flops / (sat * 1e-3) / 1e12
    line = {
        "metric": "late tails/s", "value": LATE_CHANNELS / (step_ms * 1e-3), "unit": "tails/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded decaying noise)",
        "config": {"workload": "late_reverb: hybrid FDN tails of the U-room RIR set, 8 channels x 48 kHz x 2 s, "
                               "transition 1 s, overlap 0.25", "samples_per_tail": LATE_SAMPLES,
                   "fdn_samples_per_tail": samples_per_tail, "l2": "256 MiB buffer written between steps"},
        "fdn_kernel_ms": fdn_kernel_ms,
        "fdn_cycles_per_sample": fdn_kernel_ms * 1e-3 * sampler.median_mhz() * 1e6 / samples_per_tail
        if sampler.median_mhz() else None,
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak_fp64, "unit": "T float64 ops/s",
                     "frac": achieved / peak_fp64, "traffic": None,
                     "note": "FDN kernel; peak = measured float64 add/multiply issue rate (ac_fp64_rate_probe); "
                             "8 tails occupy 8 of 148 SMs and run latency-bound"},
        "saturated_fdn": {"tails": sat_jobs, "ms": sat, "tails_per_s": sat_jobs / (sat * 1e-3),
                          "achieved_t_ops": sat_achieved, "frac_of_measured_fp64": sat_achieved / peak_fp64},
        "e2e": {"value": LATE_CHANNELS / e2e_step, "unit": "tails/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "note": "drop-in per channel from host arrays, new design per call"},
        "cpu_baseline": None if cpu is None else {"value": cpu["value"], "unit": "tails/s", "cores": cpu["cores"],
                                                  "kind": cpu["kind"], "sample": cpu["sample"]},
        "gpu_launches": 3 * args.steps,
        "clocks": sampler.summary(),
    }
    print(json.dumps(line), flush=True)
    return 0


DIRECT_PAIRS = 1024


def direct_pairs(workload, count: int, seed: int = 11) -> list[tuple[np.ndarray, np.ndarray]]:
    """Seeded source/listener pairs inside the workload's footprint (0.3 m off floor and ceiling)."""
    corners = np.asarray(workload.spec["corners"], dtype=float)
    lo, hi = corners.min(axis=0), corners.max(axis=0)
    h = float(workload.spec["height"])
    rng = np.random.default_rng(seed)
    return [(np.r_[rng.uniform(lo, hi), rng.uniform(0.3, h - 0.3)], np.r_[rng.uniform(lo, hi), rng.uniform(0.3, h - 0.3)])
            for _ in range(count)]


def reference_direct(workload, pairs, steps: int) -> dict:
    """The reference's simulate_direct (Python surface objects, one host thread) on the first pairs."""
    ref, reason = import_reference_package()
    if ref is None:
        return {"unavailable": reason}
    steam_rt, models = ref
    scene = reference_scene(steam_rt, models, workload.spec)
    cfg = models.SimConfig()
    steam_rt.simulate_direct(scene, pairs[0][0], pairs[0][1], cfg, "cardioid")
    t0 = time.perf_counter()
    for src, lst in pairs[:steps]:
        steam_rt.simulate_direct(scene, src, lst, cfg, "cardioid")
    per = (time.perf_counter() - t0) / steps
    return {"value": 1.0 / per, "seconds_per_pair": per, "cores": 1, "kind": "reference",
            "sample": f"{steps} pairs of {workload.name}, steam_rt.simulate_direct (baseline/_ref), one host thread"}


def run_direct(args) -> int:
    """Direct sound of 1024 seeded source/listener pairs in the furnished U room per step.

    value: one ac_direct launch over the pairs (scene and tables resident;
    volumetric occlusion with 32 samples, 8 transmission layers), device time.
    e2e: the batch drop-in simulate_direct_batch from host arrays to the
    reference's result dicts.  The reference's Python simulate_direct runs
    beside it on a sample of the pairs.
    """
    import torch
    from acoustic_agent_b200 import _lib, direct, runtime, workloads
    world, rank, local = _dist_setup()
    if world > 1:
        raise SystemExit("the direct workload runs on one GPU")
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    w = workloads.u_furnished(1729)
    pairs = direct_pairs(w, DIRECT_PAIRS)
    cfg = types.SimpleNamespace(direct_occlusion=True, direct_occlusion_mode="volumetric", direct_occlusion_radius_m=0.1,
                                direct_occlusion_samples=32, direct_transmission=True, num_transmission_rays=8,
                                min_distance_m=1.0, c=343.0, rt_cuda_device=local)
    ref, why = import_reference_package()
    if ref is None:
        raise SystemExit(f"the direct workload needs the reference scene objects: {why}")
    steam_rt, models = ref
    ref_scene = reference_scene(steam_rt, models, w.spec)
    device_scene = runtime.DeviceScene(steam_rt._scene_kernel_arrays(ref_scene), device=local)
    names, transmission = direct.scene_surfaces(ref_scene)
    tables = direct.DirectTables(names, transmission, device)
    queries = (_lib.ACDirectQuery * len(pairs))()
    for k, (a, b) in enumerate(pairs):
        queries[k] = direct.make_query(a, b, cfg)
    stream = torch.cuda.current_stream(device)
    for _ in range(args.warmup):
        direct.run_queries(device_scene, tables, queries, len(pairs), samples=32, stream=stream)
    times = []
    sampler = ClockSampler(local)
    with sampler:
        for _ in range(args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            # device time of the launch alone (the table copy and the result read are in e2e)
            lib = _lib.load()
            t = _lib.ACDirectTables()
            t.unit_samples = tables.samples(32).data_ptr()
            t.num_samples = 32
            t.transmission = tables.transmission.data_ptr()
            t.surface_group = tables.groups.data_ptr()
            size = ctypes.c_size_t()
            lib.ac_direct_workspace_size(len(pairs), ctypes.byref(size))
            ws = torch.empty(int(size.value), dtype=torch.uint8, device=device)
            res = torch.empty(len(pairs) * ctypes.sizeof(_lib.ACDirectResult), dtype=torch.uint8, device=device)
            staging = torch.empty(int(size.value), dtype=torch.uint8, pin_memory=True)
            e0.record(stream)
            _lib.check(lib.ac_direct(device_scene.handle, queries, len(pairs), ctypes.byref(t),
                                     ctypes.c_void_p(res.data_ptr()), ctypes.c_void_p(ws.data_ptr()), ws.numel(),
                                     ctypes.c_void_p(staging.data_ptr()), ctypes.c_void_p(stream.cuda_stream)),
                       "ac_direct")
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
    step_ms = float(np.median(times))
    e2e = []
    for _ in range(max(3, args.steps)):
        t0 = time.perf_counter()
        direct.direct_results(device_scene, tables, pairs, cfg, "cardioid")
        e2e.append(time.perf_counter() - t0)
    e2e_s = float(np.median(e2e))
    cpu = None if args.no_cpu_baseline else reference_direct(w, pairs, 40)
    line = {
        "metric": "direct paths/s", "value": len(pairs) / (step_ms * 1e-3), "unit": "paths/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded pairs)",
        "config": {"workload": f"direct: {len(pairs)} source/listener pairs in the furnished U room "
                               f"({len(names)} surfaces), volumetric occlusion 32 samples, 8 transmission layers"},
        "e2e": {"value": len(pairs) / e2e_s, "unit": "paths/s", "h2d_bytes_per_step": len(pairs) * 72,
                "d2h_bytes_per_step": len(pairs) * 64, "note": "direct_results from host pairs to result dicts"},
        "cpu_baseline": None if cpu is None or "unavailable" in cpu else {
            "value": cpu["value"], "unit": "paths/s", "cores": 1, "kind": "reference", "sample": cpu["sample"]},
        "gpu_launches": args.steps, "clocks": sampler.summary(),
    }
    print(json.dumps(line), flush=True)
    device_scene.close()
    return 0


BVH_SURFACES = 1 << 20
BVH_SAMPLE = 1 << 16


def bvh_build_inputs(n: int, seed: int = 2024) -> tuple[np.ndarray, np.ndarray]:
    """Padded surface AABBs of a seeded 400 x 400 m warehouse floor (steam_rt.py:234-262 pads by 2e-6).

    Seven in eight surfaces are rotated boxes (side 0.3-2 m, height up to 3 m, the
    reference's cabinet proxies); the rest are wall pieces on a 2 m grid, whose
    shared grid coordinates give the sorts many exact ties.
    """
    rng = np.random.default_rng(seed)
    boxes = n - n // 8
    centre = rng.uniform(0.0, 400.0, (boxes, 2))
    half = rng.uniform(0.15, 1.0, (boxes, 2))
    angle = rng.uniform(0.0, np.pi / 2, boxes)
    c, s = np.abs(np.cos(angle)), np.abs(np.sin(angle))
    ext = np.stack([half[:, 0] * c + half[:, 1] * s, half[:, 0] * s + half[:, 1] * c], axis=1)
    z1 = rng.uniform(0.4, 3.0, boxes)
    lo_b = np.column_stack([centre - ext, np.zeros(boxes)])
    hi_b = np.column_stack([centre + ext, z1])
    walls = n - boxes
    a = rng.integers(0, 200, (walls, 2)).astype(np.float64) * 2.0
    horizontal = rng.random(walls) < 0.5
    b = a + np.where(horizontal[:, None], [2.0, 0.0], [0.0, 2.0])
    lo_w = np.column_stack([np.minimum(a, b), np.zeros(walls)])
    hi_w = np.column_stack([np.maximum(a, b), np.full(walls, 3.0)])
    lo = np.concatenate([lo_b, lo_w]) - 2e-6
    hi = np.concatenate([hi_b, hi_w]) + 2e-6
    order = rng.permutation(n)
    return np.ascontiguousarray(lo[order]), np.ascontiguousarray(hi[order])


def reference_bvh(steps: int) -> dict:
    """The reference's build_bvh (bvh.py:8-77, baseline/_ref) on the first BVH_SAMPLE surfaces, one host thread."""
    ref, why = import_reference_package()
    if ref is None:
        return {"unavailable": why}
    from acoustic_agent.bvh import build_bvh  # the reference package put on sys.path above
    lo, hi = bvh_build_inputs(BVH_SURFACES)
    lo, hi = lo[:BVH_SAMPLE], hi[:BVH_SAMPLE]
    build_bvh(lo[:4096], hi[:4096])
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        build_bvh(lo, hi)
        times.append(time.perf_counter() - t0)
    per = float(np.median(times))
    return {"value": BVH_SAMPLE / per, "seconds": per, "cores": 1, "kind": "reference",
            "sample": f"the first {BVH_SAMPLE} of the {BVH_SURFACES} warehouse surfaces, acoustic_agent.bvh.build_bvh "
                      f"(baseline/_ref), one host thread, median of {steps}"}


def run_bvh_build(args) -> int:
    """The reference's BVH over 2^20 warehouse surfaces, built on the GPU (ac_bvh_build_device).

    value: surfaces/s of one build from resident device bounds to the device
    tree (keys kernel, cooperative large-node kernel, subtree kernel), device
    time, L2 flushed between steps.  e2e: the drop-in bvh.build_bvh from numpy
    bounds to the numpy dict (bounds up, tree down).  The oracle (the numpy
    restatement of the same recursion) and the host C++ builder run beside it.
    """
    import torch
    from acoustic_agent_b200 import _lib, bvh
    from oracle import oracle
    world, rank, local = _dist_setup()
    if world > 1:
        raise SystemExit("the bvh_build workload runs on one GPU")
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    lo, hi = bvh_build_inputs(BVH_SURFACES)
    b = bvh.builder(local)
    dlo, dhi = torch.from_numpy(lo).to(device), torch.from_numpy(hi).to(device)
    tree = b.build(dlo, dhi)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=device)
    for _ in range(args.warmup):
        b.build(dlo, dhi, check=False)
    sampler = ClockSampler(local)
    with sampler:
        times = _device_timed(lambda: b.build(dlo, dhi, check=False), args.steps, device, flush)
    if int(b.status.item()) != 0:
        raise SystemExit(f"device BVH build failed (status {int(b.status.item())})")
    step_ms = float(np.median(times))
    e2e = []
    for _ in range(max(3, args.steps)):
        t0 = time.perf_counter()
        bvh.build_bvh(lo, hi)
        e2e.append(time.perf_counter() - t0)
    e2e_s = float(np.median(e2e))
    t0 = time.perf_counter()
    host = _lib.build_bvh(lo, hi, 4)
    host_s = time.perf_counter() - t0
    assert host["node_count"] == tree.node_count
    nodes = tree.node_count
    # algorithmic bytes of one build: bounds in (48 B/surface), tree out (72 B/node + 8 B/surface)
    algo_bytes = 48 * BVH_SURFACES + 72 * nodes + 8 * BVH_SURFACES
    peaks = _peaks()
    achieved = algo_bytes / (step_ms * 1e-3) / 1e9
    cpu = None
    if not args.no_cpu_baseline:
        t0 = time.perf_counter()
        oracle.build_bvh(lo[:BVH_SAMPLE], hi[:BVH_SAMPLE])
        port_s = time.perf_counter() - t0
        cpu = {"value": BVH_SAMPLE / port_s, "unit": "surfaces/s", "cores": 1, "kind": "port",
               "sample": f"the first {BVH_SAMPLE} surfaces, oracle.build_bvh (numpy restatement), one host thread, "
                         f"one run"}
    line = {
        "metric": "BVH surfaces/s", "value": BVH_SURFACES / (step_ms * 1e-3), "unit": "surfaces/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded warehouse AABBs)",
        "config": {"workload": f"bvh_build: the reference's BVH (leaf 4) over {BVH_SURFACES} warehouse surfaces, "
                               f"{nodes} nodes, depth {tree.max_depth}",
                   "l2": "flushed between timed steps (256 MiB write)"},
        "e2e": {"value": BVH_SURFACES / e2e_s, "unit": "surfaces/s", "h2d_bytes_per_step": 48 * BVH_SURFACES,
                "d2h_bytes_per_step": 72 * nodes + 8 * BVH_SURFACES,
                "note": "bvh.build_bvh from numpy bounds to the numpy dict"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "traffic": _profiled_value("bvh_build_warehouse_1m",
                                                                                    "traffic_bytes_per_build_1m"),
                     "traffic_note": "DRAM bytes of the four kernels at 2^18 surfaces (ncu), times 4",
                     "peak_source": peaks["source"], "kernel": "the whole build (4 launches)",
                     "algorithmic_bytes": algo_bytes},
        "cpu_baseline": cpu,
        "host_builder": {"seconds": host_s, "value": BVH_SURFACES / host_s, "unit": "surfaces/s",
                         "note": "ac_bvh_build, the C++ restatement, one host thread, full size"},
        "gpu_launches": 4 * args.steps, "clocks": sampler.summary(),
    }
    print(json.dumps(line), flush=True)
    return 0


def _profiled_value(summary: str, key: str):
    """A `key: number` line of a committed profile summary (profiles/<summary>.md), or None."""
    path = REPO / "profiles" / f"{summary}.md"
    if not path.exists():
        return None
    for text in path.read_text().splitlines():
        if text.strip().lower().startswith(key + ":"):
            try:
                return float(text.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


def _cpu_baseline(port, ref_cpu):
    """The reference's float64 Numba path on the host cores; the C restatement when the package is absent."""
    if ref_cpu and "unavailable" not in ref_cpu:
        return {"value": ref_cpu["value"], "unit": "RIRs/s", "cores": ref_cpu["threads"], "kind": "reference",
                "sample": ref_cpu["sample"],
                "port": ({"value": port["value"], "cores": port["cores"], "sample": port["sample"]} if port else None)}
    if port:
        return {"value": port["value"], "unit": "RIRs/s", "cores": port["cores"], "kind": "port",
                "sample": port["sample"]}
    return None


def _reference_cuda_line(ref_cuda):
    """The reference's own Numba-CUDA float32 backend on this GPU (trace on the GPU, synthesis on the host)."""
    if not ref_cuda:
        return None
    if "unavailable" in ref_cuda:
        return {"unavailable": ref_cuda["unavailable"]}
    return {"value": ref_cuda["value"], "unit": "RIRs/s", "seconds_per_rir": ref_cuda["seconds_per_rir"],
            "trace_seconds_per_rir": ref_cuda["trace_seconds"], "sample": ref_cuda["sample"]}


def l2_read_gbs(device) -> float:
    """Measured L2 read bandwidth: 16-byte loads cached in L2 only over a 32 MiB buffer (ac_read_bandwidth_probe).

    The tracer's scenes (tens of KB) live in L1/L2, so this, beside the HBM
    copy peak, is the roof its node and surface fetches run against.
    """
    from acoustic_agent_b200 import runtime
    return runtime.read_bandwidth_gbs(device, 32 << 20)


# Figures of the trace launch read from one ncu capture of the same kernel code, per workload (constants,
# recorded with the summary that gives them and the commit of the kernel it measured): issue-active fraction,
# SIMT efficiency (thread instructions per warp instruction / 32) and DRAM bytes per ray-bounce
# (dram__bytes_read.sum + dram__bytes_write.sum of the captured launch over its ray-bounces).
PROFILED = {
    "u_room_20_boxes": {"issue_active": 0.6706, "simt_efficiency": 14.41 / 32.0,
                        "dram_bytes_per_ray_bounce": (3123456 + 734208) / 52028160,
                        "profile": "profiles/trace_kernel_u_room_20_boxes.md", "kernel_commit": "2860a90"},
    "mixed_batch": {"issue_active": 0.6255, "simt_efficiency": 13.11 / 32.0,
                    "dram_bytes_per_ray_bounce": (32922624 + 1248512) / 2209616616,
                    "profile": "profiles/trace_kernel_mixed_batch_24_scenes.md", "kernel_commit": "2860a90"},
}


def roofline_line(achieved: float, bytes_per_rb: float, workload: str, device, ray_bounces: int) -> dict:
    """The trace launch's roofline.

    `achieved` = algorithmic bytes of one launch (the reference traversal's node, surface and material fetches
    per ray-bounce x the launch's ray-bounces) over its CUDA-event duration.  Scenes are kilobytes, so those
    bytes are served from L1/L2 and the memory roof is the L2 read rate measured in this run; the HBM copy
    peak is given beside it.  The launch is issue-bound (divergent per-lane traversal), which the ncu figures
    of the same kernel show: `bound` says so and `frac` is taken against the L2 roof.
    """
    peaks = _peaks()
    l2 = l2_read_gbs(device)
    prof = PROFILED.get(workload)
    out = {"bound": "issue", "achieved": achieved, "peak": l2, "unit": "GB/s", "frac": achieved / l2,
           "traffic": prof["dram_bytes_per_ray_bounce"] * ray_bounces if prof else None,
           "peak_source": "measured in this run: L2-cached 16-byte loads over a 32 MiB buffer (ac_read_bandwidth_probe)",
           "hbm_peak": peaks["hbm_gbs"], "hbm_peak_source": peaks["source"], "frac_of_hbm": achieved / peaks["hbm_gbs"],
           "kernel": "trace_fast_kernel (ac_trace_batch)", "bytes_per_ray_bounce": bytes_per_rb}
    if prof:
        out.update({"issue_active": prof["issue_active"], "simt_efficiency": prof["simt_efficiency"],
                    "ncu_profile": prof["profile"], "ncu_kernel_commit": prof["kernel_commit"],
                    "traffic_basis": "DRAM bytes per ray-bounce of the profiled launch x this launch's ray-bounces"})
    return out


if __name__ == "__main__":
    raise SystemExit(main())
