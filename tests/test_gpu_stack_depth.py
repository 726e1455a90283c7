"""The traversal stack depth is a schedule knob: every depth a scene allows gives the same rays and bins.

Each lane's BVH traversal stack lives in the launch's dynamic shared memory,
`stack_entries` deep (ac_trace_params / ac_batch_config / ac_service_config).
The builder reports the entries a ray can need (`bvh_stack_need`, sentinel
included); any depth from there to 32 bounds every push, so the visiting order
and therefore the closest hits, counters and fixed-point bins do not change.
The autotuner times the depths per scene and records its choice.
"""
from __future__ import annotations

from dataclasses import replace

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rt():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from acoustic_agent_b200 import runtime
    return runtime


def _workload_jobs(w, rays, bounces):
    from acoustic_agent_b200 import batching, scene as scene_mod
    specs, jobs = batching.workload_jobs([w])
    arrays = scene_mod.compile_scene(specs[0])
    spec = replace(jobs[0].spec, num_rays=rays, num_bounces=bounces, rng="philox", precision="float32")
    return arrays, spec


def _scenes():
    from acoustic_agent_b200 import workloads
    return {"u_room": _workload_jobs(workloads.u_furnished(channels=1), 20_000, 100),
            "apartment": _workload_jobs(workloads.apartment(rooms=8), 20_000, 200)}


@pytest.mark.parametrize("name", ["u_room", "apartment"])
@pytest.mark.parametrize("width", [2, 4])
def test_every_stack_depth_traces_the_same_rays(rt, name, width):
    from acoustic_agent_b200 import autotune
    arrays, spec = _scenes()[name]
    scene = rt.DeviceScene(arrays, traversal="bvh", bvh_width=width)
    try:
        need = scene.bvh_stack_need
        assert scene.bvh_nodes > 0 and 2 <= need <= rt.MAX_STACK_ENTRIES
        got = {}
        for entries in autotune.stack_candidates(need):
            buffers = rt.trace(scene, replace(spec, stack_entries=entries), record_rays=True)
            torch.cuda.synchronize()
            got[entries] = (buffers.ray_surfaces.cpu().numpy(), buffers.echogram_fx.cpu().numpy(),
                            buffers.hit_counts.cpu().numpy(), buffers.counters.cpu().numpy())
        ref = got[rt.MAX_STACK_ENTRIES]
        for entries, arrays_out in got.items():
            for a, b, what in zip(arrays_out, ref, ("rays", "echogram", "hits", "counters")):
                np.testing.assert_array_equal(a, b, err_msg=f"{name} width {width}: {entries} entries, {what}")
    finally:
        scene.close()


def test_batched_launch_at_the_smallest_common_depth(rt):
    """One launch over both scenes at the larger of their needs equals each scene traced alone at 32."""
    scenes = _scenes()
    dev = torch.device("cuda", 0)
    jobs, alone = [], []
    for arrays, spec in scenes.values():
        scene = rt.DeviceScene(arrays, traversal="bvh")
        jobs.append((scene, spec, rt.TraceBuffers.allocate(scene.num_surfaces, int(spec.num_bins), dev)))
        alone.append(rt.trace(scene, replace(spec, stack_entries=rt.MAX_STACK_ENTRIES)))
    try:
        need = max(s.bvh_stack_need for s, _, _ in jobs)
        rt.trace_batch(jobs, rt.BatchWorkspace(dev), stack_entries=need)
        torch.cuda.synchronize()
        for (_, _, b), a in zip(jobs, alone):
            np.testing.assert_array_equal(b.echogram_fx.cpu().numpy(), a.echogram_fx.cpu().numpy())
            np.testing.assert_array_equal(b.counters.cpu().numpy()[:4], a.counters.cpu().numpy()[:4])
        with pytest.raises(ValueError, match="stack_entries"):
            rt.trace_batch(jobs, rt.BatchWorkspace(dev), stack_entries=need - 1)
    finally:
        for s, _, _ in jobs:
            s.close()


def test_a_stack_below_the_need_is_refused_before_any_launch(rt):
    arrays, spec = _scenes()["apartment"]
    spec = replace(spec, num_rays=256)
    scene = rt.DeviceScene(arrays, traversal="bvh")
    try:
        for bad in (scene.bvh_stack_need - 1, rt.MAX_STACK_ENTRIES + 1, -1):
            with pytest.raises(ValueError, match="stack_entries"):
                rt.trace(scene, replace(spec, stack_entries=bad))
        with pytest.raises(ValueError, match="stack_entries"):
            rt.DeviceScene(arrays, traversal="bvh", stack_entries=scene.bvh_stack_need - 1)
        service = rt.TraceService(0, capacity=64, stack_entries=scene.bvh_stack_need - 1)
        try:
            buffers = rt.TraceBuffers.allocate(scene.num_surfaces, int(spec.num_bins), torch.device("cuda", 0))
            with pytest.raises(ValueError, match="stack entries"):
                service.submit([(scene, spec, buffers)])
        finally:
            service.close()
    finally:
        scene.close()


def test_tuner_records_a_stack_depth_per_scene(rt):
    from acoustic_agent_b200 import autotune
    arrays, spec = _scenes()["apartment"]
    cache = autotune.TuneCache()
    choice = autotune.tune_scene(arrays, spec, sample_rays=4096, reps=2, cache=cache)
    if choice.traversal == "scan":
        assert choice.stack_entries == 0
        return
    timed = dict(choice.stack_ms)
    assert choice.stack_entries in timed and choice.ms == timed[choice.stack_entries]
    scene = rt.DeviceScene(arrays, **choice.options())
    try:
        assert scene.stack_entries == choice.stack_entries >= scene.bvh_stack_need
        assert sorted(timed) == autotune.stack_candidates(scene.bvh_stack_need)
    finally:
        scene.close()
    assert cache.get(autotune.fingerprint(arrays)) == choice
