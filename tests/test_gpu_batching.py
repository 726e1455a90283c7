"""Batched rendering: a job's band IRs do not depend on what else is in the batch.

Every job's rays are keyed by (seed, stream key, ray index), its echogram bins
are exact fixed-point sums, and its synthesis noise is keyed by its own seed,
so one persistent launch over a mixed batch and the same job rendered alone
give bit-identical band IRs.  These tests run mixed-size batches (one to
several rooms, linear and BVH scenes, several sources and channels, different
lengths) through RIRRenderer eagerly and as a CUDA graph.
"""
from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mix():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from acoustic_agent_b200 import batching, scene, workloads
    population = workloads.mixed_batch(11, 6, max_rays=20_000, min_rays=2_000)
    specs, jobs = batching.workload_jobs(population)
    arrays = [scene.compile_scene(s) for s in specs]
    return batching, arrays, jobs


def _render(batching, arrays, jobs, graph=False):
    renderer = batching.RIRRenderer(0)
    plan = renderer.plan(arrays, jobs)
    if graph:
        renderer.capture(plan)
    renderer.launch(plan)
    torch.cuda.synchronize()
    out = renderer.results(plan)
    rb = [int(b.counters[2].item()) for b in plan.buffers]
    for s in plan.scenes:
        s.close()
    return out, rb


def test_mixed_batch_equals_each_job_alone(mix):
    batching, arrays, jobs = mix
    assert len({j.scene_index for j in jobs}) > 1 and len({j.spec.num_bins for j in jobs}) > 1
    together, rb = _render(batching, arrays, jobs)
    picks = sorted({0, len(jobs) // 2, len(jobs) - 1})
    for k in picks:
        job = jobs[k]
        alone, rb_alone = _render(batching, [arrays[job.scene_index]],
                                  [batching.Job(0, job.spec, job.fs, job.workload, job.source, job.channel)])
        assert rb_alone[0] == rb[k]
        np.testing.assert_array_equal(alone[0], together[k])
        assert np.isfinite(together[k]).all() and np.abs(together[k]).max() > 0


def test_graph_replay_equals_eager_launch(mix):
    batching, arrays, jobs = mix
    eager, _ = _render(batching, arrays, jobs)
    graphed, _ = _render(batching, arrays, jobs, graph=True)
    for a, b in zip(eager, graphed):
        np.testing.assert_array_equal(a, b)


def test_pipelined_steps_synthesise_the_previous_trace(mix):
    """A pipelined step traces every job beside the synthesis of the previous step's echograms."""
    batching, arrays, jobs = mix
    renderer = batching.RIRRenderer(0)
    plan = renderer.plan(arrays, jobs)
    renderer.launch(plan)
    torch.cuda.synchronize()
    expected = renderer.results(plan)
    plan.ir_store.fill_(float("nan"))
    renderer.launch_pipelined(plan)          # eager: synthesises the echograms traced by launch()
    torch.cuda.synchronize()
    for a, b in zip(renderer.results(plan), expected):
        np.testing.assert_array_equal(a, b)
    renderer.capture_pipelined(plan)
    plan.ir_store.fill_(float("nan"))
    for _ in range(2):
        renderer.launch_pipelined(plan)      # graph replays
    torch.cuda.synchronize()
    for a, b in zip(renderer.results(plan), expected):
        np.testing.assert_array_equal(a, b)
    for s in plan.scenes:
        s.close()
