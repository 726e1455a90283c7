"""Host logic of the serving path that needs no GPU: request streams, the jobs of a request, footprints, and
the continuous server's scene map (the device scene is a stand-in)."""
from __future__ import annotations

import numpy as np
import pytest

from acoustic_agent_b200 import rng, serving, workloads
from acoustic_agent_b200.scene import point_in_polygon


@pytest.fixture(scope="module")
def population():
    return workloads.mixed_batch(1730, 12)


def test_request_streams_are_seeded_poisson_arrivals(population):
    a = workloads.request_stream(5, rate_hz=200.0, duration_s=2.0, population=population)
    b = workloads.request_stream(5, rate_hz=200.0, duration_s=2.0, population=population)
    assert [(e["arrival_s"], e["workload"].name, e["moving"]) for e in a] == \
           [(e["arrival_s"], e["workload"].name, e["moving"]) for e in b]
    times = np.array([e["arrival_s"] for e in a])
    assert np.all(np.diff(times) > 0) and times[-1] <= 2.0
    assert 250 < len(a) < 550                                  # 400 expected
    moving = [e for e in a if e["moving"]]
    assert 0.1 < len(moving) / len(a) < 0.3                    # 20 % expected
    for e in a:
        assert len(e["sources"]) == (8 if e["moving"] else 1)
        corners = e["workload"].spec["corners"]
        for src in e["sources"]:                               # keyframes stay inside the room outline
            assert point_in_polygon(src[:2], corners)


def test_request_jobs_are_keyed_by_request_and_keyframe(population):
    stream = workloads.request_stream(6, rate_hz=100.0, duration_s=1.0, population=population)
    requests = serving.requests_from_stream(stream)
    seen = set()
    for req in requests:
        specs = serving.request_jobs(req)
        assert len(specs) == len(req.sources) * len(req.workload.listeners) == req.num_rirs
        keys = [s.stream_key for s in specs]
        per_keyframe = len(req.workload.listeners)
        for k in range(len(req.sources)):                       # one key per keyframe, shared by its channels
            block = keys[k * per_keyframe:(k + 1) * per_keyframe]
            assert set(block) == {rng.stream_key(req.workload.name, req.id, k)}
        assert not seen & set(keys)                              # distinct from every other request's
        seen |= set(keys)
        again = serving.request_jobs(req)                       # the same request, the same jobs
        assert [s.stream_key for s in again] == keys
        assert all(s.rng == "philox" and s.precision == "float32" for s in specs)
        for s in specs:
            assert s.direct_delay == pytest.approx(np.linalg.norm(s.source - s.listener) / s.speed_of_sound)


def test_job_footprint_grows_with_the_work_it_holds(population):
    req = serving.requests_from_stream(workloads.request_stream(7, rate_hz=50.0, duration_s=0.5,
                                                                population=population))[0]
    spec = serving.request_jobs(req)[0]
    fs = req.workload.config.fs
    base = serving.job_bytes(spec, fs, 100)
    assert serving.job_bytes(spec, fs, 1000) > base              # per-surface outputs
    assert serving.job_bytes(spec, fs, 100, late_tail=True) > base
    from dataclasses import replace
    assert serving.job_bytes(replace(spec, num_bins=2 * spec.num_bins), fs, 100) > base


class FakeScene:
    device_bytes = 1 << 20

    def __init__(self, arrays, device=0, **options):
        self.options = options
        self.closed = False

    def close(self):
        assert not self.closed
        self.closed = True


def test_continuous_scene_map_reuses_and_bounds_compiled_arrays(monkeypatch, population):
    from acoustic_agent_b200 import runtime
    monkeypatch.setattr(runtime, "DeviceScene", FakeScene)
    cache = serving.SceneCache(0, tune=False)
    cache.max_arrays = 4
    req = serving.requests_from_stream(workloads.request_stream(8, rate_hz=50.0, duration_s=0.5,
                                                                population=population))[0]
    spec = serving.request_jobs(req)[0]
    scene = cache.acquire(req.workload, spec)
    assert cache.acquire(req.workload, spec) is scene and cache.hits == 1 and cache.misses == 1
    cache.release(req.workload)
    cache.release(req.workload)
    for w in population:                                         # more workloads than the map may hold
        cache.key_of(w)
    assert len(cache.arrays) <= 4
