"""Continuous batching at kernel level: the trace service (ac_service_*) and the server built on it.

A persistent trace launch takes jobs from a device ring while the host appends
more.  Each job's outputs must equal the same job traced alone (exact
fixed-point sums), whether it was submitted before the launch started or
while it ran; every wait in the launch is bounded, so an idle launch ends by
itself and the next submission starts another; a full ring asks the caller
to poll first.  The server on top admits requests as they arrive and each
served request equals the request rendered alone.
"""
from __future__ import annotations

import time
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


def _jobs(rt, rays=(30_000, 4_000, 60_000, 7_000)):
    from acoustic_agent_b200 import batching, scene as scene_mod, workloads
    ws = [workloads.u_furnished(11, rays=1, bounces=60, channels=2),
          workloads.apartment(12, rays=1, bounces=120, rooms=3, fs=16000, duration=1.0, bin_duration=0.01)]
    specs, jobs = batching.workload_jobs(ws)
    scenes = [rt.DeviceScene(scene_mod.compile_scene(s)) for s in specs]
    out = []
    for k, j in enumerate(jobs):
        spec = replace(j.spec, num_rays=rays[k % len(rays)], stream_key=1000 + k)
        out.append((scenes[j.scene_index], spec))
    return scenes, out


def _alone(rt, scene, spec):
    b = rt.trace(scene, spec)
    torch.cuda.synchronize()
    return b


def _wait_all(svc, seqs, limit_s=60.0, done=None):
    done, t0 = set() if done is None else done, time.time()
    while not set(seqs) <= done:
        done.update(svc.poll())
        if time.time() - t0 >= limit_s:
            stuck = sorted(set(seqs) - done)[:4]
            raise AssertionError(f"service jobs did not finish: {[svc.job_state(q) for q in stuck]}")
        time.sleep(0.001)
    return done


def test_jobs_submitted_while_the_launch_runs_equal_jobs_alone(rt):
    scenes, jobs = _jobs(rt)
    svc = rt.TraceService(0, idle_timeout_s=0.05)
    try:
        bufs = [rt.TraceBuffers.allocate(sc.num_surfaces, sp.num_bins, torch.device("cuda")) for sc, sp in jobs]
        first = svc.submit([(sc, sp, b) for (sc, sp), b in zip(jobs[:2], bufs[:2])])
        time.sleep(0.002)   # the launch is running: the rest join it
        rest = svc.submit([(sc, sp, b) for (sc, sp), b in zip(jobs[2:], bufs[2:])])
        assert svc.info()["running_launches"] >= 1
        _wait_all(svc, first + rest)
        torch.cuda.synchronize()
        for (sc, sp), b in zip(jobs, bufs):
            want = _alone(rt, sc, sp)
            np.testing.assert_array_equal(b.echogram_fx.cpu().numpy(), want.echogram_fx.cpu().numpy())
            np.testing.assert_array_equal(b.hit_counts.cpu().numpy(), want.hit_counts.cpu().numpy())
            np.testing.assert_array_equal(b.counters[:4].cpu().numpy(), want.counters[:4].cpu().numpy())
            np.testing.assert_array_equal(b.echogram.cpu().numpy(), want.echogram.cpu().numpy())
            np.testing.assert_array_equal(b.surface_energy.cpu().numpy(), want.surface_energy.cpu().numpy())
    finally:
        svc.close()
        for sc in scenes:
            sc.close()


def test_idle_launch_ends_by_itself_and_the_next_submit_starts_one(rt):
    scenes, jobs = _jobs(rt, rays=(2_000,))
    svc = rt.TraceService(0, idle_timeout_s=0.005)
    try:
        sc, sp = jobs[0]
        b1 = rt.TraceBuffers.allocate(sc.num_surfaces, sp.num_bins, torch.device("cuda"))
        _wait_all(svc, svc.submit([(sc, sp, b1)]))
        t0 = time.time()
        while svc.info()["running_launches"] and time.time() - t0 < 5.0:
            time.sleep(0.005)
        assert svc.info()["running_launches"] == 0, "the idle launch did not end"
        b2 = rt.TraceBuffers.allocate(sc.num_surfaces, sp.num_bins, torch.device("cuda"))
        _wait_all(svc, svc.submit([(sc, sp, b2)]))
        assert svc.info()["launches"] == 2
        torch.cuda.synchronize()
        np.testing.assert_array_equal(b1.echogram_fx.cpu().numpy(), b2.echogram_fx.cpu().numpy())
    finally:
        svc.close()
        for sc in scenes:
            sc.close()


def test_a_full_ring_asks_the_caller_to_poll(rt):
    from acoustic_agent_b200 import _lib
    scenes, jobs = _jobs(rt, rays=(500,))
    svc = rt.TraceService(0, capacity=64, idle_timeout_s=0.01)
    try:
        sc, sp = jobs[0]
        batch = [(sc, replace(sp, stream_key=k), rt.TraceBuffers.allocate(sc.num_surfaces, sp.num_bins,
                                                                          torch.device("cuda"))) for k in range(32)]
        seqs = svc.submit(batch)
        with pytest.raises(_lib.BackendError) as err:
            svc.submit(batch[:1])
        assert err.value.code == _lib.AC_ERR_CAPACITY
        _wait_all(svc, seqs)
        more = svc.submit(batch[:4])   # room again once the jobs are reported done
        _wait_all(svc, more)
        assert svc.info()["in_flight"] == 0
    finally:
        svc.close()
        for sc in scenes:
            sc.close()


def test_the_ring_wraps_across_many_launches_and_every_job_equals_it_alone(rt):
    """A 64-slot ring (32-job windows) wrapped several times by trickled submissions, so that launches
    start and end while jobs wait and slots are rewritten; every job's sums equal the job traced alone and
    its progress record ends complete."""
    from acoustic_agent_b200 import _lib
    scenes, jobs = _jobs(rt, rays=(1_500, 300, 4_000))
    svc = rt.TraceService(0, capacity=64, idle_timeout_s=0.002)
    dev = torch.device("cuda")
    try:
        submitted, done, keys = [], set(), {}
        k = 0
        for round_ in range(24):
            batch = []
            for _ in range(7 + round_ % 5):
                sc, sp = jobs[k % len(jobs)]
                sp = replace(sp, stream_key=5000 + k)
                batch.append((sc, sp, rt.TraceBuffers.allocate(sc.num_surfaces, sp.num_bins, dev)))
                k += 1
            while True:
                try:
                    seqs = svc.submit(batch)
                    break
                except _lib.BackendError as exc:   # the ring is full: poll, then retry
                    if exc.code != _lib.AC_ERR_CAPACITY:
                        raise
                    done.update(svc.poll())
                    time.sleep(0.001)
            for q, item in zip(seqs, batch):
                keys[q] = item
            submitted += seqs
            done.update(svc.poll())
            time.sleep(0.001 * (round_ % 4))
        _wait_all(svc, submitted, done=done)
        assert svc.info()["launches"] >= 4 and submitted[-1] >= 3 * 64
        for q in submitted[-64:]:
            st = svc.job_state(q)
            assert st["done_seq"] == q and st["rays_finished"] == st["rays"] and st["in_flight"] == 0
            assert st["chunks_taken"] >= st["chunks"]
        torch.cuda.synchronize()
        for q in submitted[::5]:
            sc, sp, b = keys[q]
            want = _alone(rt, sc, sp)
            np.testing.assert_array_equal(b.echogram_fx.cpu().numpy(), want.echogram_fx.cpu().numpy())
            np.testing.assert_array_equal(b.counters[:4].cpu().numpy(), want.counters[:4].cpu().numpy())
            np.testing.assert_array_equal(b.echogram.cpu().numpy(), want.echogram.cpu().numpy())
    finally:
        svc.close()
        for sc in scenes:
            sc.close()


@pytest.fixture(scope="module")
def served_continuously():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from acoustic_agent_b200 import serving, workloads
    population = workloads.mixed_batch(21, 6, max_rays=20_000, min_rays=2_000)
    stream = workloads.request_stream(5, rate_hz=300.0, duration_s=0.1, population=population, keyframes=3)
    requests = serving.requests_from_stream(stream)
    server = serving.ContinuousServer(0, tune=True)
    report = server.serve(requests, realtime=True)
    server.close()
    return serving, requests, report


def test_continuous_server_serves_every_request(served_continuously):
    serving, requests, report = served_continuously
    assert [r.request.id for r in report.results] == [r.id for r in requests]
    assert all(r.error is None and len(r.band_irs) == r.request.num_rirs for r in report.results)
    s = report.summary()
    assert s["p99_ms"] >= s["p50_ms"] > 0 and s["rirs"] == sum(r.num_rirs for r in requests)


def test_continuous_results_equal_the_request_alone(served_continuously):
    serving, requests, report = served_continuously
    picks = [report.results[0], report.results[-1]] + [r for r in report.results if r.request.moving][:1]
    for res in picks:
        alone = serving.render_alone(res.request)
        assert len(alone) == len(res.band_irs)
        for a, b in zip(alone, res.band_irs):
            np.testing.assert_array_equal(a, b)


def test_overload_is_shed_with_a_reason():
    from acoustic_agent_b200 import serving, workloads
    population = workloads.mixed_batch(22, 4, max_rays=200_000, min_rays=100_000)
    stream = workloads.request_stream(6, rate_hz=400.0, duration_s=0.05, population=population, keyframes=2)
    requests = serving.requests_from_stream(stream)
    server = serving.ContinuousServer(0, tune=False, slo_s=0.05, capacity_rb_per_s=1e9)
    report = server.serve(requests, realtime=True)
    server.close()
    rejected = report.rejected
    assert rejected and all("overloaded" in r.error for r in rejected)
    assert len(rejected) < len(requests)
    assert all(r.band_irs for r in report.results if r.error is None)
