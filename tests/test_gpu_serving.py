"""Serving loop: HBM admission, continuous batching, results independent of the mix.

A Poisson stream of requests over a mixed-size scene population (one to
several rooms, several channels, moving sources with keyframes) is served
with a device-memory budget of about two requests, so requests queue for
memory, batches overlap on two streams and idle scenes are evicted.  Each
served result must equal the same request rendered alone, and one result's
per-band energy decay must match the float64 oracle traced on the same
counter-based random stream within 0.5 dB over the first 30 dB.
"""
from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def served():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from acoustic_agent_b200 import serving, workloads
    population = workloads.mixed_batch(21, 6, max_rays=20_000, min_rays=2_000)
    stream = workloads.request_stream(5, rate_hz=300.0, duration_s=0.1, population=population, keyframes=3)
    requests = serving.requests_from_stream(stream)
    sizer = serving.Server(0, max_inflight=2, tune=False)
    largest = max(sizer.footprint(r, serving.request_jobs(r)) for r in requests)
    sizer.close()
    server = serving.Server(0, max_inflight=2, hbm_budget=2 * largest + (1 << 20), tune=True)
    report = server.serve(requests, realtime=True)
    server.close()
    return serving, requests, report


def test_every_request_is_served(served):
    serving, requests, report = served
    assert len(requests) >= 10 and any(r.moving for r in requests)
    assert [r.request.id for r in report.results] == [r.id for r in requests]
    for res in report.results:
        assert len(res.band_irs) == res.request.num_rirs
        assert res.done_s >= res.admitted_s >= res.request.arrival_s - 1e-3
        assert all(np.isfinite(ir).all() for ir in res.band_irs)
    s = report.summary()
    assert s["p99_ms"] >= s["p50_ms"] > 0 and s["rirs"] == sum(r.num_rirs for r in requests)
    assert report.batches >= 2 and report.scene_hits > 0


def test_each_result_equals_the_request_alone(served):
    serving, requests, report = served
    picks = [report.results[0], report.results[-1]] + [r for r in report.results if r.request.moving][:1]
    for res in picks:
        alone = serving.render_alone(res.request)
        assert len(alone) == len(res.band_irs)
        for a, b in zip(alone, res.band_irs):
            np.testing.assert_array_equal(a, b)


def test_served_result_tracks_the_float64_oracle(served):
    """Per-band EDC of the served band IRs vs the oracle's float64 trace + synthesis, same Philox stream."""
    from acoustic_agent_b200 import bands, metrics, scene
    from oracle import oracle
    serving, requests, report = served
    res = max((r for r in report.results if not r.request.moving), key=lambda r: r.request.workload.config.rt_num_rays)
    req = res.request
    spec = serving.request_jobs(req)[0]
    cfg = req.workload.config
    arrays = scene.compile_scene(req.workload.spec)
    dirs, rnd, idx = oracle.philox_workspace(spec.num_rays, spec.num_bounces, spec.seed, spec.stream_key)
    _, bank, _, _ = oracle.workspace(1, 0, 0)
    ref = oracle.trace(arrays, source=spec.source, listener=spec.listener, directions=dirs, diffuse_bank=bank,
                       diffuse_random=rnd, diffuse_indices=idx, num_bins=spec.num_bins, bin_dur=spec.bin_duration,
                       c=spec.speed_of_sound, max_path_len=spec.max_path_length, direct_delay=spec.direct_delay,
                       source_forward=spec.source_forward, dipole_weight=spec.dipole_weight,
                       dipole_power=spec.dipole_power, use_bvh=spec.use_bvh)
    spb = bands.samples_per_bin(spec.bin_duration, cfg.fs)
    white = oracle.philox_noise(spec.num_bins * spb, spec.seed + 7)
    expected = oracle.synthesize(ref["echogram"].astype(np.float32), fs=cfg.fs, bin_dur=spec.bin_duration,
                                 direct_delay=spec.direct_delay, c=spec.speed_of_sound, white=white)

    def bin_energy(ir):
        return (ir.astype(np.float64) ** 2).reshape(6, spec.num_bins, spb).sum(axis=2)

    err = metrics.edc_error_db(bin_energy(res.band_irs[0]), bin_energy(expected))
    assert float(err.max()) <= 0.5, err


def test_a_request_larger_than_the_budget_is_rejected_not_fatal(served):
    serving, requests, report = served
    small = requests[:3]
    sizer = serving.Server(0, max_inflight=2, tune=False)
    sizes = [sizer.footprint(r, serving.request_jobs(r)) for r in small]
    sizer.close()
    budget = sorted(sizes)[1] + (64 << 10)       # the largest of the three cannot fit
    big = small[int(np.argmax(sizes))]
    server = serving.Server(0, max_inflight=2, hbm_budget=budget, tune=False)
    out = server.serve([serving.Request(r.id, r.workload, r.sources, 0.0, r.moving) for r in small], realtime=False)
    server.close()
    rejected = [r.request.id for r in out.rejected]
    assert big.id in rejected and "budget" in out.results[[r.request.id for r in out.results].index(big.id)].error
    assert all(r.band_irs for r in out.results if r.error is None)
    assert out.summary()["rejected"] == len(rejected) >= 1


def test_served_late_tails_equal_the_request_alone():
    """With late_tail, each served RIR is its band IRs crossfaded into the FDN late tail; a request gives the
    same hybrid band IRs in the mix (two batches in flight) as alone, and its tail equals the per-call
    drop-in on its band IRs."""
    from types import SimpleNamespace
    from acoustic_agent_b200 import bands, late_reverb, runtime, serving, workloads
    population = workloads.mixed_batch(23, 4, max_rays=20_000, min_rays=5_000)
    stream = workloads.request_stream(9, rate_hz=200.0, duration_s=0.05, population=population, keyframes=2)
    requests = serving.requests_from_stream(stream)[:6]
    server = serving.Server(0, max_inflight=2, tune=False, late_tail=True)
    report = server.serve(requests, realtime=True)
    server.close()
    assert all(r.error is None for r in report.results)
    for res in (report.results[0], report.results[-1]):
        alone = serving.render_alone(res.request, late_tail=True)
        plain = serving.render_alone(res.request)
        for a, b, p in zip(alone, res.band_irs, plain):
            np.testing.assert_array_equal(a, b)
            assert not np.array_equal(a, p)   # the tail changed the band IRs
    # the first RIR's tail against the drop-in, with the RT60s estimated from its own trace
    res = report.results[0]
    spec = serving.request_jobs(res.request)[0]
    w = res.request.workload
    scene = runtime.DeviceScene(serving.SceneCache(0, tune=False).key_of(w)[1])
    b = runtime.trace(scene, spec)
    echogram = b.echogram.cpu().numpy()
    scene.close()
    rt60 = late_reverb.estimate_reverb_times(echogram, spec.bin_duration, spec.speed_of_sound)
    cfg = SimpleNamespace(fs=w.config.fs, seed=int(spec.seed), late_tail=True, hybrid_transition_s=1.0,
                          hybrid_overlap_fraction=0.25, rt_bin_duration_s=spec.bin_duration)
    plain_first = serving.render_alone(res.request)[0]
    out, _, _ = late_reverb.render_parametric_fdn_late_reverb(plain_first, {"bin_duration_s": spec.bin_duration},
                                                              dict(zip(bands.FREQUENCY_BANDS, rt60)), cfg)
    np.testing.assert_array_equal(out, res.band_irs[0])
