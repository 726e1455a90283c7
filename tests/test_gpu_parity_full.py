"""Parity of the production float32 kernel at the benchmark's own sizes, against the float64 oracle.

The oracle (a C restatement of the reference's Numba float64 tracer, pinned to
the reference's own outputs by tests/test_oracle_golden.py) and the GPU trace
the SAME rays: the reference's random stream (jittered Fibonacci directions,
PCG64 uniforms and bank indices from the seed) is drawn once and fed to both.

* config 1: the furnished U room (30 surfaces, cardioid source, 8-mic circular
  array), 200,000 rays x 100 bounces, 1 ms bins, fs 48 kHz, 2 s; two channels;
* config 2: the 8-room apartment (428 surfaces, 0.15 m shared walls, open
  doors, 10-25 boxes per room), 100,000 rays x 200 bounces, mono receiver.

Checked on each:

1. the rays whose hit-surface sequences are identical in float32 and float64,
   traced again on their own by both, have per-band energies within 1e-4
   relative (the float32 arithmetic itself, with no path change);
2. the rays that leave the float64 path are the precision-sensitive ones:
   traced again in float64 with their initial direction turned by about
   1e-6 rad (32 seeded turns; float32 rounds a unit vector by up to 6e-8),
   at least 90 % of them change path -- and for most of them some turned
   float64 trace follows the float32 path through its first differing
   bounce -- while at most 10 % of a control sample of identical rays
   changes path under the same turns (oracle.path_sensitivity); the
   fractions are printed;
3. the whole echogram: per-band EDC within 0.5 dB over the first 30 dB, T30,
   EDT and C50 (early/late ratio) within 1 %, band energies within 1 %;
4. the on-device Philox stream (the bench's own stream) at the same size,
   against the float64 oracle fed the same Philox rays (its numpy
   restatement of the stream): EDC within 0.5 dB, T30, EDT and C50 within
   1 %; the comparison with the reference stream's float64 trace (different
   rays: a Monte-Carlo difference, large where little energy crosses from
   the source's room to the listener's) is printed.
"""
from __future__ import annotations

from dataclasses import replace

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

ENERGY_RTOL_SAME_RAYS = 1e-4
DECAY_RTOL = 0.01
EDC_DB = 0.5
SENSITIVE_MIN = 0.90        # divergent rays whose float64 path changes under float32-scale turns, at least
CONTROL_MAX = 0.10          # identical rays whose float64 path changes under the same turns, at most
SAMPLE = 300


@pytest.fixture(scope="module")
def rt():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from acoustic_agent_b200 import runtime
    return runtime


def _oracle_kwargs(spec):
    return dict(source=np.asarray(spec.source, dtype=float), listener=np.asarray(spec.listener, dtype=float),
                num_bins=int(spec.num_bins), bin_dur=spec.bin_duration, c=spec.speed_of_sound,
                max_path_len=spec.max_path_length, direct_delay=spec.direct_delay,
                listener_radius=spec.listener_radius, source_radius=spec.source_radius,
                irradiance_min_distance=spec.irradiance_min_distance, specular_exponent=spec.specular_exponent,
                source_forward=np.asarray(spec.source_forward, dtype=float), dipole_weight=spec.dipole_weight,
                dipole_power=spec.dipole_power, use_bvh=bool(spec.use_bvh))


def _device_workspace(dirs, rnd, idx):
    return (torch.as_tensor(np.ascontiguousarray(dirs), dtype=torch.float32, device="cuda"),
            torch.as_tensor(np.ascontiguousarray(rnd), dtype=torch.float32, device="cuda"),
            torch.as_tensor(np.ascontiguousarray(idx), dtype=torch.int32, device="cuda"))


def _gpu_trace(rt, scene, spec, workspace, record_rays=True):
    buffers = rt.trace(scene, spec, record_rays=record_rays, workspace=workspace)
    torch.cuda.synchronize()
    out = {"echogram": rt.fixed_to_float64(buffers.echogram_fx, buffers.scale.value)}
    if record_rays:
        out["ray_surfaces"] = buffers.ray_surfaces.cpu().numpy()
    return out


def check_full_size(rt, workload, channel: int, rays: int, label: str):
    from acoustic_agent_b200 import batching, metrics, scene as scene_mod
    from oracle import oracle
    arrays = scene_mod.compile_scene(workload.spec)
    _, jobs = batching.workload_jobs([workload], precision="float32", rng_mode="reference")
    spec = replace(jobs[channel].spec, num_rays=rays)
    B = int(spec.num_bounces)
    dirs, bank, rnd, idx = oracle.workspace(rays, B, int(spec.seed))
    kw = _oracle_kwargs(spec)
    scene = rt.DeviceScene(arrays)
    try:
        gpu = _gpu_trace(rt, scene, spec, _device_workspace(dirs, rnd, idx))
        ref = oracle.trace(arrays, directions=dirs, diffuse_bank=bank, diffuse_random=rnd, diffuse_indices=idx,
                           record_rays=True, **kw)
        same = np.all(gpu["ray_surfaces"] == ref["ray_surfaces"], axis=1)
        divergent = np.flatnonzero(~same)
        print(f"\n{label}: {rays} rays x {B} bounces, {same.mean():.4%} of ray paths identical")

        # 1. identical rays, traced again on their own: the float32 arithmetic alone
        sel = np.flatnonzero(same)
        sub_spec = replace(spec, num_rays=int(sel.size))
        sub_ws = (dirs[sel], rnd[:, sel], idx[:, sel])
        gpu_same = _gpu_trace(rt, scene, sub_spec, _device_workspace(*sub_ws))
        ref_same = oracle.trace(arrays, directions=sub_ws[0], diffuse_bank=bank, diffuse_random=sub_ws[1],
                                diffuse_indices=sub_ws[2], record_rays=True, **kw)
        np.testing.assert_array_equal(gpu_same["ray_surfaces"], ref_same["ray_surfaces"])
        e_gpu, e_ref = gpu_same["echogram"].sum(axis=1), ref_same["echogram"].sum(axis=1)
        rel = np.abs(e_gpu - e_ref) / e_ref
        print(f"  identical rays alone: per-band energy relative difference max {rel.max():.2e}")
        np.testing.assert_allclose(e_gpu, e_ref, rtol=ENERGY_RTOL_SAME_RAYS)

        # 2. the rays that left the float64 path are those whose float64 path is not robust at float32 scale
        if divergent.size:
            rng = np.random.default_rng(0)
            pick = rng.choice(divergent, size=min(SAMPLE, divergent.size), replace=False)
            control = rng.choice(np.flatnonzero(same), size=min(SAMPLE, int(same.sum())), replace=False)
            ws = dict(directions=dirs, diffuse_bank=bank, diffuse_random=rnd, diffuse_indices=idx)
            div_s = oracle.path_sensitivity(arrays, rays=pick, target_surfaces=gpu["ray_surfaces"], **ws, **kw)
            ctl_s = oracle.path_sensitivity(arrays, rays=control, **ws, **kw)
            print(f"  divergent rays sampled {div_s['rays']} of {divergent.size}: float64 path changes under "
                  f"float32-scale turns for {div_s['sensitive']:.1%}, a turned float64 trace follows the float32 "
                  f"path for {div_s['reproduced']:.1%}; control (identical rays): {ctl_s['sensitive']:.1%}")
            assert div_s["sensitive"] >= SENSITIVE_MIN and ctl_s["sensitive"] <= CONTROL_MAX, (div_s, ctl_s)

        # 3. the whole echogram
        p = metrics.parity(gpu["echogram"], ref["echogram"], spec.bin_duration)
        print("  whole echogram: " + ", ".join(f"{k} {v:.3g}" for k, v in p.items()))
        assert p["edc_err_db_max"] <= EDC_DB
        assert p["t30_rel"] <= DECAY_RTOL and p["edt_rel"] <= DECAY_RTOL and p["c50_rel"] <= DECAY_RTOL
        assert p["band_energy_rel"] <= DECAY_RTOL

        # 4. the bench's on-device Philox stream at the same size, against the float64 oracle on the same rays
        pspec = replace(spec, rng="philox", stream_key=11)
        philox = rt.trace(scene, pspec)
        torch.cuda.synchronize()
        e_philox = rt.fixed_to_float64(philox.echogram_fx, philox.scale.value)
        pd, pr, pi = oracle.philox_workspace(rays, B, int(pspec.seed), int(pspec.stream_key))
        ref_p = oracle.trace(arrays, directions=pd, diffuse_bank=bank, diffuse_random=pr, diffuse_indices=pi, **kw)
        q = metrics.parity(e_philox, ref_p["echogram"], spec.bin_duration)
        print("  Philox stream vs float64 on the same rays: " + ", ".join(f"{k} {v:.3g}" for k, v in q.items()))
        assert q["edc_err_db_max"] <= EDC_DB
        assert q["t30_rel"] <= DECAY_RTOL and q["edt_rel"] <= DECAY_RTOL and q["c50_rel"] <= DECAY_RTOL
        m = metrics.parity(e_philox, ref["echogram"], spec.bin_duration)
        print("  Philox stream vs float64 on the reference stream (different rays): " +
              ", ".join(f"{k} {v:.3g}" for k, v in m.items()))
    finally:
        scene.close()


@pytest.mark.parametrize("channel", [0, 5])
def test_config1_u_room_full_size(rt, channel):
    from acoustic_agent_b200 import workloads
    check_full_size(rt, workloads.u_furnished(1729), channel, 200_000, f"U room channel {channel}")


def test_config2_apartment_8_rooms(rt):
    from acoustic_agent_b200 import workloads
    w = workloads.apartment(1729, rays=100_000, bounces=200, rooms=8)
    check_full_size(rt, w, 0, 100_000, "8-room apartment")
