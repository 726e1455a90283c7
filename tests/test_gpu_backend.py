"""The drop-in ``trace_energy_field`` on the GPU: result contract and error behaviour."""
from __future__ import annotations

from dataclasses import replace

import numpy as np
import pytest

from conftest import load_case

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

# Keys of the reference CUDA backend's result (steam_rt.py:1892-1923).
REFERENCE_KEYS = {
    "echogram", "ambisonic_echogram", "num_bins", "bin_duration_s", "direct_delay_s", "actual_bounces",
    "active_ray_count", "last_energy_time_s", "surface_hit_count", "surface_contribution_count", "surface_energy",
    "visual_candidates", "accelerator", "precision", "cuda", "device_input_cache", "kernel_time_s",
    "transfer_time_s", "intersection_backend", "source_directivity",
}


@pytest.fixture(scope="module")
def backend():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from acoustic_agent_b200 import backend as b
    return b


def small_config(**over):
    from acoustic_agent_b200.workloads import TraceConfig
    cfg = TraceConfig(duration_s=0.3, rt_duration_s=0.3, rt_num_rays=256, rt_num_bounces=6, rt_precision="float32",
                      intersection_backend="auto")
    return replace(cfg, **over)


def test_result_dictionary_matches_reference_contract(backend):
    from acoustic_agent_b200 import scene, workloads
    w = workloads.shoebox(3)
    arrays = scene.compile_scene(w.spec)
    field = backend.trace_energy_field(arrays, np.asarray(w.sources[0]), np.asarray(w.listeners[0]), small_config(),
                                       render_ambisonics=True)
    assert set(field) == REFERENCE_KEYS
    assert field["echogram"].dtype == np.float32 and field["echogram"].shape == (6, field["num_bins"])
    assert field["ambisonic_echogram"].shape == (6, 4, field["num_bins"])
    assert field["accelerator"] == "b200" and field["precision"] == "float32"
    assert field["intersection_backend"] == "linear"
    assert field["cuda"]["compute_capability"].startswith("10.")
    assert field["actual_bounces"] == 6
    assert sum(field["surface_hit_count"].values()) > 0
    assert field["kernel_time_s"] > 0.0


def test_drop_in_float64_equals_golden(backend):
    case = load_case("u_room_kat")
    tr = case["trace"]
    cfg = small_config(duration_s=tr["duration"], rt_duration_s=tr["duration"], rt_num_rays=tr["rays"],
                       rt_num_bounces=tr["bounces"], seed=tr["seed"], rt_precision="fp64")
    field = backend.trace_energy_field(case["arrays"], np.asarray(tr["source"]), np.asarray(tr["listener"]), cfg,
                                       render_ambisonics=True)
    names = case["arrays"]["names"]
    expected = {names[i]: int(v) for i, v in enumerate(case["hit_counts"]) if v > 0}
    assert field["surface_hit_count"] == expected
    np.testing.assert_allclose(field["echogram"], case["echogram"].astype(np.float32), rtol=2e-6, atol=1e-12)
    assert field["active_ray_count"] == int(case["active_ray_count"])


def test_invalid_configuration_is_rejected(backend):
    from acoustic_agent_b200 import scene, workloads
    w = workloads.shoebox(3)
    arrays = scene.compile_scene(w.spec)
    with pytest.raises(ValueError):
        backend.trace_energy_field(arrays, np.asarray(w.sources[0]), np.asarray(w.listeners[0]),
                                   small_config(rt_precision="float16"))
    with pytest.raises(ValueError):
        backend.trace_energy_field(arrays, np.asarray(w.sources[0]), np.asarray(w.listeners[0]),
                                   small_config(intersection_backend="octree"))
    with pytest.raises(ValueError):
        backend.trace_energy_field(arrays, np.asarray(w.sources[0]), np.asarray(w.listeners[0]), small_config(),
                                   source_model="laser")


def test_install_routes_only_the_b200_accelerator(backend):
    import types
    calls = []
    fake = types.SimpleNamespace(
        trace_energy_field=lambda *a, **k: calls.append("reference") or {"accelerator": "numba"},
        _normalize_rt_accelerator=lambda v: v if v in {"auto", "numba", "cuda"} else (_ for _ in ()).throw(
            ValueError("rt_accelerator must be auto, numba, or cuda")))
    handle = backend.install(fake)
    from acoustic_agent_b200 import scene, workloads
    w = workloads.shoebox(3)
    arrays = scene.compile_scene(w.spec)
    field = fake.trace_energy_field(arrays, np.asarray(w.sources[0]), np.asarray(w.listeners[0]), small_config())
    assert field["accelerator"] == "b200"
    assert fake.trace_energy_field(arrays, None, None, small_config(rt_accelerator="numba"))["accelerator"] == "numba"
    assert fake._normalize_rt_accelerator("b200") == "b200"
    with pytest.raises(ValueError):
        fake._normalize_rt_accelerator("metal")
    handle.uninstall()
    with pytest.raises(ValueError):
        fake._normalize_rt_accelerator("b200")


def test_capacity_and_sizes_are_checked_before_launch(backend):
    """num_rays * num_bounces must stay below 2^32 (exact fixed-point sums); bad sizes never launch."""
    from acoustic_agent_b200 import _lib, runtime, scene, workloads
    w = workloads.shoebox(3)
    dev = runtime.DeviceScene(scene.compile_scene(w.spec))
    buffers = runtime.TraceBuffers.allocate(dev.num_surfaces, 10, torch.device("cuda", 0))
    base = dict(source=w.sources[0], listener=w.listeners[0], num_bins=10, bin_duration=0.01,
                speed_of_sound=343.0, max_path_length=343.0, direct_delay=0.01, rng="philox")
    too_big = runtime.TraceSpec(num_rays=(1 << 31) - 1, num_bounces=3, **base)
    with pytest.raises(_lib.BackendError) as err:   # AC_ERR_CAPACITY, with the library's message
        runtime.trace(dev, too_big, buffers)
    assert err.value.code == _lib.AC_ERR_CAPACITY and "2^32" in str(err.value)
    with pytest.raises(ValueError):
        runtime.trace(dev, runtime.TraceSpec(num_rays=0, num_bounces=3, **base), buffers)
    torch.cuda.synchronize()
    dev.close()


def test_scene_destroyed_while_its_trace_is_queued_keeps_its_result(backend):
    """A scene may be destroyed right after a trace that reads it is enqueued on a non-blocking stream: its
    memory returns to the pool only after that trace, so a scene uploaded next (which may get the same block)
    cannot overwrite it under the running trace.  Repeated a few times to give the pool the chance to reuse."""
    from acoustic_agent_b200 import runtime, scene, workloads
    w = workloads.u_furnished(7, rays=100_000, bounces=100, channels=1)
    other = workloads.u_furnished(8, rays=1000, bounces=10, channels=1)
    arrays, other_arrays = scene.compile_scene(w.spec), scene.compile_scene(other.spec)
    cfg = w.config
    src, lst = np.asarray(w.sources[0]), np.asarray(w.listeners[0])
    spec = runtime.TraceSpec(source=src, listener=lst, num_rays=cfg.rt_num_rays, num_bounces=cfg.rt_num_bounces,
                             num_bins=cfg.num_bins, bin_duration=cfg.rt_bin_duration_s, speed_of_sound=cfg.c,
                             max_path_length=cfg.max_path_length, direct_delay=float(np.linalg.norm(src - lst)) / cfg.c,
                             precision="float32", rng="philox", seed=cfg.seed, stream_key=5, use_bvh=True)
    alone = runtime.DeviceScene(arrays, device=0)
    want = runtime.trace(alone, spec)
    torch.cuda.synchronize()
    want_bins = want.echogram_fx.cpu().numpy()
    alone.close()
    side = torch.cuda.Stream()
    for _ in range(3):
        with torch.cuda.stream(side):
            doomed = runtime.DeviceScene(arrays, device=0)
            got = runtime.trace(doomed, spec, stream=side)
            doomed.close()
            replacement = runtime.DeviceScene(other_arrays, device=0)
        side.synchronize()
        np.testing.assert_array_equal(got.echogram_fx.cpu().numpy(), want_bins)
        replacement.close()
