"""The reference's own room renderer with its reflection trace routed to this backend.

``steam_rt.simulate_steam_room`` (steam_rt.py:927-1190) computes direct sound,
diffraction, the reflection field (``trace_energy_field``), visual ray paths
from the field's candidate slots, band synthesis and decay metrics.  With
``backend.install()`` and ``rt_accelerator="b200"`` the field comes from the
GPU; everything else stays the reference's code.  The unmodified reference
package is the one installed under baseline/_ref (skipped when absent).

The float64 kernel follows the reference's rays exactly, so the render with
``rt_precision="float64"`` is the reference's own result; the float32 render
must match its per-band decay times within 2 %.
"""
from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def reference():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import bench
    ref, why = bench.import_reference_package()
    if ref is None:
        pytest.skip(why)
    return bench, ref


def test_simulate_steam_room_renders_through_the_b200_backend(reference):
    bench, (steam_rt, models) = reference
    from acoustic_agent_b200 import backend, workloads
    spec = {"corners": [(0.0, 0.0), (6.0, 0.0), (6.0, 4.0), (4.26, 4.0), (4.26, 2.08), (1.74, 2.08), (1.74, 4.0),
                        (0.0, 4.0)], "height": 2.8, "materials": workloads._uniform_materials()}
    room = bench.reference_scene(steam_rt, models, spec).room
    renders = {}
    handle = backend.install(steam_rt)
    try:
        for precision in ("float64", "float32"):
            cfg = models.SimConfig(fs=16000, duration_s=1.0, rt_duration_s=1.0, rt_num_rays=20000, rt_num_bounces=64,
                                   late_tail=False, adaptive_geometry_bounces=False, rt_accelerator="b200",
                                   rt_precision=precision, seed=11)
            renders[precision] = steam_rt.simulate_steam_room(room, [0.8, 3.2, 1.4], [5.2, 3.2, 1.4], cfg)
    finally:
        handle.uninstall()
    for precision, out in renders.items():
        refl = out.metadata["reflections"]
        assert refl["accelerator"] == "b200" and refl["precision"] == precision
        assert refl["cuda"]["compute_capability"].startswith("10.")
        assert out.metadata["rt_visual"]["retained_path_count"] > 0   # paths built from the GPU's candidate slots
        assert np.isfinite(out.rir).all() and np.abs(out.rir).max() > 0
    t64 = np.array(list(renders["float64"].rt60_bands.values()))
    t32 = np.array(list(renders["float32"].rt60_bands.values()))
    assert (t64 > 0).all()
    np.testing.assert_allclose(t32, t64, rtol=0.02)


def test_late_tail_routes_to_the_gpu_fdn(reference):
    """With late_tail on, install() also routes _render_parametric_fdn_late_reverb (steam_rt.py:1029) to the GPU
    FDN; the rendered RIR equals the one with the reference's own CPU FDN to float32 rounding."""
    bench, (steam_rt, models) = reference
    from acoustic_agent_b200 import backend, workloads
    spec = {"corners": [(0.0, 0.0), (6.0, 0.0), (6.0, 4.0), (0.0, 4.0)], "height": 3.0,
            "materials": workloads._uniform_materials()}
    room = bench.reference_scene(steam_rt, models, spec).room
    cfg = models.SimConfig(fs=16000, duration_s=1.0, rt_duration_s=1.0, rt_num_rays=4000, rt_num_bounces=64,
                           late_tail=True, hybrid_transition_s=0.5, adaptive_geometry_bounces=False,
                           rt_accelerator="b200", rt_precision="float64", seed=11)
    handle = backend.install(steam_rt)
    try:
        gpu = steam_rt.simulate_steam_room(room, [1.5, 1.2, 1.5], [4.2, 2.9, 1.6], cfg)
        routed = steam_rt._render_parametric_fdn_late_reverb
        steam_rt._render_parametric_fdn_late_reverb = handle.originals["_render_parametric_fdn_late_reverb"]
        try:
            cpu = steam_rt.simulate_steam_room(room, [1.5, 1.2, 1.5], [4.2, 2.9, 1.6], cfg)
        finally:
            steam_rt._render_parametric_fdn_late_reverb = routed
    finally:
        handle.uninstall()
    g_meta, c_meta = gpu.metadata["reflections"]["late_tail"], cpu.metadata["reflections"]["late_tail"]
    assert g_meta["applied"] and c_meta["applied"]
    assert g_meta["delay_samples"] == c_meta["delay_samples"]
    for band, scale in c_meta["scale_by_band"].items():
        assert g_meta["scale_by_band"][band] == pytest.approx(scale, rel=1e-7)
    scale = float(np.abs(cpu.rir).max())
    np.testing.assert_allclose(gpu.rir, cpu.rir, rtol=1e-5, atol=1e-6 * scale)


def test_direct_path_routes_to_the_gpu(reference):
    """install() also routes simulate_direct (steam_rt.py:942) to the GPU queries; in the furnished U room, where
    walls and cabinets block the direct path, the render equals the one with the reference's own Python queries."""
    bench, (steam_rt, models) = reference
    from acoustic_agent_b200 import backend, workloads
    w = workloads.u_furnished(1729)
    room = bench.reference_scene(steam_rt, models, w.spec).room
    cfg = models.SimConfig(fs=16000, duration_s=0.5, rt_duration_s=0.5, rt_num_rays=2000, rt_num_bounces=32,
                           late_tail=False, adaptive_geometry_bounces=False, rt_accelerator="b200",
                           rt_precision="float64", seed=5)
    handle = backend.install(steam_rt)
    try:
        gpu = steam_rt.simulate_steam_room(room, list(w.sources[0]), list(w.listeners[0]), cfg, "cardioid")
        routed = steam_rt.simulate_direct
        steam_rt.simulate_direct = handle.originals["simulate_direct"]
        try:
            cpu = steam_rt.simulate_steam_room(room, list(w.sources[0]), list(w.listeners[0]), cfg, "cardioid")
        finally:
            steam_rt.simulate_direct = routed
    finally:
        handle.uninstall()
    np.testing.assert_array_equal(gpu.rir, cpu.rir)


def test_scene_bvh_build_routes_to_the_gpu(reference):
    """install(gpu_bvh_min_surfaces=1) routes the reference's build_bvh (called by _scene_kernel_arrays at
    steam_rt.py:881) to the GPU build; the scene's BVH arrays equal the reference's own, array for array."""
    bench, (steam_rt, models) = reference
    from acoustic_agent_b200 import backend, workloads
    w = workloads.u_furnished(1729)
    scene = bench.reference_scene(steam_rt, models, w.spec)
    steam_rt._SCENE_ARRAY_CACHE.clear()
    ref = steam_rt._scene_kernel_arrays(scene)
    handle = backend.install(steam_rt, gpu_bvh_min_surfaces=1)
    try:
        steam_rt._SCENE_ARRAY_CACHE.clear()
        gpu = steam_rt._scene_kernel_arrays(scene)
    finally:
        handle.uninstall()
        steam_rt._SCENE_ARRAY_CACHE.clear()
    for k in ("bvh_bounds_min", "bvh_bounds_max", "bvh_start", "bvh_count", "bvh_escape", "bvh_primitives",
              "bvh_node_count", "bvh_leaf_count", "bvh_max_depth", "bvh_leaf_size"):
        np.testing.assert_array_equal(np.asarray(gpu[k]), np.asarray(ref[k]), err_msg=k)


def test_acoustic_agent_facade_runs_through_the_b200_backend(reference):
    """The reference's public facade, unchanged: AcousticAgent.create(scene="geometry", room=Room(...),
    config=SimConfig(rt_accelerator="b200"), receiver_model=<8-mic circular array>).run() traces every channel
    of its channel loop (engine.py:64-73) on the GPU.  With rt_precision="float64" the B200 kernel follows the
    reference's rays, so the 8-channel RIR equals the one the reference's own float64 Numba path renders."""
    bench, (steam_rt, models) = reference
    from acoustic_agent import api
    from acoustic_agent_b200 import backend, workloads
    w = workloads.u_furnished(1729)
    room = bench.reference_scene(steam_rt, models, w.spec).room
    array = {"type": "circular", "count": 8, "radius_m": 0.05}

    def run(accelerator, precision, rays=3000):
        cfg = models.SimConfig(fs=16000, duration_s=1.0, rt_duration_s=1.0, rt_num_rays=rays, rt_num_bounces=60,
                               rt_bin_duration_s=0.001, intersection_backend="bvh", late_tail=False,
                               adaptive_geometry_bounces=False, rt_accelerator=accelerator, rt_precision=precision,
                               seed=1729)
        agent = api.AcousticAgent.create(scene="geometry", room=room, config=cfg, receiver_model=array,
                                         source_model="cardioid", source=w.sources[0], receiver=(1.079, 6.252, 1.348))
        return agent.run()

    handle = backend.install(steam_rt)
    try:
        gpu64 = run("b200", "float64")
        gpu32 = run("b200", "float32")
    finally:
        handle.uninstall()
    cpu64 = run("numba", "float64")
    assert gpu64.rir.shape == (8, 16000) and gpu64.metadata["array_channel_count"] == 8
    refl = gpu64.metadata["steam_audio"]["reflections"]
    assert refl["accelerator"] == "b200" and refl["precision"] == "float64"
    assert gpu32.metadata["steam_audio"]["reflections"]["precision"] == "float32"
    scale = float(np.abs(cpu64.rir).max())
    np.testing.assert_allclose(gpu64.rir, cpu64.rir, rtol=1e-5, atol=1e-6 * scale)
    # the traced field's decay (rounded to 0.1 ms by the reference) is the same field
    assert gpu64.rt60["traced_rt60_bands"] == cpu64.rt60["traced_rt60_bands"]
    t32 = np.array(list(gpu32.rt60["traced_rt60_bands"].values()))
    t64 = np.array(list(cpu64.rt60["traced_rt60_bands"].values()))
    np.testing.assert_allclose(t32, t64, rtol=0.02)
