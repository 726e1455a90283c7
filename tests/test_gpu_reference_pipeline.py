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
