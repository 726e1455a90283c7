"""Host-side pieces that need no GPU: scene compiler, native BVH builder, ABI surface, validation."""
from __future__ import annotations

import ctypes
import re

import numpy as np
import pytest

from conftest import REPO, load_case

from acoustic_agent_b200 import _lib, scene, workloads
from acoustic_agent_b200.directivity import source_directivity, source_forward
from acoustic_agent_b200.backend import normalize_precision, resolve_intersection_backend

ARRAY_KEYS = ("kinds", "wall_a", "wall_delta", "wall_z", "z_values", "box_center", "box_axis_u", "box_axis_v",
              "box_half", "box_z", "normals", "reflection", "scattering", "corners", "surface_bounds_min",
              "surface_bounds_max", "bvh_bounds_min", "bvh_bounds_max", "bvh_start", "bvh_count", "bvh_escape",
              "bvh_primitives")


def test_scene_compiler_matches_reference_arrays(golden_case):
    _, case = golden_case
    compiled = scene.compile_scene(case["spec"])
    for key in ARRAY_KEYS:
        np.testing.assert_array_equal(np.asarray(compiled[key]), case["arrays"][key], err_msg=key)
    assert tuple(compiled["names"]) == case["arrays"]["names"]


def test_native_bvh_builder_matches_reference(golden_case):
    _, case = golden_case
    a = case["arrays"]
    bvh = _lib.build_bvh(a["surface_bounds_min"], a["surface_bounds_max"])
    for key in ("bounds_min", "bounds_max", "start", "count", "escape", "primitives"):
        np.testing.assert_array_equal(bvh[key], a[f"bvh_{key}"], err_msg=key)


def test_native_bvh_large_random_scene_matches_oracle():
    from oracle import oracle
    rng = np.random.default_rng(3)
    lo = rng.uniform(0, 50, (3000, 3))
    hi = lo + rng.uniform(0, 2, (3000, 3))
    hi[::7] = lo[::7]  # degenerate boxes and centroid ties
    ours = _lib.build_bvh(lo, hi)
    ref = oracle.build_bvh(lo, hi)
    for key in ("bounds_min", "bounds_max", "start", "count", "escape", "primitives"):
        np.testing.assert_array_equal(ours[key], ref[key])
    assert ours["max_depth"] == ref["max_depth"] and ours["leaf_count"] == ref["leaf_count"]


@pytest.mark.parametrize("lo,hi,message", [
    (np.zeros((0, 3)), np.zeros((0, 3)), "at least one surface"),
    (np.asarray([[0.0, 0.0, np.nan]]), np.ones((1, 3)), "finite"),
    (np.ones((1, 3)), np.zeros((1, 3)), "below minimum"),
])
def test_bvh_builder_rejects_what_the_reference_rejects(lo, hi, message):
    with pytest.raises(ValueError, match=message):
        _lib.build_bvh(lo, hi)


def test_library_exports_every_declared_symbol():
    header = (REPO / "include" / "acoustic_rt.h").read_text()
    declared = set(re.findall(r"^(?:const char \*|int )\s*\*?(ac_\w+)\(", header, flags=re.M))
    assert declared, "no declarations parsed"
    lib = ctypes.CDLL(str(_lib.LIBRARY_PATH))
    missing = [name for name in sorted(declared) if not hasattr(lib, name)]
    assert not missing
    assert declared == set(_lib.SIGNATURES), "ctypes binding and header disagree"
    assert _lib.load().ac_abi_version() == 2


# ctypes mirror -> C type name in the public header
MIRRORS = {"ACBvh": "ac_bvh", "ACSceneDesc": "ac_scene_desc", "ACSceneInfo": "ac_scene_info",
           "ACTraceParams": "ac_trace_params", "ACTraceOutputs": "ac_trace_outputs", "ACJob": "ac_job",
           "ACBatchConfig": "ac_batch_config", "ACServiceConfig": "ac_service_config",
           "ACServiceStats": "ac_service_stats", "ACServiceJobState": "ac_service_job_state", "ACSynthParams": "ac_synth_params", "ACSynthJob": "ac_synth_job",
           "ACSynthBatchConfig": "ac_synth_batch_config", "ACFdnJob": "ac_fdn_job",
           "ACLateTailJob": "ac_late_tail_job", "ACDirectQuery": "ac_direct_query",
           "ACDirectResult": "ac_direct_result", "ACDirectTables": "ac_direct_tables"}


def test_ctypes_mirrors_match_the_header_layout(tmp_path):
    """Every field of every ctypes mirror sits at the header's offset, and the sizes agree (gcc, C11)."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("gcc not found")
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "acoustic_rt.h"', "int main(void) {"]
    expected = []
    for mirror, ctype in MIRRORS.items():
        cls = getattr(_lib, mirror)
        lines.append(f'    printf("{ctype} sizeof %zu\\n", sizeof({ctype}));')
        expected.append(f"{ctype} sizeof {ctypes.sizeof(cls)}")
        for name, *_ in cls._fields_:
            lines.append(f'    printf("{ctype} {name} %zu\\n", offsetof({ctype}, {name}));')
            expected.append(f"{ctype} {name} {getattr(cls, name).offset}")
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", str(REPO / "include"), str(src), "-o", str(exe)], check=True,
                   capture_output=True)
    got = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    assert [g for g in got if g] == expected


def test_stack_depth_candidates_start_at_the_need():
    from acoustic_agent_b200 import autotune
    assert autotune.stack_candidates(0) == [0]
    assert autotune.stack_candidates(7) == [7, 8, 12, 16, 24, 32]
    assert autotune.stack_candidates(16) == [16, 24, 32]
    assert autotune.stack_candidates(32) == [32]
    choice = autotune.SceneChoice("bvh", 1, 1.0, 2, 12, ((12, 1.0), (16, 1.1)))
    assert choice.options()["stack_entries"] == 12


def test_scene_create_rejects_bad_descriptions_without_touching_the_gpu():
    lib = _lib.load()
    handle = ctypes.c_void_p()
    assert lib.ac_scene_create(None, ctypes.byref(handle)) == _lib.AC_ERR_INVALID
    desc = _lib.ACSceneDesc()
    desc.num_surfaces = 0
    assert lib.ac_scene_create(ctypes.byref(desc), ctypes.byref(handle)) == _lib.AC_ERR_INVALID
    assert b"at least one surface" in lib.ac_last_error()


def test_trace_validation_happens_before_launch():
    lib = _lib.load()
    params = _lib.ACTraceParams()
    outputs = _lib.ACTraceOutputs()
    assert lib.ac_trace(None, ctypes.byref(params), ctypes.byref(outputs), None) == _lib.AC_ERR_INVALID


def test_directivity_and_config_normalisation_match_reference_rules():
    assert source_directivity("cardioid")["dipole_weight"] == 0.5
    assert source_directivity({"type": "weighted_dipole", "pattern": "focused"})["dipole_power"] == 4.0
    np.testing.assert_allclose(source_forward(source_directivity({"type": "omni", "orientation_deg": 90})),
                               [0.0, 1.0, 0.0], atol=1e-15)
    with pytest.raises(ValueError):
        source_directivity("laser")
    with pytest.raises(ValueError):
        source_directivity({"type": "weighted_dipole", "dipole_weight": 1.5})
    assert normalize_precision("fp64") == "float64"
    with pytest.raises(ValueError):
        normalize_precision("float16")
    assert resolve_intersection_backend("auto", 16, 16) == "bvh"
    assert resolve_intersection_backend("auto", 15, 16) == "linear"
    with pytest.raises(ValueError):
        resolve_intersection_backend("octree", 10, 16)


def test_workloads_are_seeded_and_shaped_like_the_configs():
    a = workloads.shoebox(1729)
    assert scene.count_surfaces(a.spec) == 6 and a.config.num_bins == 100
    u = workloads.u_furnished(1729)
    assert u.num_traces == 8 and u.config.num_bins == 2000 and u.config.rt_num_rays == 200_000
    s = scene.compile_scene(u.spec)
    assert s.num_surfaces == 30
    apt = workloads.apartment(1729)
    sa = scene.compile_scene(apt.spec)
    assert 6 <= apt.meta["rooms"] <= 8 and 4 <= apt.meta["doors"] <= 8
    assert sa.num_surfaces > 200
    again = workloads.apartment(1729)
    assert again.spec == apt.spec
    mix = workloads.mixed_batch(5, 8)
    assert len(mix) == 8 and all(1 <= len(w.sources) <= 4 and 1 <= len(w.listeners) <= 8 for w in mix)


def test_synthesis_batch_validation_happens_on_the_host():
    lib = _lib.load()
    cfg = _lib.ACSynthBatchConfig()
    cfg.num_rates = 1
    cfg.sample_rates[0] = 16000
    jobs = (_lib.ACSynthJob * 2)()
    for j in jobs:
        j.num_bins, j.samples_per_bin, j.rate_index, j.rng_mode = 10, 160, 0, _lib.AC_RNG_PHILOX
    size = ctypes.c_size_t()
    assert lib.ac_synth_batch_workspace_size(jobs, 2, ctypes.byref(cfg), ctypes.byref(size)) == _lib.AC_OK
    assert size.value >= 2 * 6 * 1600 * 8          # the raw band signals alone
    jobs[1].rate_index = 1
    assert lib.ac_synth_batch_workspace_size(jobs, 2, ctypes.byref(cfg), ctypes.byref(size)) == _lib.AC_ERR_INVALID
    assert b"rate_index" in lib.ac_last_error()
    jobs[1].rate_index = 0
    jobs[1].rng_mode = _lib.AC_RNG_REFERENCE
    # reference noise without a noise buffer, and null echograms, are refused before any device work
    assert lib.ac_synthesize_batch(jobs, 2, ctypes.byref(cfg), None, 0, None, None) == _lib.AC_ERR_INVALID
    cfg.num_rates = 0
    assert lib.ac_synth_batch_workspace_size(jobs, 2, ctypes.byref(cfg), ctypes.byref(size)) == _lib.AC_ERR_INVALID


def test_scene_size_limit_is_checked_before_any_device_work():
    lib = _lib.load()
    desc = _lib.ACSceneDesc()
    desc.num_surfaces = 1 << 22
    handle = ctypes.c_void_p()
    assert lib.ac_scene_create(ctypes.byref(desc), ctypes.byref(handle)) == _lib.AC_ERR_CAPACITY
    assert b"surfaces" in lib.ac_last_error()


def test_empty_batches_are_accepted():
    lib = _lib.load()
    cfg = _lib.ACBatchConfig(0, 0, 0, 0)
    size = ctypes.c_size_t()
    assert lib.ac_batch_workspace_size(None, 0, ctypes.byref(cfg), ctypes.byref(size)) == _lib.AC_OK
    scfg = _lib.ACSynthBatchConfig()
    scfg.num_rates = 1
    scfg.sample_rates[0] = 16000
    assert lib.ac_synth_batch_workspace_size(None, 0, ctypes.byref(scfg), ctypes.byref(size)) == _lib.AC_OK
    assert lib.ac_synthesize_batch(None, 0, ctypes.byref(scfg), None, 0, None, None) == _lib.AC_OK


def test_batch_queue_rejects_null_arguments_without_a_device():
    """The queue entry points validate their pointers before any CUDA call (usable on a CPU-only host)."""
    import ctypes
    from acoustic_agent_b200 import _lib
    lib = _lib.load()
    done = ctypes.c_int32(7)
    assert lib.ac_batch_poll(None, ctypes.byref(done)) == _lib.AC_ERR_INVALID and done.value == 7
    assert lib.ac_batch_wait(None) == _lib.AC_ERR_INVALID
    assert lib.ac_batch_release(None) == _lib.AC_OK
    assert lib.ac_batch_submit(None, 0, None, None, 0, None, None, None) == _lib.AC_ERR_INVALID


def test_service_config_and_arguments_are_checked_before_any_cuda_call():
    """ac_service_create refuses bad configurations (ring size, launch shape, stack depth, reserved blocks)
    and the other service entry points refuse null handles, all before touching a device."""
    import ctypes
    from acoustic_agent_b200 import _lib
    lib = _lib.load()
    handle = ctypes.c_void_p()
    bad = [dict(capacity=100), dict(capacity=32), dict(block_size=48), dict(block_size=512), dict(blocks_per_sm=9),
           dict(stack_entries=33), dict(stack_entries=-1), dict(reserve_blocks=-1), dict(idle_timeout_ns=-1),
           dict(chunk_rays=-5)]
    for fields in bad:
        cfg = _lib.ACServiceConfig()
        for k, v in fields.items():
            setattr(cfg, k, v)
        assert lib.ac_service_create(ctypes.byref(cfg), ctypes.byref(handle)) == _lib.AC_ERR_INVALID, fields
        assert not handle.value
    assert lib.ac_service_create(None, ctypes.byref(handle)) == _lib.AC_ERR_INVALID
    first = ctypes.c_int64()
    assert lib.ac_service_submit(None, None, 0, ctypes.byref(first), None) == _lib.AC_ERR_INVALID
    n = ctypes.c_int32()
    assert lib.ac_service_poll(None, None, 0, ctypes.byref(n)) == _lib.AC_ERR_INVALID
    state = _lib.ACServiceJobState()
    assert lib.ac_service_inspect(None, 0, ctypes.byref(state)) == _lib.AC_ERR_INVALID
    stats = _lib.ACServiceStats()
    assert lib.ac_service_info(None, ctypes.byref(stats)) == _lib.AC_ERR_INVALID
    assert lib.ac_service_destroy(None) == _lib.AC_OK


def test_tune_cache_persists_stack_choices(tmp_path):
    """Scene choices, the stack depth and its per-depth timings included, survive a JSON round trip."""
    from acoustic_agent_b200 import autotune
    path = tmp_path / "tune.json"
    cache = autotune.TuneCache(path)
    choice = autotune.SceneChoice("bvh", 1, 0.5, 2, 12, ((12, 0.5), (16, 0.52), (32, 0.55)))
    cache.put("abc", choice)
    again = autotune.TuneCache(path)
    assert again.get("abc") == choice
    assert again.get("abc").options() == {"traversal": "bvh", "bvh_leaf": 1, "bvh_width": 2, "stack_entries": 12}
    import json                             # an entry written before the stack knob existed still loads
    path.write_text(json.dumps({"old": {"traversal": "hybrid", "bvh_leaf": 1, "ms": 1.0, "bvh_width": 2}}))
    old = autotune.TuneCache(path)
    assert old.get("old").stack_entries == 0 and old.get("old").stack_ms == ()


def test_launch_stack_depth_is_the_largest_scene_choice():
    """A launch over several scenes takes the largest of their tuned depths; a BVH scene without a choice
    (0) leaves the launch at the library's maximum; scan-only scenes need no stack."""
    from types import SimpleNamespace
    from acoustic_agent_b200 import runtime
    bvh = lambda entries: SimpleNamespace(bvh_nodes=9, stack_entries=entries)   # noqa: E731
    scan = SimpleNamespace(bvh_nodes=0, stack_entries=0)
    assert runtime.launch_stack_entries([bvh(8), bvh(14), scan]) == 14
    assert runtime.launch_stack_entries([bvh(8), bvh(0)]) == 0
    assert runtime.launch_stack_entries([scan, scan]) == 0
    assert runtime.launch_stack_entries([]) == 0


def test_parity_metrics_treat_equal_infinite_c50_as_equal():
    """A band with no energy after 50 ms has C50 = +inf in both echograms: no difference, not NaN."""
    import warnings
    from acoustic_agent_b200 import metrics
    e = np.zeros((2, 100))
    e[0, :3] = [1.0, 0.5, 0.25]           # band 0: all energy in the first 50 ms
    e[1, :60] = np.exp(-np.arange(60) / 10.0)
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        same = metrics.parity(e, e, 0.01)
    assert same["c50_db"] == 0.0 and same["c50_rel"] == 0.0 and same["edc_err_db_max"] == 0.0
    late = e.copy()
    late[0, 10] = 0.01                      # band 0 now has late energy: a finite C50 against +inf
    assert metrics.parity(late, e, 0.01)["c50_db"] == np.inf
    assert metrics.parity(late, e, 0.01)["c50_rel"] == np.inf
