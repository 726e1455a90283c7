"""BVH fixture pins (CPU): the oracle and the host builder reproduce the reference's trees, and the
device build's host plan gives the reference's node counts (acoustic_agent/bvh.py:8-77)."""
from __future__ import annotations

import sys

import numpy as np
import pytest

from conftest import GOLDEN

sys.path.insert(0, str(GOLDEN))
import bvh_cases  # noqa: E402

KEYS = ("bounds_min", "bounds_max", "start", "count", "escape", "primitives")


def golden(name: str) -> dict:
    g = np.load(GOLDEN / "bvh.npz")
    out = {k: g[f"{name}_{k}"] for k in KEYS}
    out["node_count"], out["leaf_count"], out["max_depth"], out["leaf_size"] = (int(v) for v in g[f"{name}_meta"])
    return out


@pytest.mark.parametrize("name", list(bvh_cases.CASES))
def test_oracle_and_host_builder_match_the_reference_tree(name):
    from acoustic_agent_b200 import _lib
    from oracle import oracle
    lo, hi, leaf = bvh_cases.inputs(name)
    ref = golden(name)
    for tree in (oracle.build_bvh(lo, hi, leaf), _lib.build_bvh(lo, hi, leaf)):
        for k in KEYS:
            np.testing.assert_array_equal(np.asarray(tree[k]), ref[k], err_msg=f"{name} {k}")
        assert (tree["node_count"], tree["leaf_count"], tree["max_depth"]) == (
            ref["node_count"], ref["leaf_count"], ref["max_depth"])


@pytest.mark.parametrize("name", list(bvh_cases.CASES))
def test_device_plan_node_count_matches_the_reference(name):
    from acoustic_agent_b200 import _lib
    n, leaf = bvh_cases.CASES[name]
    _, _, nodes = _lib.device_bvh_plan(n, leaf)
    assert nodes == golden(name)["node_count"]


def test_device_plan_sizes_over_a_sweep():
    """Node counts of the plan equal the host builder's for sizes around the shared-memory subtree limit."""
    from acoustic_agent_b200 import _lib
    rng = np.random.default_rng(5)
    for n in (1, 2, 3, 7, 8, 9, 1023, 2047, 2048, 2049, 4095, 4096, 4097, 8193, 20000):
        for leaf in (1, 3, 4, 8, 255):
            ws, staging, nodes = _lib.device_bvh_plan(n, leaf)
            lo = rng.random((n, 3))
            assert nodes == _lib.build_bvh(lo, lo + 1.0, leaf)["node_count"], (n, leaf)
            assert ws % 256 == 0 and ws >= 32 * n and staging > 0


def test_device_plan_rejects_bad_sizes():
    from acoustic_agent_b200 import _lib
    with pytest.raises(ValueError, match="at least one surface"):
        _lib.device_bvh_plan(0, 4)
    with pytest.raises(ValueError, match="leaf size"):
        _lib.device_bvh_plan(10, 0)
    with pytest.raises(_lib.BackendError):
        _lib.device_bvh_plan(1 << 30, 4)


def test_install_routes_build_bvh_only_when_asked_and_above_the_threshold(monkeypatch):
    """install(gpu_bvh_min_surfaces=N) swaps steam_rt.build_bvh (called at steam_rt.py:881); smaller scenes keep
    the reference's function, uninstall restores it."""
    import types
    from acoustic_agent_b200 import backend, bvh
    calls = []

    def reference_build(lo, hi, *, leaf_size=4):
        calls.append(("reference", len(lo), leaf_size))
        return "reference"

    fake = types.SimpleNamespace(trace_energy_field=lambda *a, **k: None,
                                 _normalize_rt_accelerator=lambda v: str(v), build_bvh=reference_build)
    handle = backend.install(fake)
    assert fake.build_bvh is reference_build          # not asked: untouched
    handle.uninstall()
    monkeypatch.setattr(bvh, "build_bvh", lambda lo, hi, *, leaf_size=4: calls.append(("gpu", len(lo), leaf_size)) or "gpu")
    handle = backend.install(fake, gpu_bvh_min_surfaces=100)
    lo = np.zeros((99, 3))
    assert fake.build_bvh(lo, lo) == "reference"
    assert fake.build_bvh(np.zeros((100, 3)), np.zeros((100, 3)), leaf_size=2) == "gpu"
    assert calls == [("reference", 99, 4), ("gpu", 100, 2)]
    handle.uninstall()
    assert fake.build_bvh is reference_build


def test_bench_bvh_inputs_and_profiled_traffic():
    """The bvh_build workload's seeded warehouse bounds are valid input for build_bvh, and the bench finds the
    committed per-build DRAM traffic."""
    import bench
    lo, hi = bench.bvh_build_inputs(4096, seed=5)
    assert lo.shape == hi.shape == (4096, 3) and np.isfinite(lo).all() and (hi >= lo).all()
    assert np.array_equal(lo, bench.bvh_build_inputs(4096, seed=5)[0])          # seeded
    traffic = bench._profiled_value("bvh_build_warehouse_1m", "traffic_bytes_per_build_1m")
    assert traffic is not None and traffic > 96_468_920   # above the algorithmic bytes of a 2^20 build


def test_bench_reference_arm_runs_the_references_build_bvh():
    """bench.py --impl reference --workload bvh_build times the reference's own build_bvh (baseline/_ref)."""
    import bench
    ref = bench.reference_bvh(1)
    if "unavailable" in ref:
        pytest.skip(ref["unavailable"])
    assert ref["kind"] == "reference" and ref["cores"] == 1 and ref["value"] > 0
    assert str(bench.BVH_SAMPLE) in ref["sample"]


def test_host_builder_equals_the_oracle_on_random_tied_scenes():
    """Property: for any bounds drawn from a handful of values (ties on every axis, signed zeros, zero-size
    boxes) and any leaf size, the C++ restatement builds the oracle's tree array for array."""
    from hypothesis import given, settings, strategies as st
    from acoustic_agent_b200 import _lib
    from oracle import oracle
    values = st.sampled_from([-2.0, -0.5, -0.0, 0.0, 0.25, 0.5, 1.0, 3.0])

    @settings(max_examples=60, deadline=None, derandomize=True)
    @given(st.integers(1, 160).flatmap(lambda n: st.tuples(
        st.lists(st.tuples(values, values, values), min_size=n, max_size=n),
        st.lists(st.tuples(values, values, values), min_size=n, max_size=n))), st.integers(1, 8))
    def check(pairs, leaf):
        a = np.asarray(pairs[0], dtype=np.float64)
        b = np.asarray(pairs[1], dtype=np.float64)
        lo, hi = np.minimum(a, b), np.maximum(a, b)
        ours, ref = _lib.build_bvh(lo, hi, leaf), oracle.build_bvh(lo, hi, leaf)
        for k in KEYS:
            np.testing.assert_array_equal(np.asarray(ours[k]), np.asarray(ref[k]), err_msg=k)
        assert (ours["node_count"], ours["leaf_count"], ours["max_depth"]) == (
            ref["node_count"], ref["leaf_count"], ref["max_depth"])

    check()
