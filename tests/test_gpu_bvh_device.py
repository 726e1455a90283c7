"""GPU BVH build (ac_bvh_build_device) against the reference's trees (acoustic_agent/bvh.py:8-77).

Bit-exact, array by array: the reference's own trees on the seeded fixture cases and on the scene
fixtures' BVHs, the host restatement on sizes around the shared-memory subtree limit (2048 surfaces)
and at up to 2^20 surfaces (many levels of the cooperative median search), with ties on every axis,
identical boxes and signed zeros.  Invalid bounds raise the reference's errors.
"""
from __future__ import annotations

import sys

import numpy as np
import pytest

from conftest import GOLDEN, TRACE_CASES, load_case

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

sys.path.insert(0, str(GOLDEN))
import bvh_cases  # noqa: E402

KEYS = ("bounds_min", "bounds_max", "start", "count", "escape", "primitives")


@pytest.fixture(scope="module")
def bvh():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from acoustic_agent_b200 import bvh as module
    return module


def assert_same_tree(tree: dict, ref: dict, what: str) -> None:
    for k in KEYS:
        np.testing.assert_array_equal(np.asarray(tree[k]), np.asarray(ref[k]), err_msg=f"{what}: {k}")
    for k in ("node_count", "leaf_count", "max_depth"):
        assert int(tree[k]) == int(ref[k]), (what, k)


@pytest.mark.parametrize("name", list(bvh_cases.CASES))
def test_reference_trees(bvh, name):
    lo, hi, leaf = bvh_cases.inputs(name)
    g = np.load(GOLDEN / "bvh.npz")
    ref = {k: g[f"{name}_{k}"] for k in KEYS}
    ref["node_count"], ref["leaf_count"], ref["max_depth"], _ = (int(v) for v in g[f"{name}_meta"])
    assert_same_tree(bvh.build_bvh(lo, hi, leaf_size=leaf), ref, name)


@pytest.mark.parametrize("case", [c for c in TRACE_CASES if c.endswith("_bvh")])
def test_scene_fixture_trees(bvh, case):
    a = load_case(case)["arrays"]
    tree = bvh.build_bvh(a["surface_bounds_min"], a["surface_bounds_max"])
    ref = {k: a[f"bvh_{k}"] for k in KEYS}
    ref.update(node_count=len(ref["start"]), leaf_count=int(np.sum(ref["count"] > 0)),
               max_depth=tree["max_depth"])
    assert_same_tree(tree, ref, case)


def _inputs(kind: str, n: int, seed: int):
    rng = np.random.default_rng(seed)
    if kind == "random":
        lo = rng.uniform(-50.0, 50.0, (n, 3))
        return lo, lo + rng.uniform(0.0, 2.0, (n, 3))
    if kind == "ties":
        lo = rng.integers(0, 16, (n, 3)).astype(np.float64)
        return lo, lo + rng.integers(0, 2, (n, 3))
    if kind == "flat":       # every centroid on one plane: the z extent is zero everywhere
        lo = rng.uniform(0.0, 10.0, (n, 3))
        lo[:, 2] = 0.0
        return lo, lo + np.array([0.5, 0.5, 0.0])
    raise ValueError(kind)


@pytest.mark.parametrize("n,leaf,kind", [
    (2048, 4, "random"), (2049, 4, "random"), (4096, 1, "ties"), (4097, 4, "ties"), (8193, 2, "flat"),
    (65537, 4, "random"), (100_000, 3, "ties"), (300_000, 4, "random"),
])
def test_host_restatement_at_sizes(bvh, n, leaf, kind):
    from acoustic_agent_b200 import _lib
    lo, hi = _inputs(kind, n, n + leaf)
    assert_same_tree(bvh.build_bvh(lo, hi, leaf_size=leaf), _lib.build_bvh(lo, hi, leaf), f"{kind} {n} leaf {leaf}")


def test_a_million_surfaces_with_ties(bvh):
    from acoustic_agent_b200 import _lib
    lo, hi = _inputs("ties", 1 << 20, 11)
    assert_same_tree(bvh.build_bvh(lo, hi), _lib.build_bvh(lo, hi, 4), "ties 2^20")


def test_device_resident_builds_repeat_exactly(bvh):
    """The scatter's atomics order surfaces inside a child arbitrarily; the tree must not depend on it."""
    lo, hi = _inputs("ties", 200_000, 3)
    b = bvh.builder(0)
    dlo, dhi = torch.from_numpy(lo).cuda(), torch.from_numpy(hi).cuda()
    first = b.build(dlo, dhi).to_numpy()
    for _ in range(3):
        assert_same_tree(b.build(dlo, dhi).to_numpy(), first, "repeat")


def test_invalid_bounds_raise_the_reference_errors(bvh):
    lo = np.zeros((3000, 3))
    hi = np.ones((3000, 3))
    bad = hi.copy()
    bad[1234, 1] = np.nan
    with pytest.raises(ValueError, match="BVH bounds must be finite"):
        bvh.build_bvh(lo, bad)
    bad = hi.copy()
    bad[17, 2] = -1.0
    with pytest.raises(ValueError, match="maximum bounds must not be below minimum bounds"):
        bvh.build_bvh(lo, bad)
    with pytest.raises(ValueError, match=r"shape \[surface, 3\]"):
        bvh.build_bvh(lo[:, :2], hi[:, :2])
    with pytest.raises(ValueError, match="at least one surface"):
        bvh.build_bvh(lo[:0], hi[:0])
    # the builder stays usable after a rejected build
    tree = bvh.build_bvh(lo, hi)
    assert tree["node_count"] == 2047 and sorted(tree["primitives"].tolist()) == list(range(3000))


def test_grid_barrier_wait_is_bounded(bvh):
    """The build's grid barrier gives up after its poll limit with AC_BVH_STATUS_TIMEOUT instead of waiting for
    ever: two blocks wait for a third arrival that never comes; the kernel returns, the status says so, and the
    context stays usable for a build."""
    import ctypes
    import time
    from acoustic_agent_b200 import _lib
    lib = _lib.load()
    ws = torch.zeros(2, dtype=torch.int32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()

    def probe(blocks, expected):
        _lib.check(lib.ac_bvh_barrier_probe(blocks, expected, 1 << 16, ctypes.c_void_p(ws.data_ptr()),
                                            ctypes.c_void_p(status.data_ptr()), ctypes.c_void_p(stream.cuda_stream)),
                   "ac_bvh_barrier_probe")
        torch.cuda.synchronize()
        return int(status.item())

    assert probe(2, 2) == 0
    t0 = time.perf_counter()
    assert probe(2, 3) & _lib.AC_BVH_STATUS_TIMEOUT
    assert time.perf_counter() - t0 < 5.0
    from acoustic_agent_b200 import _lib as lib_module
    lo, hi = _inputs("random", 5000, 1)
    assert_same_tree(bvh.build_bvh(lo, hi), lib_module.build_bvh(lo, hi, 4), "after a timed-out barrier")


def test_concurrent_builds_through_one_builder(bvh):
    """Threads sharing the process's builder get their own trees (builds through one builder are serialised)."""
    from concurrent.futures import ThreadPoolExecutor
    from acoustic_agent_b200 import _lib
    inputs = [_inputs("random", 9000 + 1000 * k, k) for k in range(4)]
    with ThreadPoolExecutor(4) as pool:
        trees = list(pool.map(lambda io: bvh.build_bvh(*io), inputs))
    for (lo, hi), tree in zip(inputs, trees):
        assert_same_tree(tree, _lib.build_bvh(lo, hi, 4), "concurrent")
