"""Direct-path occlusion and transmission on the GPU against the reference's simulate_direct.

tests/golden/direct.npz holds, from the reference (make_golden.py), the
simulate_direct results (steam_rt.py:1315-1350) for 16 seeded source/listener
pairs in each of five golden scenes (shoebox, furnished U room, mixed object
proxies, 3-room apartment, open room) under three configurations: volumetric
occlusion, the blocking-surface ("raycast") mode, and a wide 45-sample sphere
with transmission off and two layers.  The GPU path (ac_direct, float64, the
reference's Python surface tests) must give the same occlusion fractions,
blocking surfaces and transmission products, and the same band gains.
"""
from __future__ import annotations

import json
from types import SimpleNamespace

import numpy as np
import pytest

from conftest import GOLDEN, load_case

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from acoustic_agent_b200 import bands, direct, runtime  # noqa: E402

SCENES = ("shoebox_linear", "u_furnished_bvh", "objects_mix_bvh", "apartment3_bvh", "open_room_bvh")
CONFIGS = ("volumetric", "raycast", "wide_opaque")


@pytest.fixture(scope="module")
def golden():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    g = np.load(GOLDEN / "direct.npz")
    return {k: g[k] for k in g.files}


@pytest.mark.parametrize("name", SCENES)
@pytest.mark.parametrize("label", CONFIGS)
def test_direct_path_matches_reference(golden, name, label):
    case = load_case(name)
    scene = runtime.DeviceScene(case["arrays"])
    names = [str(n) for n in golden[f"{name}_names"]]
    assert tuple(names) == tuple(case["arrays"]["names"])
    tables = direct.DirectTables(names, golden[f"{name}_transmission"], torch.device("cuda", 0))
    cfg = SimpleNamespace(**json.loads(str(golden["configs_json"]))[label])
    pairs = [(p[0], p[1]) for p in golden[f"{name}_pairs"]]
    res = direct.direct_results(scene, tables, pairs, cfg, "cardioid")
    occ = np.asarray([r["occlusion"] for r in res])
    np.testing.assert_array_equal(occ, golden[f"{name}_{label}_occlusion"])
    assert [r["occlusion_surface"] or "" for r in res] == [str(s) for s in golden[f"{name}_{label}_surface"]]
    np.testing.assert_array_equal(np.stack([r["transmission"] for r in res]), golden[f"{name}_{label}_transmission"])
    gains = np.asarray([[r["band_gains"][b] for b in bands.FREQUENCY_BANDS] for r in res])
    np.testing.assert_allclose(gains, golden[f"{name}_{label}_gains"], rtol=1e-13, atol=0)
    scene.close()


def test_batch_equals_single_queries(golden):
    name = "u_furnished_bvh"
    case = load_case(name)
    scene = runtime.DeviceScene(case["arrays"])
    tables = direct.DirectTables([str(n) for n in golden[f"{name}_names"]], golden[f"{name}_transmission"],
                                 torch.device("cuda", 0))
    cfg = SimpleNamespace(**json.loads(str(golden["configs_json"]))["volumetric"])
    pairs = [(p[0], p[1]) for p in golden[f"{name}_pairs"]]
    batch = direct.direct_results(scene, tables, pairs, cfg)
    for pair, b in zip(pairs, batch):
        one = direct.direct_results(scene, tables, [pair], cfg)[0]
        assert one["occlusion"] == b["occlusion"] and one["occlusion_surface"] == b["occlusion_surface"]
        np.testing.assert_array_equal(one["transmission"], b["transmission"])
    scene.close()
