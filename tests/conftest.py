"""Shared fixtures.  `-m gpu` tests need a CUDA device; everything else runs on CPU."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parent.parent
GOLDEN = Path(__file__).resolve().parent / "golden"
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))

TRACE_CASES = ("shoebox_linear", "shoebox_bvh", "u_room_kat", "circle24_bvh", "u_furnished_bvh",
               "u_furnished_linear", "objects_mix_bvh", "apartment3_bvh", "foa_single_ray", "open_room_linear",
               "open_room_bvh")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run on the B200 box)")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    from oracle import oracle
    oracle.build()
    from acoustic_agent_b200 import build as backend_build
    backend_build.build()
    yield


def load_case(name: str) -> dict:
    g = np.load(GOLDEN / f"{name}.npz")
    case = {k: g[k] for k in g.files}
    case["arrays"] = {k[6:]: g[k] for k in g.files if k.startswith("array_")}
    case["arrays"]["names"] = tuple(str(x) for x in g["array_names"])
    case["arrays"]["height"] = float(g["array_height"])
    case["spec"] = json.loads(str(g["spec_json"]))
    case["trace"] = json.loads(str(g["trace_json"]))
    case["ray_surfaces"] = g["ray_surfaces"].astype(np.int32)
    return case


@pytest.fixture(params=TRACE_CASES)
def golden_case(request):
    return request.param, load_case(request.param)
