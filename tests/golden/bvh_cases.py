"""Inputs of the BVH fixture (tests/golden/bvh.npz): seeded surface bounds with the shapes the
reference's build_bvh (acoustic_agent/bvh.py:8-77) meets, and the degenerate ones its stable sorts
must order (ties on every axis, identical boxes, signed zeros).  Shared by make_golden.py, which
stores the reference's trees for them, and by the tests, which rebuild the inputs from the seeds."""
from __future__ import annotations

import numpy as np

# name: (surfaces, leaf size)
CASES = {
    "single": (1, 4),
    "four": (4, 4),
    "five": (5, 4),
    "random_2500": (2500, 4),
    "grid_5000": (5000, 4),
    "identical_3000": (3000, 4),
    "zeros_700": (700, 2),
    "quant_4500_leaf1": (4500, 1),
    "quant_2100_leaf8": (2100, 8),
}


def inputs(name: str) -> tuple[np.ndarray, np.ndarray, int]:
    n, leaf = CASES[name]
    rng = np.random.default_rng(sum(map(ord, name)))
    if name == "grid_5000":          # centroids on an 8x8x4 lattice: thousands of exact ties per axis
        lo = rng.integers(0, 8, (n, 3)).astype(np.float64)
        lo[:, 2] = rng.integers(0, 4, n)
        hi = lo + rng.integers(0, 3, (n, 3))
    elif name == "identical_3000":
        lo = np.tile([1.25, -2.0, 0.0], (n, 1))
        hi = np.tile([3.5, 4.0, 2.75], (n, 1))
    elif name == "zeros_700":        # -0.0 and +0.0 compare equal in the reference's sorts
        lo = rng.choice([-0.0, 0.0, 0.5, -0.5], (n, 3))
        hi = lo.copy()
    elif name.startswith("quant"):   # multiples of 1/16: ties, exact halves
        lo = rng.integers(0, 64, (n, 3)) / 16.0
        hi = lo + rng.integers(0, 16, (n, 3)) / 16.0
    else:
        lo = rng.uniform(-20.0, 20.0, (n, 3))
        hi = lo + rng.uniform(0.0, 3.0, (n, 3))
    return np.ascontiguousarray(lo), np.ascontiguousarray(hi), leaf
