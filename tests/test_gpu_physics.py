"""Physics known answers for the float32 production path.

Mirrors the reference's shoebox RT60 check (benchmark.py:268-298): a 6 x 4 x
2.8 m shoebox with uniform absorption 0.25 and scattering 0.05, source at
(1.3, 1.1, 1.4), receiver at (4.7, 2.9, 1.4).  The traced decay time (the
reference's own Schroeder fit, -5 to -25 dB, median over the six bands) must
be within 15 % of Eyring's formula -- the reference's "quick" tolerance.  The
float64 oracle (the reference algorithm) gives 0.397 s against Eyring's 0.362 s
(+9.8 %) and Sabine's 0.416 s on this case.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

SIZE = (6.0, 4.0, 2.8)
ALPHA = 0.25


@pytest.fixture(scope="module")
def shoebox_field():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from acoustic_agent_b200 import metrics, runtime, scene
    spec = {"corners": [(0.0, 0.0), (SIZE[0], 0.0), (SIZE[0], SIZE[1]), (0.0, SIZE[1])], "height": SIZE[2],
            "materials": {k: {"absorption": [ALPHA] * 6, "scattering": [0.05] * 6}
                          for k in ("wall", "floor", "ceiling")}}
    arrays = scene.compile_scene(spec)
    src, rcv = np.array([1.3, 1.1, 1.4]), np.array([4.7, 2.9, 1.4])
    dev = runtime.DeviceScene(arrays)
    c, duration, bin_dur = 343.0, 1.2, 0.01
    tspec = runtime.TraceSpec(source=src, listener=rcv, num_rays=200_000, num_bounces=200,
                              num_bins=int(math.ceil(duration / bin_dur)), bin_duration=bin_dur, speed_of_sound=c,
                              max_path_length=duration * c, direct_delay=float(np.linalg.norm(src - rcv)) / c,
                              precision="float32", rng="philox", seed=7, stream_key=1)
    buffers = runtime.trace(dev, tspec)
    torch.cuda.synchronize()
    echogram = buffers.echogram.cpu().numpy()
    dev.close()
    return metrics, echogram, bin_dur


def test_shoebox_rt60_matches_eyring(shoebox_field):
    metrics, echogram, bin_dur = shoebox_field
    volume = SIZE[0] * SIZE[1] * SIZE[2]
    surface = 2.0 * (SIZE[0] * SIZE[1] + SIZE[0] * SIZE[2] + SIZE[1] * SIZE[2])
    eyring = 0.161 * volume / (-surface * math.log(1.0 - ALPHA))
    sabine = 0.161 * volume / (surface * ALPHA)
    rt60 = np.array([metrics.schroeder_rt60(echogram[b], bin_dur) for b in range(6)])
    assert (rt60 > 0).all()
    measured = float(np.median(rt60))
    assert abs(measured - eyring) / eyring <= 0.15, (measured, eyring, sabine)
    # uniform absorption: the six bands decay alike
    assert float(rt60.max() - rt60.min()) / measured < 0.02
