"""ac_synthesize_static: band synthesis for callers that cannot allocate device memory.

Some callers of this library must not allocate device memory: a real-time
audio thread (cudaMalloc can block on the driver for milliseconds) or a host
engine that owns the whole device-memory budget.  ac_synthesize_static takes
the same inputs and outputs as ac_synthesize but draws its workspace from a
static device array inside the library.  These tests call it through the C
ABI and check it against ac_synthesize on two calls in a row; the file is
named to run last so that a failure here never hides the other tests.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import GOLDEN

from acoustic_agent_b200 import _lib, bands


def _params(num_rirs, num_bins, bin_dur, fs, white_ptr, air_ptr):
    from acoustic_agent_b200 import runtime  # noqa: F401  (torch import only where a GPU test needs it)
    p = _lib.ACSynthParams()
    p.num_rirs = num_rirs
    p.num_bins = num_bins
    p.samples_per_bin = bands.samples_per_bin(bin_dur, fs)
    p.sample_rate = fs
    p.rng_mode = _lib.AC_RNG_REFERENCE
    p.white_shared = 1
    p.white = white_ptr
    p.air = air_ptr
    p.air_coefficients[:] = list(bands.AIR_ABSORPTION_NP_PER_M)
    p.speed_of_sound = 343.0
    p.crossover[:] = [float(v) for v in bands.crossover_table(fs).reshape(-1)]
    return p


def test_static_entry_point_rejects_sizes_beyond_its_scratch():
    """Checked on the host before any GPU work: 8 RIRs x 2 s at 48 kHz need more than the static array."""
    p = _params(8, 2000, 0.001, 48000, 1, 1)
    rc = _lib.load().ac_synthesize_static(ctypes.c_void_p(1), ctypes.byref(p), ctypes.c_void_p(1), None)
    assert rc == _lib.AC_ERR_CAPACITY
    assert b"static scratch" in _lib.load().ac_last_error()


@pytest.mark.gpu
def test_static_entry_point_matches_workspace_entry_point_twice():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    s = np.load(GOLDEN / "synthesis.npz")
    fs, bin_dur, delay, seed = s["furnished_f32_meta"]
    fs = int(fs)
    echogram = s["furnished_f32_input"]
    nb = echogram.shape[1]
    spb = bands.samples_per_bin(float(bin_dur), fs)
    n = nb * spb
    batch = np.stack([echogram, echogram * 0.25]).astype(np.float32)
    dev = torch.device("cuda", 0)
    echo = torch.as_tensor(batch, device=dev)
    white = torch.as_tensor(np.random.default_rng(int(seed) + 7).uniform(-1.0, 1.0, size=n), device=dev)
    air_np = np.stack([bands.air_gain_table(nb, spb, fs, float(delay), 343.0)] * 2)
    air = torch.as_tensor(air_np, device=dev)
    p = _params(2, nb, float(bin_dur), fs, white.data_ptr(), air.data_ptr())
    lib = _lib.load()

    size = ctypes.c_size_t()
    _lib.check(lib.ac_synth_workspace_size(ctypes.byref(p), ctypes.byref(size)), "ac_synth_workspace_size")
    assert size.value <= _lib.AC_SYNTH_STATIC_BYTES
    workspace = torch.empty(size.value, dtype=torch.uint8, device=dev)
    expected = torch.empty(2, 6, n, dtype=torch.float32, device=dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    _lib.check(lib.ac_synthesize(ctypes.c_void_p(echo.data_ptr()), ctypes.byref(p),
                                 ctypes.c_void_p(expected.data_ptr()), ctypes.c_void_p(workspace.data_ptr()),
                                 size.value, stream), "ac_synthesize")
    torch.cuda.synchronize(dev)
    reference = expected.cpu().numpy()
    np.testing.assert_array_equal(reference[0], s["furnished_f32_output"])

    for _ in range(2):
        out = torch.full((2, 6, n), float("nan"), dtype=torch.float32, device=dev)
        _lib.check(lib.ac_synthesize_static(ctypes.c_void_p(echo.data_ptr()), ctypes.byref(p),
                                            ctypes.c_void_p(out.data_ptr()), stream), "ac_synthesize_static")
        torch.cuda.synchronize(dev)
        # the synthesis tests' bar: bit-identical output
        np.testing.assert_array_equal(out.cpu().numpy(), reference)


@pytest.mark.gpu
def test_static_entry_point_with_philox_noise_and_delay_derived_air():
    """The scratch regions the reference-noise case leaves unused: Philox noise drawn into the scratch and the
    air-absorption table built there from each RIR's direct delay (no caller table), two calls in a row."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    s = np.load(GOLDEN / "synthesis.npz")
    fs, bin_dur, delay, seed = s["furnished_f32_meta"]
    fs = int(fs)
    echogram = s["furnished_f32_input"]
    nb = echogram.shape[1]
    n = nb * bands.samples_per_bin(float(bin_dur), fs)
    dev = torch.device("cuda", 0)
    echo = torch.as_tensor(np.stack([echogram, echogram * 0.5]).astype(np.float32), device=dev)
    delays = torch.tensor([float(delay), 0.5 * float(delay)], dtype=torch.float64, device=dev)
    p = _params(2, nb, float(bin_dur), fs, None, None)
    p.rng_mode = _lib.AC_RNG_PHILOX
    p.seed = int(seed) + 7
    p.direct_delays = delays.data_ptr()
    lib = _lib.load()
    size = ctypes.c_size_t()
    _lib.check(lib.ac_synth_workspace_size(ctypes.byref(p), ctypes.byref(size)), "ac_synth_workspace_size")
    assert size.value <= _lib.AC_SYNTH_STATIC_BYTES
    workspace = torch.empty(size.value, dtype=torch.uint8, device=dev)
    expected = torch.empty(2, 6, n, dtype=torch.float32, device=dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    _lib.check(lib.ac_synthesize(ctypes.c_void_p(echo.data_ptr()), ctypes.byref(p),
                                 ctypes.c_void_p(expected.data_ptr()), ctypes.c_void_p(workspace.data_ptr()),
                                 size.value, stream), "ac_synthesize")
    torch.cuda.synchronize(dev)
    reference = expected.cpu().numpy()
    assert np.isfinite(reference).all() and np.abs(reference).max() > 0.0
    for _ in range(2):
        out = torch.full((2, 6, n), float("nan"), dtype=torch.float32, device=dev)
        _lib.check(lib.ac_synthesize_static(ctypes.c_void_p(echo.data_ptr()), ctypes.byref(p),
                                            ctypes.c_void_p(out.data_ptr()), stream), "ac_synthesize_static")
        torch.cuda.synchronize(dev)
        np.testing.assert_array_equal(out.cpu().numpy(), reference)
