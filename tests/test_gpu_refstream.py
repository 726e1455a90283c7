"""The reference's random workspace drawn on the device (ac_reference_stream) against numpy's own draws."""
from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rng_mod():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from acoustic_agent_b200 import rng
    return rng


@pytest.mark.parametrize("rays,bounces,seed,bank", [(1000, 5, 1729, 128), (1, 7, 3, 128), (31, 9, 4, 128),
                                                     (4097, 3, 5, 64), (513, 4, 6, 1), (200_003, 12, 1729, 128)])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_device_stream_equals_numpy(rng_mod, rays, bounces, seed, bank, dtype):
    dt = getattr(torch, dtype)
    rnd, idx = rng_mod.device_diffuse_random_sequence(rays, bounces, bank, seed, dtype=dt, device=torch.device("cuda"))
    torch.cuda.synchronize()
    want_r, want_i = rng_mod.diffuse_random_sequence(rays, bounces, bank, seed)
    np.testing.assert_array_equal(rnd.cpu().numpy(), want_r.astype(np.dtype(dtype)))
    np.testing.assert_array_equal(idx.cpu().numpy(), want_i)


def test_golden_workspace_on_the_device(rng_mod):
    """The reference's own draws (its `_diffuse_random_sequence`, 1,000 rays x 5 bounces, seed 1729)."""
    from conftest import GOLDEN
    g = np.load(GOLDEN / "workspace.npz")
    rnd, idx = rng_mod.device_diffuse_random_sequence(1000, 5, 128, 1729, dtype=torch.float64,
                                                      device=torch.device("cuda"))
    np.testing.assert_array_equal(rnd.cpu().numpy(), g["random"])
    np.testing.assert_array_equal(idx.cpu().numpy(), g["indices"])


def test_non_power_of_two_bank_is_left_to_the_host(rng_mod):
    assert rng_mod.device_diffuse_random_sequence(100, 3, 100, 1, dtype=torch.float32,
                                                  device=torch.device("cuda")) is None


def test_drop_in_default_stream_uses_device_draws(rng_mod):
    """runtime.reference_stream (the drop-in's default) gives the reference's workspace, drawn on the device."""
    from acoustic_agent_b200 import runtime
    spec = runtime.TraceSpec(source=(1.0, 1.0, 1.0), listener=(2.0, 2.0, 1.0), num_rays=3001, num_bounces=6,
                             num_bins=10, bin_duration=0.01, speed_of_sound=343.0, max_path_length=100.0,
                             direct_delay=0.0, precision="float32", rng="reference", seed=77)
    d, r, i = runtime.reference_stream(spec, torch.device("cuda"))
    want_d = rng_mod.sphere_samples(3001, 77)
    want_r, want_i = rng_mod.diffuse_random_sequence(3001, 6, 128, 77)
    np.testing.assert_array_equal(d.cpu().numpy(), want_d.astype(np.float32))
    np.testing.assert_array_equal(r.cpu().numpy(), want_r.astype(np.float32))
    np.testing.assert_array_equal(i.cpu().numpy(), want_i)
