"""Ray and scattering random streams.

Two modes feed the tracer:

* reference stream: the exact host arrays Acoustic Agent draws
  (acoustic_agent/steam_rt.py:3959-3968 ``_sphere_samples``, :3990-4006
  ``_diffuse_sample_bank``, :4009-4044 ``_diffuse_random_sequence``), so a GPU
  trace can be compared ray by ray with the reference's own tracer;
* Philox: the kernels draw the same quantities from a counter-based stream
  keyed by (seed, scene, ray, bounce) and need no workspace at all.

The diffuse sample bank (a bit-reversed cosine-weighted disc) is used by
both modes.
"""
from __future__ import annotations

import math
from collections import OrderedDict
from threading import Lock

import numpy as np

_CACHE_LOCK = Lock()
_STREAM_CACHE: OrderedDict[tuple[int, int, int, int], tuple[np.ndarray, np.ndarray]] = OrderedDict()
_STREAM_CACHE_BYTES = 256 * 1024 * 1024
_stream_bytes = 0


def sphere_samples(n: int, seed: int) -> np.ndarray:
    """Jittered Fibonacci sphere directions [n, 3] (steam_rt.py:3959-3968)."""
    n = max(1, int(n))
    rng = np.random.default_rng(seed)
    i = np.arange(n) + 0.5
    z = 1.0 - 2.0 * i / n
    r = np.sqrt(np.clip(1.0 - z * z, 0.0, 1.0))
    theta = i * (math.pi * (3.0 - math.sqrt(5.0))) + rng.uniform(-0.02, 0.02, n)
    return np.stack([np.cos(theta) * r, np.sin(theta) * r, z], axis=1)


def diffuse_sample_bank(count: int) -> np.ndarray:
    """Bit-reversed cosine-hemisphere bank [count, 3] (steam_rt.py:3990-4006)."""
    count = max(1, int(count))
    i = np.arange(count, dtype=np.uint64)
    bits = i.copy()
    inverse = np.zeros(count, dtype=np.float64)
    factor = 0.5
    while np.any(bits):
        inverse += factor * (bits & 1)
        bits >>= 1
        factor *= 0.5
    u = (np.arange(count, dtype=np.float64) + 0.5) / count
    r = np.sqrt(u)
    theta = 2.0 * math.pi * inverse
    return np.stack([r * np.cos(theta), r * np.sin(theta), np.sqrt(np.clip(1.0 - u, 0.0, 1.0))], axis=1)


def diffuse_random_sequence(num_rays: int, num_bounces: int, sample_count: int, seed: int
                            ) -> tuple[np.ndarray, np.ndarray]:
    """Per-(bounce, ray) uniforms and bank indices from default_rng(seed + 1) (steam_rt.py:4009-4044).

    Cached up to 256 MiB like the reference's workspace cache.
    """
    global _stream_bytes
    key = (int(num_rays), int(num_bounces), int(sample_count), int(seed))
    with _CACHE_LOCK:
        hit = _STREAM_CACHE.get(key)
        if hit is not None:
            _STREAM_CACHE.move_to_end(key)
            return hit
    rng = np.random.default_rng(int(seed) + 1)
    random_values = np.empty((num_bounces, num_rays), dtype=np.float64)
    sample_indices = np.empty((num_bounces, num_rays), dtype=np.int32)
    for bounce in range(num_bounces):
        random_values[bounce] = rng.random(num_rays)
        sample_indices[bounce] = rng.integers(0, sample_count, size=num_rays, dtype=np.int32)
    random_values.setflags(write=False)
    sample_indices.setflags(write=False)
    size = random_values.nbytes + sample_indices.nbytes
    if size <= _STREAM_CACHE_BYTES:
        with _CACHE_LOCK:
            while _STREAM_CACHE and _stream_bytes + size > _STREAM_CACHE_BYTES:
                _, old = _STREAM_CACHE.popitem(last=False)
                _stream_bytes -= old[0].nbytes + old[1].nbytes
            _STREAM_CACHE[key] = (random_values, sample_indices)
            _stream_bytes += size
    return random_values, sample_indices


def pcg64_state(seed: int) -> tuple[int, int]:
    """(state, increment) of numpy's ``default_rng(seed)`` PCG64 before its first draw, as 128-bit integers."""
    st = np.random.default_rng(int(seed)).bit_generator.state
    if st["bit_generator"] != "PCG64" or st["has_uint32"]:
        raise RuntimeError("numpy's default generator is not a fresh PCG64")
    return int(st["state"]["state"]), int(st["state"]["inc"])


def device_diffuse_random_sequence(num_rays: int, num_bounces: int, sample_count: int, seed: int, *, dtype, device,
                                   stream=None):
    """`diffuse_random_sequence` drawn on the device (ac_reference_stream), bit for bit the same draws.

    Returns (uniforms [B, R] in `dtype`, bank indices [B, R] int32) as device tensors, or None when the bank
    size is not a power of two (numpy can then redraw a word, which only the host sequence reproduces).
    """
    import ctypes

    import torch

    from acoustic_agent_b200 import _lib
    if sample_count < 1 or sample_count & (sample_count - 1):
        return None
    state, inc = pcg64_state(int(seed) + 1)
    mask = (1 << 64) - 1
    random_values = torch.empty(int(num_bounces), int(num_rays), dtype=dtype, device=device)
    indices = torch.empty(int(num_bounces), int(num_rays), dtype=torch.int32, device=device)
    s = stream if stream is not None else torch.cuda.current_stream(device)
    precision = _lib.AC_PRECISION_FP64 if dtype == torch.float64 else _lib.AC_PRECISION_FP32
    _lib.check(_lib.load().ac_reference_stream(state >> 64, state & mask, inc >> 64, inc & mask, int(num_rays),
                                               int(num_bounces), int(sample_count), precision,
                                               ctypes.c_void_p(random_values.data_ptr()),
                                               ctypes.c_void_p(indices.data_ptr()), ctypes.c_void_p(s.cuda_stream)),
               "ac_reference_stream")
    return random_values, indices


def reference_white_noise(num_samples: int, seed: int) -> np.ndarray:
    """Coherent band noise of reconstruct_band_irs: default_rng(seed + 7).uniform(-1, 1) (steam_rt.py:2209-2210)."""
    rng = np.random.default_rng(int(seed) + 7)
    return rng.uniform(-1.0, 1.0, size=int(num_samples)).astype(np.float64)


def stream_key(*parts: object) -> int:
    """Stable 64-bit key for a scene / job identity (FNV-1a over the parts' reprs)."""
    h = 0xCBF29CE484222325
    for part in parts:
        for byte in repr(part).encode("utf-8"):
            h ^= byte
            h = (h * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h
