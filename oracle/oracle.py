"""CPU oracle for the reflection hot path.  TEST INFRASTRUCTURE ONLY.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this module, always as the checker or the CPU baseline,
never as part of the product path.

* ``trace``        float64 tracer restated in C (trace_oracle.c), following
                   acoustic_agent/steam_rt.py:4258-4850 operation by operation
* ``synthesize``   echogram -> band signals (steam_rt.py:2205-2232, 3070-3083, 4131-4212)
* ``build_bvh``    numpy restatement of acoustic_agent/bvh.py:8-77
* ``workspace``    the reference's random workspace (steam_rt.py:3959-4044)
* ``fdn_impulse``  the sixteen-line FDN of steam_rt.py:2235-2327, restated in C
* ``fdn_design`` / ``late_reverb``  the FDN's delay and filter design and the
                   hybrid late-tail render (steam_rt.py:2330-2640), restated in numpy
* ``philox_workspace`` numpy Philox4x32-10 (Salmon et al., SC'11) producing the
                   directions / uniforms / bank indices the GPU's counter-based
                   mode draws, so that mode can be checked ray by ray

Parity is pinned against golden vectors produced by running the reference
itself (tests/golden/make_golden.py).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from pathlib import Path
from typing import Any, Mapping

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
SOURCE = ORACLE_DIR / "trace_oracle.c"
LIBRARY = ORACLE_DIR / "liboracle.so"

_d = ctypes.POINTER(ctypes.c_double)
_i64 = ctypes.POINTER(ctypes.c_int64)
_i32 = ctypes.POINTER(ctypes.c_int32)
_f32 = ctypes.POINTER(ctypes.c_float)


class _Scene(ctypes.Structure):
    _fields_ = [("num_surfaces", ctypes.c_int64), ("kinds", _i64), ("wall_a", _d), ("wall_delta", _d),
                ("wall_z", _d), ("z_values", _d), ("box_center", _d), ("box_axis_u", _d), ("box_axis_v", _d),
                ("box_half", _d), ("box_z", _d), ("normals", _d), ("reflection", _d), ("scattering", _d),
                ("num_corners", ctypes.c_int64), ("corners", _d), ("num_nodes", ctypes.c_int64), ("bvh_min", _d),
                ("bvh_max", _d), ("bvh_start", _i64), ("bvh_count", _i64), ("bvh_escape", _i64), ("bvh_prims", _i64),
                ("use_bvh", ctypes.c_int64)]


class _Params(ctypes.Structure):
    _fields_ = [("source", ctypes.c_double * 3), ("listener", ctypes.c_double * 3),
                ("source_forward", ctypes.c_double * 3), ("num_rays", ctypes.c_int64),
                ("num_bounces", ctypes.c_int64), ("num_bins", ctypes.c_int64), ("num_bank", ctypes.c_int64),
                ("bin_dur", ctypes.c_double), ("c", ctypes.c_double), ("max_path_len", ctypes.c_double),
                ("direct_delay", ctypes.c_double), ("listener_radius", ctypes.c_double),
                ("source_radius", ctypes.c_double), ("irradiance_min_distance", ctypes.c_double),
                ("specular_exponent", ctypes.c_double), ("dipole_weight", ctypes.c_double),
                ("dipole_power", ctypes.c_double), ("render_ambisonics", ctypes.c_int64),
                ("num_threads", ctypes.c_int64), ("directions", _d), ("diffuse_bank", _d), ("diffuse_random", _d),
                ("diffuse_indices", _i32)]


class _Outputs(ctypes.Structure):
    _fields_ = [("echogram", _d), ("ambisonic", _d), ("hit_counts", _i64), ("contrib_counts", _i64),
                ("surface_energy", _d), ("actual_bounces", ctypes.c_int64), ("active_count", ctypes.c_int64),
                ("ray_surfaces", _i32), ("ray_bounces", _i32), ("closest_queries", ctypes.c_int64),
                ("shadow_queries", ctypes.c_int64), ("nodes_visited", ctypes.c_int64),
                ("prims_tested", ctypes.c_int64 * 3), ("polygon_edges", ctypes.c_int64), ("ray_states", _d)]


def build(force: bool = False) -> Path:
    """Compile the C restatement (gcc, OpenMP, no FP contraction)."""
    if not force and LIBRARY.exists() and LIBRARY.stat().st_mtime >= SOURCE.stat().st_mtime:
        return LIBRARY
    tmp = LIBRARY.with_suffix(".so.tmp")
    cmd = ["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-std=c11",
           str(SOURCE), "-o", str(tmp), "-lm"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    os.replace(tmp, LIBRARY)
    return LIBRARY


_LIB: ctypes.CDLL | None = None


def _lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        if not LIBRARY.exists():
            build()
        lib = ctypes.CDLL(str(LIBRARY))
        lib.oracle_trace.restype = ctypes.c_int
        lib.oracle_trace.argtypes = [ctypes.POINTER(_Scene), ctypes.POINTER(_Params), ctypes.POINTER(_Outputs)]
        lib.oracle_closest_hit.restype = ctypes.c_int
        lib.oracle_closest_hit.argtypes = [ctypes.POINTER(_Scene), _d, _d, _d, _d]
        lib.oracle_synthesize.restype = ctypes.c_int
        lib.oracle_synthesize.argtypes = [_d, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, _d, _d, _d, _f32]
        lib.oracle_bandlimit.restype = ctypes.c_int
        lib.oracle_bandlimit.argtypes = [_d, ctypes.c_int64, _d, _f32]
        lib.oracle_fdn_impulse.restype = ctypes.c_int
        lib.oracle_fdn_impulse.argtypes = [_i64, ctypes.c_int64, _d, ctypes.c_int64, ctypes.c_int64, _i64,
                                           ctypes.c_int64, _d, _d]
        _LIB = lib
    return _LIB


def _p(a: np.ndarray, t):
    return a.ctypes.data_as(t)


class Scene:
    """Holds contiguous copies of a scene's arrays for the C oracle."""

    def __init__(self, arrays: Mapping[str, Any], use_bvh: bool) -> None:
        f = lambda k: np.ascontiguousarray(arrays[k], dtype=np.float64)
        i = lambda k: np.ascontiguousarray(arrays[k], dtype=np.int64)
        self.keep = {k: f(k) for k in ("wall_a", "wall_delta", "wall_z", "z_values", "box_center", "box_axis_u",
                                       "box_axis_v", "box_half", "box_z", "normals", "reflection", "scattering",
                                       "bvh_bounds_min", "bvh_bounds_max")}
        self.keep["corners"] = np.ascontiguousarray(np.asarray(arrays["corners"], dtype=np.float64)[:, :2])
        self.keep.update({k: i(k) for k in ("kinds", "bvh_start", "bvh_count", "bvh_escape", "bvh_primitives")})
        k = self.keep
        self.struct = _Scene(
            k["kinds"].shape[0], _p(k["kinds"], _i64), _p(k["wall_a"], _d), _p(k["wall_delta"], _d),
            _p(k["wall_z"], _d), _p(k["z_values"], _d), _p(k["box_center"], _d), _p(k["box_axis_u"], _d),
            _p(k["box_axis_v"], _d), _p(k["box_half"], _d), _p(k["box_z"], _d), _p(k["normals"], _d),
            _p(k["reflection"], _d), _p(k["scattering"], _d), k["corners"].shape[0], _p(k["corners"], _d),
            k["bvh_start"].shape[0], _p(k["bvh_bounds_min"], _d), _p(k["bvh_bounds_max"], _d),
            _p(k["bvh_start"], _i64), _p(k["bvh_count"], _i64), _p(k["bvh_escape"], _i64),
            _p(k["bvh_primitives"], _i64), 1 if use_bvh else 0)

    def closest_hit(self, origin, direction) -> tuple[int, float, np.ndarray]:
        o = np.ascontiguousarray(origin, dtype=np.float64)
        d = np.ascontiguousarray(direction, dtype=np.float64)
        t = np.zeros(1)
        n = np.zeros(3)
        s = _lib().oracle_closest_hit(ctypes.byref(self.struct), _p(o, _d), _p(d, _d), _p(t, _d), _p(n, _d))
        return int(s), float(t[0]), n


def trace(arrays: Mapping[str, Any], *, source, listener, directions, diffuse_bank, diffuse_random, diffuse_indices,
          num_bins: int, bin_dur: float, c: float, max_path_len: float, direct_delay: float,
          listener_radius: float = 0.1, source_radius: float = 0.1, irradiance_min_distance: float = 1.0,
          specular_exponent: float = 100.0, source_forward=(1.0, 0.0, 0.0), dipole_weight: float = 0.0,
          dipole_power: float = 1.0, use_bvh: bool = False, render_ambisonics: bool = False, threads: int = 0,
          record_rays: bool = False, record_states: bool = False) -> dict[str, Any]:
    """float64 trace of steam_rt.py:4708-4850 (plus per-ray hit sequences and traversal counts).

    `record_states` adds ``ray_states`` [R, B, 7]: each ray's origin, direction and path length before
    every closest-hit query (NaN after it ends).
    """
    scene = Scene(arrays, use_bvh)
    dirs = np.ascontiguousarray(directions, dtype=np.float64)
    bank = np.ascontiguousarray(diffuse_bank, dtype=np.float64)
    rnd = np.ascontiguousarray(diffuse_random, dtype=np.float64)
    idx = np.ascontiguousarray(diffuse_indices, dtype=np.int32)
    R = dirs.shape[0]
    B = rnd.shape[0]
    S = scene.keep["kinds"].shape[0]
    params = _Params()
    params.source[:] = [float(v) for v in source]
    params.listener[:] = [float(v) for v in listener]
    params.source_forward[:] = [float(v) for v in source_forward]
    params.num_rays, params.num_bounces, params.num_bins, params.num_bank = R, B, int(num_bins), bank.shape[0]
    params.bin_dur, params.c, params.max_path_len, params.direct_delay = float(bin_dur), float(c), float(max_path_len), float(direct_delay)
    params.listener_radius, params.source_radius = float(listener_radius), float(source_radius)
    params.irradiance_min_distance, params.specular_exponent = float(irradiance_min_distance), float(specular_exponent)
    params.dipole_weight, params.dipole_power = float(dipole_weight), float(dipole_power)
    params.render_ambisonics = 1 if render_ambisonics else 0
    params.num_threads = int(threads)
    params.directions, params.diffuse_bank = _p(dirs, _d), _p(bank, _d)
    params.diffuse_random, params.diffuse_indices = _p(rnd, _d), _p(idx, _i32)
    echogram = np.zeros((6, int(num_bins)))
    ambisonic = np.zeros((6, 4, int(num_bins))) if render_ambisonics else None
    hits = np.zeros(S, np.int64)
    contrib = np.zeros(S, np.int64)
    energy = np.zeros(S)
    ray_surfaces = np.zeros((R, B), np.int32) if record_rays else None
    ray_bounces = np.zeros(R, np.int32) if record_rays else None
    out = _Outputs()
    out.echogram = _p(echogram, _d)
    out.ambisonic = _p(ambisonic, _d) if ambisonic is not None else None
    out.hit_counts, out.contrib_counts, out.surface_energy = _p(hits, _i64), _p(contrib, _i64), _p(energy, _d)
    out.ray_surfaces = _p(ray_surfaces, _i32) if record_rays else None
    out.ray_bounces = _p(ray_bounces, _i32) if record_rays else None
    ray_states = np.zeros((R, B, 7)) if record_states else None
    out.ray_states = _p(ray_states, _d) if record_states else None
    rc = _lib().oracle_trace(ctypes.byref(scene.struct), ctypes.byref(params), ctypes.byref(out))
    if rc != 0:
        raise RuntimeError(f"oracle_trace failed ({rc})")
    result = {
        "echogram": echogram, "ambisonic_echogram": ambisonic, "hit_counts": hits, "contrib_counts": contrib,
        "surface_energy": energy, "actual_bounces": int(out.actual_bounces), "active_ray_count": int(out.active_count),
        "closest_queries": int(out.closest_queries), "shadow_queries": int(out.shadow_queries),
        "nodes_visited": int(out.nodes_visited), "prims_tested": [int(v) for v in out.prims_tested],
        "polygon_edges": int(out.polygon_edges),
    }
    if record_rays:
        result["ray_surfaces"] = ray_surfaces
        result["ray_bounces"] = ray_bounces
    if record_states:
        result["ray_states"] = ray_states
    return result


def first_divergence(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Per ray, the first bounce where two [R, B] hit-surface sequences differ (-1: identical)."""
    diff = np.asarray(a) != np.asarray(b)
    first = np.argmax(diff, axis=1)
    return np.where(diff.any(axis=1), first, -1)


def path_sensitivity(arrays: Mapping[str, Any], *, rays: np.ndarray, directions, diffuse_bank, diffuse_random,
                     diffuse_indices, trials: int = 32, eps: float = 1e-6, seed: int = 0,
                     target_surfaces: np.ndarray | None = None, **trace_kwargs) -> dict[str, Any]:
    """How robust each of `rays` is to float32-scale changes: every ray is traced again `trials` times in
    float64 with its initial direction turned by about `eps` radians (a seeded random offset of norm ~eps,
    renormalised; float32 rounds a unit vector's components by up to 6e-8).

    `sensitive`: the fraction of rays whose float64 hit sequence changes under at least one such turn.
    With `target_surfaces` ([R_total, B] hit sequences of another trace, e.g. a float32 one, indexed by ray):
    `reproduced`, the fraction of rays for which some turned float64 trace follows the target sequence up
    to and including the first bounce where the target leaves the unturned float64 path.
    """
    rays = np.asarray(rays, dtype=np.int64)
    dirs = np.asarray(directions, dtype=np.float64)
    rnd = np.asarray(diffuse_random, dtype=np.float64)
    idx = np.asarray(diffuse_indices, dtype=np.int32)
    base = trace(arrays, directions=dirs[rays], diffuse_bank=diffuse_bank, diffuse_random=rnd[:, rays],
                 diffuse_indices=idx[:, rays], record_rays=True, **trace_kwargs)["ray_surfaces"]
    rng = np.random.default_rng(seed)
    rep = np.repeat(rays, trials)
    turned = dirs[rep] + eps * rng.normal(size=(rep.size, 3)) / math.sqrt(3.0)
    turned /= np.linalg.norm(turned, axis=1, keepdims=True)
    pert = trace(arrays, directions=turned, diffuse_bank=diffuse_bank, diffuse_random=rnd[:, rep],
                 diffuse_indices=idx[:, rep], record_rays=True, **trace_kwargs)["ray_surfaces"]
    pert = pert.reshape(rays.size, trials, -1)
    sensitive = np.array([np.any(pert[k] != base[k][None]) for k in range(rays.size)])
    out: dict[str, Any] = {"rays": int(rays.size), "sensitive": float(sensitive.mean()) if rays.size else 0.0}
    if target_surfaces is not None:
        tgt = np.asarray(target_surfaces)[rays]
        reproduced = []
        for k in range(rays.size):
            diff = np.flatnonzero(tgt[k] != base[k])
            upto = (int(diff[0]) if diff.size else tgt.shape[1] - 1) + 1
            reproduced.append(bool(np.any(np.all(pert[k][:, :upto] == tgt[k][None, :upto], axis=1))))
        out["reproduced"] = float(np.mean(reproduced)) if reproduced else 0.0
    return out


def synthesize(echogram: np.ndarray, *, fs: int, bin_dur: float, direct_delay: float, c: float,
               white: np.ndarray) -> np.ndarray:
    """reconstruct_band_irs (steam_rt.py:2205-2232) for one echogram; float32 [6, N]."""
    e = np.asarray(echogram)
    is_f32 = e.dtype == np.float32
    e64 = np.ascontiguousarray(e, dtype=np.float64)
    num_bins = e64.shape[1]
    spb = max(1, int(math.ceil(float(bin_dur) * int(fs))))
    N = num_bins * spb
    air = air_gains(num_bins, spb, fs, direct_delay, c)
    xo = crossover_table(fs)
    w = np.ascontiguousarray(white, dtype=np.float64)
    if w.shape[0] < N:
        raise ValueError("white noise shorter than the signal")
    out = np.zeros((6, N), dtype=np.float32)
    rc = _lib().oracle_synthesize(_p(e64, _d), 1 if is_f32 else 0, num_bins, spb, _p(air, _d), _p(w, _d),
                                  _p(xo, _d), _p(out, _f32))
    if rc != 0:
        raise RuntimeError(f"oracle_synthesize failed ({rc})")
    return out


_AIR = (0.0, 0.00011513, 0.00034539, 0.00057565, 0.0011513, 0.0034539)  # acoustics.py:12-22


def air_gains(num_bins: int, spb: int, fs: int, direct_delay: float, c: float) -> np.ndarray:
    """steam_rt.py:2190-2193 / 2226-2227 per-bin air amplitude at the bin centre."""
    out = np.empty((6, num_bins))
    dd = max(0.0, float(direct_delay))
    for band, coeff in enumerate(_AIR):
        for b in range(num_bins):
            t = dd + (b + 0.5) * spb / int(fs)
            out[band, b] = math.exp(-max(0.0, coeff) * (max(0.0, t) * max(0.0, float(c))))
    return np.ascontiguousarray(out)


def crossover_table(fs: int) -> np.ndarray:
    """[5, 4, 5] low-pass sections at the inner crossovers (steam_rt.py:4123-4170)."""
    nyquist = fs * 0.5
    rows = []
    for cutoff_hz in (176.78, 353.55, 707.11, 1414.2, 2828.4):
        cutoff = float(np.clip(cutoff_hz, 1e-3, nyquist * 0.999))
        sections = []
        for s in range(4):
            q = 1.0 / (2.0 * math.cos((2.0 * s + 1.0) * math.pi / 16.0))
            w0 = 2.0 * math.pi * cutoff / fs
            cw0, sw0 = math.cos(w0), math.sin(w0)
            alpha = sw0 / (2.0 * q)
            a0 = 1.0 + alpha
            b0 = ((1.0 - cw0) / 2.0) / a0
            sections.append((b0, (1.0 - cw0) / a0, b0, (-2.0 * cw0) / a0, (1.0 - alpha) / a0))
        rows.append(sections)
    return np.ascontiguousarray(rows, dtype=np.float64)


def build_bvh(bounds_min: np.ndarray, bounds_max: np.ndarray, leaf_size: int = 4) -> dict[str, Any]:
    """acoustic_agent/bvh.py:8-77."""
    lower = np.asarray(bounds_min, dtype=np.float64)
    upper = np.asarray(bounds_max, dtype=np.float64)
    centroids = 0.5 * (lower + upper)
    mn, mx, st, ct, esc, prims = [], [], [], [], [], []
    depth_max = [0]
    leaves = [0]

    def node(ix: np.ndarray, depth: int) -> None:
        k = len(mn)
        mn.append(np.min(lower[ix], axis=0))
        mx.append(np.max(upper[ix], axis=0))
        st.append(-1)
        ct.append(0)
        esc.append(-1)
        depth_max[0] = max(depth_max[0], depth)
        if ix.size <= leaf_size:
            ordered = np.sort(ix, kind="stable")
            st[k] = len(prims)
            ct[k] = int(ordered.size)
            prims.extend(int(v) for v in ordered)
            leaves[0] += 1
        else:
            axis = int(np.argmax(np.ptp(centroids[ix], axis=0)))
            srt = ix[np.argsort(centroids[ix, axis], kind="stable")]
            half = srt.size // 2
            node(srt[:half], depth + 1)
            node(srt[half:], depth + 1)
        esc[k] = len(mn)

    node(np.arange(lower.shape[0], dtype=np.int64), 1)
    return {"bounds_min": np.asarray(mn), "bounds_max": np.asarray(mx), "start": np.asarray(st, np.int64),
            "count": np.asarray(ct, np.int64), "escape": np.asarray(esc, np.int64),
            "primitives": np.asarray(prims, np.int64), "node_count": len(mn), "leaf_count": leaves[0],
            "max_depth": depth_max[0]}


def workspace(num_rays: int, num_bounces: int, seed: int, bank_size: int = 128):
    """The reference's host random workspace (steam_rt.py:3959-4044)."""
    n = max(1, int(num_rays))
    rng = np.random.default_rng(seed)
    i = np.arange(n) + 0.5
    z = 1.0 - 2.0 * i / n
    r = np.sqrt(np.clip(1.0 - z * z, 0.0, 1.0))
    theta = i * (math.pi * (3.0 - math.sqrt(5.0))) + rng.uniform(-0.02, 0.02, n)
    directions = np.stack([np.cos(theta) * r, np.sin(theta) * r, z], axis=1)
    k = np.arange(bank_size, dtype=np.uint64)
    bits = k.copy()
    inverse = np.zeros(bank_size)
    factor = 0.5
    while np.any(bits):
        inverse += factor * (bits & 1)
        bits >>= 1
        factor *= 0.5
    u = (np.arange(bank_size, dtype=np.float64) + 0.5) / bank_size
    bank = np.stack([np.sqrt(u) * np.cos(2.0 * math.pi * inverse), np.sqrt(u) * np.sin(2.0 * math.pi * inverse),
                     np.sqrt(np.clip(1.0 - u, 0.0, 1.0))], axis=1)
    rng2 = np.random.default_rng(int(seed) + 1)
    rnd = np.empty((num_bounces, n))
    idx = np.empty((num_bounces, n), np.int32)
    for b in range(num_bounces):
        rnd[b] = rng2.random(n)
        idx[b] = rng2.integers(0, bank_size, size=n, dtype=np.int32)
    return directions, bank, rnd, idx


# ---------------------------------------------------------------------------
# Philox4x32-10 (vectorised numpy, uint64 arithmetic on 32-bit lanes)

_M0, _M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
_W0, _W1 = np.uint64(0x9E3779B9), np.uint64(0xBB67AE85)
_MASK = np.uint64(0xFFFFFFFF)


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    c0, c1, c2, c3 = (np.asarray(v, dtype=np.uint64) & _MASK for v in (c0, c1, c2, c3))
    k0 = np.uint64(int(k0) & 0xFFFFFFFF)
    k1 = np.uint64(int(k1) & 0xFFFFFFFF)
    for _ in range(10):
        p0 = _M0 * c0
        p1 = _M1 * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & _MASK
        hi1, lo1 = p1 >> np.uint64(32), p1 & _MASK
        c0, c1, c2, c3 = (hi1 ^ c1 ^ k0) & _MASK, lo1, (hi0 ^ c3 ^ k1) & _MASK, lo0
        k0 = (k0 + _W0) & _MASK
        k1 = (k1 + _W1) & _MASK
    return c0, c1, c2, c3


def _u01_53(hi, lo):
    bits = ((hi >> np.uint64(5)) << np.uint64(26)) | (lo >> np.uint64(6))
    return bits.astype(np.float64) * (1.0 / 9007199254740992.0)


def philox_workspace(num_rays: int, num_bounces: int, seed: int, stream_key: int, bank_size: int = 128):
    """Directions, diffuse uniforms and bank indices of the GPU's counter-based mode, in float64."""
    R = int(num_rays)
    ray = np.arange(R, dtype=np.uint64)
    key_lo, key_hi = int(stream_key) & 0xFFFFFFFF, (int(stream_key) >> 32) & 0xFFFFFFFF
    s0, s1 = int(seed) & 0xFFFFFFFF, (int(seed) >> 32) & 0xFFFFFFFF
    x, y, _, _ = philox4x32_10(ray, np.zeros(R, np.uint64), np.full(R, key_lo, np.uint64),
                               np.full(R, key_hi, np.uint64), s0, s1)
    # jitter U(-0.02, 0.02) rad in turns; angle = 2*pi*frac(i * (3 - sqrt 5)/2 + jitter)
    jitter = (-0.02 + 0.04 * _u01_53(x, y)) * 0.15915494309189535
    i = np.arange(R, dtype=np.float64) + 0.5
    z = 1.0 - 2.0 * i / R
    r = np.sqrt(np.clip(1.0 - z * z, 0.0, 1.0))
    turns = i * 0.3819660112501051 + jitter
    angle = np.pi * (2.0 * (turns - np.floor(turns)))
    directions = np.stack([np.cos(angle) * r, np.sin(angle) * r, z], axis=1)
    rnd = np.empty((num_bounces, R))
    idx = np.empty((num_bounces, R), np.int32)
    for b in range(num_bounces):
        x, y, zz, _ = philox4x32_10(ray, np.full(R, b + 1, np.uint64), np.full(R, key_lo, np.uint64),
                                    np.full(R, key_hi, np.uint64), s0, s1)
        rnd[b] = _u01_53(x, y)
        idx[b] = ((zz * np.uint64(bank_size)) >> np.uint64(32)).astype(np.int32)
    return directions, rnd, idx


def philox_noise(num_samples: int, seed: int) -> np.ndarray:
    """Synthesis noise of the counter-based mode: uniform(-1, 1), two samples per Philox block."""
    pairs = (int(num_samples) + 1) // 2
    p = np.arange(pairs, dtype=np.uint64)
    s0, s1 = int(seed) & 0xFFFFFFFF, (int(seed) >> 32) & 0xFFFFFFFF
    x, y, z, w = philox4x32_10(p, np.full(pairs, 1 << 24, np.uint64), np.zeros(pairs, np.uint64),
                               np.zeros(pairs, np.uint64), s0, s1)
    out = np.empty(2 * pairs)
    out[0::2] = -1.0 + 2.0 * _u01_53(x, y)
    out[1::2] = -1.0 + 2.0 * _u01_53(z, w)
    return out[:num_samples]


# ---- late reverberation: FDN design, impulse and hybrid tail ------------------

BANDS = ("125", "250", "500", "1000", "2000", "4000")
_INNER_EDGES = (176.78, 353.55, 707.11, 1414.2, 2828.4)
FDN_PRIMES = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53)
FDN_ALLPASS = (225, 341, 441, 556)


def bandlimit(signals: np.ndarray, fs: int) -> np.ndarray:
    """bandlimit_band_signals (steam_rt.py:3070-3083): float64 [6, n] -> float32 [6, n]."""
    x = np.ascontiguousarray(signals, dtype=np.float64)
    out = np.zeros(x.shape, dtype=np.float32)
    rc = _lib().oracle_bandlimit(_p(x, _d), x.shape[1], _p(crossover_table(fs), _d), _p(out, _f32))
    if rc != 0:
        raise RuntimeError(f"oracle_bandlimit failed ({rc})")
    return out


def fdn_delays(fs: int, seed: int) -> np.ndarray:
    """steam_rt.py:2330-2340: prime powers near 0.15 s / 16 lines plus a seeded 0-100 sample jitter."""
    target0 = max(1, int(0.15 * 10.0 * max(int(fs), 1) / len(FDN_PRIMES)))
    jitter = np.random.default_rng(int(seed) + 1701).integers(0, 101, size=len(FDN_PRIMES))
    out = np.empty(len(FDN_PRIMES), dtype=np.int64)
    for i, p in enumerate(FDN_PRIMES):
        target = max(1, target0 + int(jitter[i]))
        power = max(1, int(round(math.log(target) / math.log(p))))
        out[i] = max(1, p ** power)
    return out


def _shelf(cutoff: float, gain: float, fs: int, high: bool) -> np.ndarray:
    """RBJ shelving section, Q = 0.707 (steam_rt.py:2343-2378); `high` flips the sign of the (A-1) terms."""
    w0 = 2.0 * math.pi * float(cutoff) / max(float(fs), 1.0)
    cw, sw = math.cos(w0), math.sin(w0)
    alpha = sw / (2.0 * 0.707)
    A = math.sqrt(max(float(gain), 1e-6))
    ra = math.sqrt(A)
    if not high:
        a0 = (A + 1.0) + (A - 1.0) * cw + 2.0 * ra * alpha
        return np.asarray((A * ((A + 1.0) - (A - 1.0) * cw + 2.0 * ra * alpha) / a0,
                           2.0 * A * ((A - 1.0) - (A + 1.0) * cw) / a0,
                           A * ((A + 1.0) - (A - 1.0) * cw - 2.0 * ra * alpha) / a0,
                           -2.0 * ((A - 1.0) + (A + 1.0) * cw) / a0,
                           ((A + 1.0) + (A - 1.0) * cw - 2.0 * ra * alpha) / a0))
    a0 = (A + 1.0) - (A - 1.0) * cw + 2.0 * ra * alpha
    return np.asarray((A * ((A + 1.0) + (A - 1.0) * cw + 2.0 * ra * alpha) / a0,
                       -2.0 * A * ((A - 1.0) + (A + 1.0) * cw) / a0,
                       A * ((A + 1.0) + (A - 1.0) * cw - 2.0 * ra * alpha) / a0,
                       2.0 * ((A - 1.0) - (A + 1.0) * cw) / a0,
                       ((A + 1.0) - (A - 1.0) * cw - 2.0 * ra * alpha) / a0))


def _peak(low: float, high: float, gain: float, fs: int) -> np.ndarray:
    """RBJ peaking section between two edges (steam_rt.py:2381-2398)."""
    centre = math.sqrt(max(float(low) * float(high), 1e-12))
    bw = (float(high) - float(low)) / centre
    w0 = 2.0 * math.pi * centre / max(float(fs), 1.0)
    cw, sw = math.cos(w0), math.sin(w0)
    alpha = sw * bw / 2.0
    A = math.sqrt(max(float(gain), 1e-6))
    a0 = 1.0 + alpha / A
    return np.asarray(((1.0 + alpha * A) / a0, -2.0 * cw / a0, (1.0 - alpha * A) / a0, -2.0 * cw / a0,
                       (1.0 - alpha / A) / a0))


def multiband_sections(gains, fs: int) -> np.ndarray:
    """steam_rt.py:2401-2416: low shelf, four peaking sections, high shelf -> [6, 5]."""
    g = np.asarray(gains, dtype=np.float64).reshape(6)
    nyq = max(1.0, 0.5 * float(fs))
    edges = [0.0, *_INNER_EDGES, float(fs) * 0.5]
    rows = []
    for b in range(6):
        lo, hi = edges[b], edges[b + 1]
        if b == 0:
            rows.append(_shelf(min(max(hi, 1e-3), nyq * 0.999), g[b], fs, False))
        elif b == 5:
            rows.append(_shelf(min(max(lo, 1e-3), nyq * 0.999), g[b], fs, True))
        else:
            lower = min(max(lo, 1e-3), nyq * 0.998)
            upper = min(max(hi, lower + 1e-3), nyq * 0.999)
            rows.append(_peak(lower, upper, g[b], fs))
    return np.asarray(rows, dtype=np.float64)


def multiband_response(fs: int) -> np.ndarray:
    """steam_rt.py:2419-2435: log-gain response of the cascade at the band centres per unit log-gain of
    each section (probe gain 0.5)."""
    centres = np.minimum(np.asarray([float(b) for b in BANDS]), 0.9 * 0.5 * max(float(fs), 1.0))
    z = np.exp(-2.0j * math.pi * centres / max(float(fs), 1.0))
    m = np.empty((6, 6))
    for k in range(6):
        g = np.ones(6)
        g[k] = 0.5
        h = np.ones(6, dtype=np.complex128)
        for c in multiband_sections(g, fs):
            h *= (c[0] + c[1] * z + c[2] * z * z) / (1.0 + c[3] * z + c[4] * z * z)
        m[:, k] = np.log(np.maximum(np.abs(h), 1e-12)) / math.log(0.5)
    return m


def compensated_sections(gains, fs: int, response: np.ndarray | None = None) -> np.ndarray:
    """steam_rt.py:2438-2452: solve for section gains whose cascade hits the six targets."""
    want = np.clip(np.asarray(gains, dtype=np.float64).reshape(6), 1e-3, 0.999999)
    m = multiband_response(fs) if response is None else response
    try:
        logs = np.linalg.solve(m, np.log(want))
    except np.linalg.LinAlgError:
        logs = np.linalg.pinv(m) @ np.log(want)
    return multiband_sections(np.clip(np.exp(logs), 1e-3, 4.0), fs)


def fdn_design(fs: int, seed: int, rt60) -> dict[str, np.ndarray]:
    """Delays, per-line absorptive sections [16, 6, 5] and tone sections [6, 5] (steam_rt.py:2455-2470)."""
    delays = fdn_delays(fs, seed)
    t60 = np.asarray([max(0.1, float(v or 0.0)) for v in rt60], dtype=np.float64)
    m = multiband_response(fs)
    absorptive = np.empty((delays.size, 6, 5))
    for line, d in enumerate(delays.astype(np.float64)):
        g = np.maximum(np.exp(-(6.91 * d) / (t60 * max(float(fs), 1.0))), 1e-3)
        absorptive[line] = compensated_sections(g, fs, m)
    tone = np.sqrt(1.0 / t60)
    tone /= max(float(np.max(tone)), 1e-12)
    return {"delays": delays, "absorptive": absorptive, "tone": multiband_sections(tone, fs),
            "allpass": np.asarray(FDN_ALLPASS, dtype=np.int64)}


def fdn_impulse(delays, absorptive, num_samples: int, allpass, tone) -> np.ndarray:
    """_fdn_impulse_kernel (steam_rt.py:2235-2327): float64 [num_samples]."""
    d = np.ascontiguousarray(delays, dtype=np.int64)
    a = np.ascontiguousarray(absorptive, dtype=np.float64)
    ap = np.ascontiguousarray(allpass, dtype=np.int64)
    t = np.ascontiguousarray(tone, dtype=np.float64)
    out = np.zeros(int(num_samples))
    rc = _lib().oracle_fdn_impulse(_p(d, _i64), d.size, _p(a, _d), a.shape[1], int(num_samples), _p(ap, _i64),
                                   ap.size, _p(t, _d), _p(out, _d))
    if rc != 0:
        raise RuntimeError(f"oracle_fdn_impulse failed ({rc})")
    return out


def late_tail_start_power(signal: np.ndarray, start: int, rt60: float, fs: int, bin_samples: int) -> float:
    """steam_rt.py:2473-2497: power at the tail start, from the bin there and the last five non-empty
    bins before it, each decayed to the start at the target RT60."""
    sq = np.square(np.asarray(signal, dtype=np.float64))
    start = min(max(0, int(start)), sq.size)
    here = sq[start:min(sq.size, start + bin_samples)]
    power = float(np.mean(here)) if here.size else 0.0
    if start <= 0:
        return power
    nb = int(math.ceil(start / bin_samples))
    energy = np.asarray([float(np.sum(sq[i * bin_samples:min(start, (i + 1) * bin_samples)])) for i in range(nb)])
    nonempty = np.flatnonzero(energy > 1e-18)
    if nonempty.size == 0:
        return power
    k = 6.0 * math.log(10.0) / max(float(rt60), 0.1)
    guesses = [(energy[i] / bin_samples) * math.exp(-k * max(0.0, (start - (float(i) + 0.5) * bin_samples)
                                                               / max(float(fs), 1.0)))
               for i in nonempty[-min(5, nonempty.size):]]
    return max(power, float(np.median(guesses)))


def late_tail_windows(num_samples: int, fs: int, transition_s: float, overlap_fraction: float,
                      decay_profiles=None):
    """Per-band crossfade start / end samples and models (steam_rt.py:2508-2541)."""
    N = int(num_samples)
    fs = max(1, int(fs))
    duration = N / fs
    trans = min(max(1.0 / fs, float(transition_s)), max(1.0 / fs, (N - 1) / fs))
    ov = float(np.clip(overlap_fraction, 0.0, 0.95))
    s0 = min(N, max(0, int(math.floor((1.0 - ov) * trans * fs))))
    e0 = min(N, max(s0 + 1, int(math.ceil(trans * fs))))
    starts, ends, models = [s0] * 6, [e0] * 6, ["configured_hybrid_transition"] * 6
    profiles = decay_profiles if isinstance(decay_profiles, Mapping) else {}
    for b, band in enumerate(BANDS):
        prof = profiles.get(band)
        if not isinstance(prof, Mapping):
            continue
        bp = float(prof.get("transition_time_s", 0.0) or 0.0)
        if str(prof.get("selected_target_source", "")) == "fitted_late_slope" and 0.0 < bp < duration:
            starts[b] = min(N - 1, max(0, int(math.floor((1.0 - ov) * bp * fs))))
            ends[b] = min(N, max(starts[b] + 1, int(math.ceil(bp * fs))))
            models[b] = "coupled_space_breakpoint"
    return starts, ends, models, trans, ov, (1.0 - ov) * trans


def late_reverb(traced: np.ndarray, bin_duration_s: float, rt60_bands: Mapping[str, float], *, fs: int, seed: int,
                transition_s: float, overlap_fraction: float, late_tail: bool = True, decay_profiles=None):
    """_render_parametric_fdn_late_reverb (steam_rt.py:2500-2640) without the metadata: float32 (out, fdn
    component) plus per-band scales and anchor powers.  Returns None for the pass-through cases."""
    x = np.asarray(traced, dtype=np.float64)
    N = x.shape[1]
    fs = max(1, int(fs))
    starts, ends, models, _, _, _ = late_tail_windows(N, fs, transition_s, overlap_fraction, decay_profiles)
    if not late_tail or min(starts) >= N:
        return None
    rt60 = [float(rt60_bands.get(b, 0.0) or 0.0) for b in BANDS]
    design = fdn_design(fs, seed, rt60)
    pre = int(np.max(design["delays"]) + np.sum(design["allpass"]))
    raw = fdn_impulse(design["delays"], design["absorptive"], N + pre, design["allpass"], design["tone"])[pre:]
    fdn = bandlimit(np.repeat(raw[None, :], 6, axis=0), fs).astype(np.float64)
    bin_samples = max(1, int(round(float(bin_duration_s) * fs)))
    scales, powers = [1.0] * 6, [0.0] * 6
    for b in range(6):
        if rt60[b] <= 0.0:
            continue
        anchor = ends[b] if models[b] == "coupled_space_breakpoint" else starts[b]
        p = late_tail_start_power(x[b], anchor, rt60[b], fs, bin_samples)
        k = 6.0 * math.log(10.0) / max(rt60[b], 0.1)
        target = float(np.sum(p * np.exp(-k * np.arange(N - anchor, dtype=np.float64) / fs)))
        unit = float(np.sum(np.square(fdn[b, anchor:])))
        scales[b] = math.sqrt(target / max(unit, 1e-24)) if target > 0.0 else 0.0
        powers[b] = p
        fdn[b, starts[b]:] *= scales[b]
    out = x.copy()
    comp = np.zeros_like(x)
    for b in range(6):
        s, e = starts[b], ends[b]
        ramp = max(1, e - s)
        alpha = np.linspace(1.0, 0.0, ramp, endpoint=False)
        out[b, s:e] *= np.sqrt(alpha)
        if e < N:
            out[b, e:] = 0.0
        w = np.ones(N - s)
        w[:ramp] = np.sqrt(1.0 - alpha)
        comp[b, s:] = fdn[b, s:] * w
    out += comp
    return out.astype(np.float32), comp.astype(np.float32), {"scales": scales, "powers": powers,
                                                             "starts": starts, "ends": ends}


# ---------------------------------------------------------------------------
# numpy's PCG64 (O'Neill 2014), restated with Python integers: pins the draw positions the device
# fill of the reference's random workspace uses (steam_rt.py:4009-4044 `_diffuse_random_sequence`).

PCG64_MULTIPLIER = 0x2360ED051FC65DA44385DF649FCCF645


def pcg64_outputs(state: int, inc: int, first: int, count: int) -> list[int]:
    """Outputs `first` .. `first + count - 1` of the generator with the given 128-bit state and increment
    (each output: one LCG step, then XSL-RR of the new state), reached by Brown's arbitrary-stride jump."""
    mask = (1 << 128) - 1
    am, ap, m, c, steps = 1, 0, PCG64_MULTIPLIER, inc, first + 1
    while steps:
        if steps & 1:
            am, ap = (am * m) & mask, (ap * m + c) & mask
        c, m, steps = ((m + 1) * c) & mask, (m * m) & mask, steps >> 1
    s = (am * state + ap) & mask
    out = []
    for _ in range(count):
        rot = s >> 122
        x = ((s >> 64) ^ s) & ((1 << 64) - 1)
        out.append(((x >> rot) | (x << ((64 - rot) & 63))) & ((1 << 64) - 1))
        s = (s * PCG64_MULTIPLIER + inc) & mask
    return out


def pcg64_reference_stream(num_rays: int, num_bounces: int, seed: int, bank_size: int = 128):
    """The uniforms [B, R] and bank indices [B, R] of `_diffuse_random_sequence`, each draw taken from its
    position in the PCG64 output sequence (power-of-two banks: numpy's Lemire map never redraws)."""
    if bank_size & (bank_size - 1):
        raise ValueError("positions are fixed only for power-of-two banks")
    st = np.random.default_rng(int(seed) + 1).bit_generator.state["state"]
    state, inc = int(st["state"]), int(st["inc"])
    R, B = int(num_rays), int(num_bounces)
    u = 1 if bank_size > 1 else 0
    shift = bank_size.bit_length() - 1
    rnd = np.empty((B, R))
    idx = np.zeros((B, R), np.int32)
    for b in range(B):
        first = b * R + (b * R * u + 1) // 2
        rnd[b] = [(x >> 11) * 2.0 ** -53 for x in pcg64_outputs(state, inc, first, R)]
        if u:
            for r in range(R):
                k = b * R + r
                p = k >> 1
                x = pcg64_outputs(state, inc, (2 * p // R + 1) * R + p, 1)[0]
                word = (x >> 32) if k & 1 else (x & 0xFFFFFFFF)
                idx[b, r] = (word << shift) >> 32
    return rnd, idx
