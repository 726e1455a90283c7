"""The CPU oracle against golden vectors produced by the reference's own tracer.

These pin the oracle before it is trusted as the checker of the GPU kernels:
every per-ray hit-surface sequence, hit/contribution count, active-ray count
and bounce count must be identical; echogram bins agree to summation order.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN, load_case
from oracle import oracle


def run_oracle(case, threads=0, record_rays=True):
    tr = case["trace"]
    dirs, bank, rnd, idx = oracle.workspace(tr["rays"], tr["bounces"], tr["seed"])
    return oracle.trace(case["arrays"], source=tr["source"], listener=tr["listener"], directions=dirs,
                        diffuse_bank=bank, diffuse_random=rnd, diffuse_indices=idx,
                        num_bins=int(case["num_bins"]), bin_dur=tr["bin_dur"], c=343.0,
                        max_path_len=tr["duration"] * 343.0, direct_delay=float(case["direct_delay"]),
                        source_forward=case["source_forward"], dipole_weight=float(case["dipole_weight"]),
                        dipole_power=float(case["dipole_power"]), use_bvh=tr["backend"] == "bvh",
                        render_ambisonics=bool(tr.get("ambisonics")), threads=threads, record_rays=record_rays)


def test_oracle_matches_reference_trace(golden_case):
    name, case = golden_case
    res = run_oracle(case)
    np.testing.assert_array_equal(res["ray_surfaces"], case["ray_surfaces"])
    np.testing.assert_array_equal(res["hit_counts"], case["hit_counts"])
    np.testing.assert_array_equal(res["contrib_counts"], case["contrib_counts"])
    assert res["active_ray_count"] == int(case["active_ray_count"])
    assert res["actual_bounces"] == int(case["actual_bounces"])
    scale = max(float(np.max(np.abs(case["echogram"]))), 1e-300)
    np.testing.assert_allclose(res["echogram"], case["echogram"], rtol=1e-12, atol=1e-13 * scale)
    np.testing.assert_allclose(res["surface_energy"], case["surface_energy"], rtol=1e-12, atol=1e-13 * scale)
    if "ambisonic" in case:
        np.testing.assert_allclose(res["ambisonic_echogram"], case["ambisonic"], rtol=1e-12, atol=1e-13 * scale)


def test_oracle_thread_count_does_not_change_hits():
    case = load_case("u_room_kat")
    one = run_oracle(case, threads=1)
    many = run_oracle(case, threads=4)
    np.testing.assert_array_equal(one["ray_surfaces"], many["ray_surfaces"])
    np.testing.assert_allclose(one["echogram"], many["echogram"], rtol=1e-13, atol=1e-18)


def test_bvh_and_linear_agree_on_closed_room():
    a = run_oracle(load_case("shoebox_linear"))
    b = run_oracle(load_case("shoebox_bvh"))
    np.testing.assert_array_equal(a["ray_surfaces"], b["ray_surfaces"])
    np.testing.assert_allclose(a["echogram"], b["echogram"], rtol=1e-12)


def test_escaped_rays_count_a_surface_in_bvh_mode_only():
    """The escape-link walk's tie rule hands a missed ray the lowest visited surface (steam_rt.py:4501)."""
    lin = load_case("open_room_linear")
    bvh = load_case("open_room_bvh")
    assert int(np.sum(bvh["hit_counts"])) > int(np.sum(lin["hit_counts"]))
    np.testing.assert_allclose(lin["echogram"], bvh["echogram"], rtol=1e-12)


@pytest.mark.parametrize("label", ["shoebox_f64", "shoebox_f32", "furnished_f32"])
def test_oracle_synthesis_is_bit_exact(label):
    s = np.load(GOLDEN / "synthesis.npz")
    fs, bin_dur, delay, seed = s[f"{label}_meta"]
    echogram = s[f"{label}_input"]
    n = echogram.shape[1] * int(np.ceil(bin_dur * fs))
    white = np.random.default_rng(int(seed) + 7).uniform(-1.0, 1.0, size=n)
    out = oracle.synthesize(echogram, fs=int(fs), bin_dur=float(bin_dur), direct_delay=float(delay), c=343.0,
                            white=white)
    np.testing.assert_array_equal(out, s[f"{label}_output"])


def test_oracle_workspace_matches_reference():
    ws = np.load(GOLDEN / "workspace.npz")
    d, b, r, i = oracle.workspace(1000, 5, 1729)
    np.testing.assert_array_equal(d, ws["sphere"])
    np.testing.assert_array_equal(b, ws["bank"])
    np.testing.assert_array_equal(r, ws["random"])
    np.testing.assert_array_equal(i, ws["indices"])


def test_oracle_bvh_restatement(golden_case):
    _, case = golden_case
    a = case["arrays"]
    bvh = oracle.build_bvh(a["surface_bounds_min"], a["surface_bounds_max"])
    for key in ("bounds_min", "bounds_max", "start", "count", "escape", "primitives"):
        np.testing.assert_array_equal(bvh[key], a[f"bvh_{key}"])


def test_philox_known_answers():
    """Random123 known-answer vectors for Philox4x32-10."""
    vectors = [
        ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
        ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
        ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
         (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
    ]
    for ctr, key, expected in vectors:
        out = oracle.philox4x32_10(*[np.asarray([v]) for v in ctr], *key)
        assert tuple(int(v[0]) for v in out) == expected


def test_planted_error_is_caught():
    """A reflection coefficient changed in the oracle's input must change the echogram the tests compare."""
    case = load_case("u_room_kat")
    base = run_oracle(case, record_rays=False)
    case["arrays"] = dict(case["arrays"])
    refl = np.array(case["arrays"]["reflection"], copy=True)
    refl[0, 3] *= 0.9
    case["arrays"]["reflection"] = refl
    changed = run_oracle(case, record_rays=False)
    assert not np.allclose(changed["echogram"], base["echogram"], rtol=1e-6)


def test_reference_rt60_fit_restatement_on_a_known_decay():
    """schroeder_rt60 (steam_rt.py:3052-3067) on an exact exponential decay returns its RT60."""
    from acoustic_agent_b200 import metrics
    bin_dur, rt60 = 0.01, 0.5
    t = np.arange(200) * bin_dur
    energy = 10.0 ** (-6.0 * t / rt60)          # -60 dB per rt60 seconds
    assert abs(metrics.schroeder_rt60(energy, bin_dur) - rt60) < 1e-3
    assert metrics.schroeder_rt60(np.zeros(10), bin_dur) == 0.0


@pytest.mark.parametrize("rays,bounces,seed,bank", [(7, 5, 1729, 128), (64, 3, 3, 128), (33, 4, 99, 64),
                                                     (10, 3, 5, 1), (1, 6, 8, 2)])
def test_pcg64_draw_positions_equal_numpy(rays, bounces, seed, bank):
    """Each uniform and bank index of the reference's workspace sits at a fixed position of the PCG64 output
    sequence (odd ray counts carry a buffered half word across bounces; a one-entry bank draws no words)."""
    from oracle import oracle
    rnd, idx = oracle.pcg64_reference_stream(rays, bounces, seed, bank)
    g = np.random.default_rng(seed + 1)
    for b in range(bounces):
        np.testing.assert_array_equal(rnd[b], g.random(rays))
        np.testing.assert_array_equal(idx[b], g.integers(0, bank, size=rays, dtype=np.int32))


def test_pcg64_draw_positions_equal_golden_workspace():
    """The reference's own workspace (1,000 rays x 5 bounces, seed 1729, written by its
    `_diffuse_random_sequence`) from the position restatement."""
    from oracle import oracle
    g = np.load(GOLDEN / "workspace.npz")
    rnd, idx = oracle.pcg64_reference_stream(1000, 5, 1729, 128)
    np.testing.assert_array_equal(rnd, g["random"])
    np.testing.assert_array_equal(idx, g["indices"])
