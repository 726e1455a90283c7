"""FDN late reverberation: the oracle and the host-side design against the reference's own outputs.

tests/golden/late_reverb.npz holds, from the reference (make_golden.py):
_steam_fdn_delays / _steam_fdn_filter_coefficients for three (fs, seed, RT60)
designs, _fdn_impulse_kernel for one of them, and the full
_render_parametric_fdn_late_reverb for four configurations of one traced
signal.  Nothing here needs a GPU.
"""
from __future__ import annotations

import json
from types import SimpleNamespace

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import oracle

from acoustic_agent_b200 import _lib, bands, late_reverb

RENDER_CASES = ("basic", "breakpoint", "zero_band", "disabled")


@pytest.fixture(scope="module")
def golden():
    g = np.load(GOLDEN / "late_reverb.npz")
    return {k: g[k] for k in g.files}


def case_args(golden, name):
    case = json.loads(str(golden[f"render_{name}_case"]))
    return case, dict(zip(bands.FREQUENCY_BANDS, case["rt60"]))


def sim_config(**overrides):
    base = dict(fs=8000, seed=1729, late_tail=True, hybrid_transition_s=0.3, hybrid_overlap_fraction=0.25,
                rt_bin_duration_s=0.01)
    base.update(overrides)
    return SimpleNamespace(**base)


@pytest.mark.parametrize("k", range(3))
def test_oracle_design_matches_reference(golden, k):
    fs, seed, *rt60 = golden[f"design{k}_meta"]
    d = oracle.fdn_design(int(fs), int(seed), rt60)
    np.testing.assert_array_equal(d["delays"], golden[f"design{k}_delays"])
    np.testing.assert_array_equal(d["absorptive"], golden[f"design{k}_absorptive"])
    np.testing.assert_array_equal(d["tone"], golden[f"design{k}_tone"])


@pytest.mark.parametrize("k", range(3))
def test_backend_design_matches_reference(golden, k):
    fs, seed, *rt60 = golden[f"design{k}_meta"]
    d = late_reverb.design(int(fs), int(seed), rt60)
    np.testing.assert_array_equal(d.delays, golden[f"design{k}_delays"])
    np.testing.assert_array_equal(d.absorptive, golden[f"design{k}_absorptive"])
    np.testing.assert_array_equal(d.tone, golden[f"design{k}_tone"])
    assert d.allpass == (225, 341, 441, 556)
    assert d.preroll == int(np.max(d.delays)) + 1563


def test_oracle_fdn_impulse_is_bit_exact(golden):
    got = oracle.fdn_impulse(golden["design2_delays"], golden["design2_absorptive"], golden["impulse"].size,
                             oracle.FDN_ALLPASS, golden["design2_tone"])
    np.testing.assert_array_equal(got, golden["impulse"])
    assert np.abs(got).max() > 1e-4


@pytest.mark.parametrize("name", RENDER_CASES)
def test_oracle_late_reverb_matches_reference(golden, name):
    case, rt60 = case_args(golden, name)
    res = oracle.late_reverb(golden["render_traced"], 0.01, rt60, fs=8000, seed=1729, transition_s=0.3,
                             overlap_fraction=0.25, late_tail=case.get("late_tail", True),
                             decay_profiles=case.get("profiles"))
    if name == "disabled":
        assert res is None
        return
    out, comp, info = res
    np.testing.assert_array_equal(out, golden[f"render_{name}_out"])
    np.testing.assert_array_equal(comp, golden[f"render_{name}_fdn"])
    meta = json.loads(str(golden[f"render_{name}_meta"]))
    for b, band in enumerate(bands.FREQUENCY_BANDS):
        if band in meta["scale_by_band"]:
            assert round(info["scales"][b], 8) == meta["scale_by_band"][band]


@pytest.mark.parametrize("name", RENDER_CASES)
def test_crossfade_windows_match_reference(golden, name):
    case, _ = case_args(golden, name)
    w = late_reverb.windows(golden["render_traced"].shape[1], 8000, 0.3, 0.25, case.get("profiles"))
    meta = json.loads(str(golden[f"render_{name}_meta"]))
    if name == "disabled":
        assert meta["transition_start_s"] == round(w.start_s, 6)
        assert meta["transition_end_s"] == round(w.transition_s, 6)
        return
    for b, band in enumerate(bands.FREQUENCY_BANDS):
        ref = meta["transition_by_band"][band]
        assert ref["start_s"] == round(w.start[b] / 8000, 6)
        assert ref["end_s"] == round(w.end[b] / 8000, 6)
        assert ref["model"] == w.model[b]
        if "anchor_s" in ref:
            assert ref["anchor_s"] == round(w.anchor(b) / 8000, 6)


def test_disabled_tail_passes_through_like_the_reference(golden):
    case, rt60 = case_args(golden, "disabled")
    out, comp, meta = late_reverb.render_parametric_fdn_late_reverb(
        golden["render_traced"], {"bin_duration_s": 0.01}, rt60, sim_config(late_tail=False))
    np.testing.assert_array_equal(out, golden["render_disabled_out"])
    np.testing.assert_array_equal(comp, golden["render_disabled_fdn"])
    assert meta == json.loads(str(golden["render_disabled_meta"]))


def test_metadata_has_the_reference_keys_and_rounding(golden):
    case, rt60 = case_args(golden, "zero_band")
    ref = json.loads(str(golden["render_zero_band_meta"]))
    w = late_reverb.windows(golden["render_traced"].shape[1], 8000, 0.3, 0.25, case.get("profiles"))
    d = late_reverb.design(8000, 1729, case["rt60"])
    stats = np.zeros((6, _lib.AC_LATE_STATS))
    for b, band in enumerate(bands.FREQUENCY_BANDS):
        stats[b, _lib.AC_LATE_SCALE] = ref["scale_by_band"].get(band, 1.0)
        stats[b, _lib.AC_LATE_POWER] = ref["anchor_power_by_band"].get(band, 0.0)
        stats[b, _lib.AC_LATE_FDN_ENERGY] = ref["fdn_energy_by_band"].get(band, 0.0)
    stats[0, _lib.AC_LATE_COMPONENT] = ref["fdn_tail_energy"]
    stats[0, _lib.AC_LATE_TRACED_TAIL] = ref["traced_tail_energy"]
    stats[0, _lib.AC_LATE_RENDERED_TAIL] = ref["rendered_tail_energy"]
    stats[0, _lib.AC_LATE_CHANGED] = 1.0
    meta = late_reverb.metadata(stats, d, w, 8000, rt60)
    assert set(meta) == set(ref)
    assert meta == ref


def test_bad_shapes_raise_like_the_reference():
    with pytest.raises(ValueError, match="expected 6 traced band IRs"):
        late_reverb.render_parametric_fdn_late_reverb(np.zeros((5, 100)), {}, {}, sim_config())


def test_fdn_validation_happens_on_the_host():
    lib = _lib.load()
    job = (_lib.ACFdnJob * 1)()
    job[0].delays[:] = [500] * 16
    job[0].allpass_delays[:] = [225, 341, 441, 556]
    job[0].num_samples = 100
    size = __import__("ctypes").c_size_t()
    assert lib.ac_fdn_workspace_size(job, 1, size) == _lib.AC_OK
    job[0].delays[3] = 40   # shorter than the pipeline allows
    assert lib.ac_fdn_workspace_size(job, 1, size) == _lib.AC_ERR_INVALID
    job[0].delays[3] = 500
    job[0].allpass_delays[0] = 16
    assert lib.ac_fdn_workspace_size(job, 1, size) == _lib.AC_ERR_INVALID
    job[0].allpass_delays[0] = 225
    job[0].absorptive[7] = float("nan")
    assert lib.ac_fdn_workspace_size(job, 1, size) == _lib.AC_ERR_INVALID
    assert lib.ac_fdn_workspace_size(job, 0, size) == _lib.AC_OK


def test_every_reference_rate_has_long_enough_delay_lines():
    for fs in (8000, 11025, 16000, 22050, 32000, 44100, 48000, 96000):
        for seed in range(20):
            assert int(np.min(late_reverb.line_delays(fs, seed))) >= _lib.AC_FDN_MIN_DELAY


def test_install_routes_the_late_tail_only_for_the_b200_accelerator():
    import types
    from acoustic_agent_b200 import backend
    calls = []
    fake = types.SimpleNamespace(
        trace_energy_field=lambda *a, **k: {"accelerator": "numba"},
        _normalize_rt_accelerator=lambda v: v if v in {"auto", "numba", "cuda"} else (_ for _ in ()).throw(
            ValueError("rt_accelerator must be auto, numba, or cuda")),
        _render_parametric_fdn_late_reverb=lambda *a, **k: calls.append("reference") or "reference")
    handle = backend.install(fake)
    traced = np.zeros((6, 100))
    cfg = sim_config(rt_accelerator="numba")
    assert fake._render_parametric_fdn_late_reverb(traced, {}, {}, cfg) == "reference"
    # the b200 accelerator takes the GPU renderer; with the tail disabled it returns without a device
    out, comp, meta = fake._render_parametric_fdn_late_reverb(traced, {}, {}, sim_config(rt_accelerator="b200",
                                                                                        late_tail=False))
    assert meta["reason"] == "disabled" and calls == ["reference"]
    handle.uninstall()
    assert fake._render_parametric_fdn_late_reverb(traced, {}, {}, cfg) == "reference"
    # a module without the late-tail function still installs
    bare = types.SimpleNamespace(trace_energy_field=fake.trace_energy_field,
                                 _normalize_rt_accelerator=fake._normalize_rt_accelerator)
    backend.install(bare).uninstall()


def test_direct_sample_sphere_matches_reference():
    from acoustic_agent_b200 import direct
    g = np.load(GOLDEN / "direct.npz")
    for count in (32, 45):
        np.testing.assert_array_equal(direct.sphere_volume_samples(count), g[f"sphere_samples_{count}"])
    assert list(direct.surface_groups(["a", "b", "a", "c", "b"])) == [0, 1, 0, 2, 1]


def test_direct_query_and_sizes_are_checked_on_the_host():
    import ctypes
    from acoustic_agent_b200 import direct
    cfg = SimpleNamespace(direct_occlusion=True, direct_occlusion_mode="raycast", direct_occlusion_radius_m=0.0,
                          direct_occlusion_samples=32, direct_transmission=False, num_transmission_rays=0)
    q = direct.make_query(np.array([1.0, 2.0, 3.0]), np.array([4.0, 5.0, 6.0]), cfg)
    assert (q.occlusion, q.volumetric, q.transmission, q.max_layers) == (1, 0, 0, 1)
    assert q.radius == 1e-4   # the reference's max(1e-4, radius)
    with pytest.raises(ValueError):
        direct.make_query(np.zeros(3), np.ones(3), SimpleNamespace(**{**vars(cfg), "num_transmission_rays": 65}))
    lib = _lib.load()
    size = ctypes.c_size_t()
    assert lib.ac_direct_workspace_size(10, ctypes.byref(size)) == _lib.AC_OK and size.value >= 10 * 72
    assert lib.ac_direct_workspace_size(-1, ctypes.byref(size)) == _lib.AC_ERR_INVALID
    # a null scene is refused before anything reaches a device
    tables = _lib.ACDirectTables()
    assert lib.ac_direct(None, (_lib.ACDirectQuery * 1)(), 1, ctypes.byref(tables), None, None, 0, None,
                         None) == _lib.AC_ERR_INVALID


def test_batched_design_equals_the_per_call_design():
    rng = np.random.default_rng(5)
    for fs in (16000, 48000):
        rt60s = rng.uniform(0.05, 3.0, (24, 6))
        rt60s[3] = 0.0
        rt60s[7, 2] = 0.0
        for got, r in zip(late_reverb.design_many(fs, 11, rt60s), rt60s):
            want = late_reverb.design(fs, 11, r)
            np.testing.assert_array_equal(got.delays, want.delays)
            np.testing.assert_array_equal(got.absorptive, want.absorptive)
            np.testing.assert_array_equal(got.tone, want.tone)


@pytest.mark.parametrize("name", ("shoebox_linear", "u_furnished_bvh", "apartment3_bvh", "objects_mix_bvh"))
def test_rt60_estimate_matches_reference(name):
    g = np.load(GOLDEN / "rt60.npz")
    echogram = np.load(GOLDEN / f"{name}.npz")["echogram"]
    for label, e in (("f64", echogram.astype(np.float64)), ("f32", echogram.astype(np.float32))):
        got = late_reverb.estimate_reverb_times(e, float(g[f"{name}_bin"]), float(g["speed_of_sound"]))
        np.testing.assert_array_equal(np.asarray(got), g[f"{name}_{label}"])
