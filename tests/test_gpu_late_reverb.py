"""FDN late reverberation on the GPU against the reference's outputs and the oracle.

* ac_fdn_impulse is bit-identical to the reference's float64 _fdn_impulse_kernel
  (golden vector) and to the oracle's C restatement, alone and in mixed batches,
  up to the 48 kHz / 2 s length of the U-room workload.
* The drop-in render_parametric_fdn_late_reverb matches the reference's
  _render_parametric_fdn_late_reverb on the golden cases: the band split is
  bit-identical, the energy sums differ from numpy's pairwise order by about
  1e-15 relative, so float32 outputs agree to one float32 rounding step.
* The reference's own FDN tests (tests/test_steam_audio_parity.py:458-560)
  hold for the GPU renderer.
"""
from __future__ import annotations

import json
from types import SimpleNamespace

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import oracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from acoustic_agent_b200 import _lib, bands, late_reverb, metrics, runtime  # noqa: E402

RENDER_CASES = ("basic", "breakpoint", "zero_band")


@pytest.fixture(scope="module")
def golden():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    g = np.load(GOLDEN / "late_reverb.npz")
    return {k: g[k] for k in g.files}


def sim_config(**overrides):
    base = dict(fs=8000, seed=1729, late_tail=True, hybrid_transition_s=0.3, hybrid_overlap_fraction=0.25,
                rt_bin_duration_s=0.01)
    base.update(overrides)
    return SimpleNamespace(**base)


def fdn_on_gpu(designs):
    """designs: list of (delays, absorptive, tone, num_samples, preroll); returns the float64 outputs."""
    outs = [torch.zeros(max(1, n), dtype=torch.float64, device="cuda") for *_, n, _ in designs]
    jobs = (_lib.ACFdnJob * len(designs))()
    for k, (delays, absorptive, tone, n, pre) in enumerate(designs):
        jobs[k].absorptive[:] = np.asarray(absorptive, dtype=np.float64).reshape(-1).tolist()
        jobs[k].tone[:] = np.asarray(tone, dtype=np.float64).reshape(-1).tolist()
        jobs[k].delays[:] = [int(v) for v in delays]
        jobs[k].allpass_delays[:] = list(oracle.FDN_ALLPASS)
        jobs[k].num_samples = n
        jobs[k].preroll = pre
        jobs[k].out = outs[k].data_ptr()
    ws = runtime.FdnWorkspace(torch.device("cuda"))
    runtime.fdn_impulse(jobs, len(designs), ws)
    torch.cuda.synchronize()
    return [o.cpu().numpy()[:n] for o, (*_, n, _) in zip(outs, designs)]


def test_fdn_impulse_matches_reference_bit_for_bit(golden):
    d, a, t, ref = golden["design2_delays"], golden["design2_absorptive"], golden["design2_tone"], golden["impulse"]
    whole, tail, nothing = fdn_on_gpu([(d, a, t, ref.size, 0), (d, a, t, ref.size - 1234, 1234), (d, a, t, 0, 77)])
    np.testing.assert_array_equal(whole, ref)
    np.testing.assert_array_equal(tail, ref[1234:])
    assert nothing.size == 0


def test_fdn_batch_of_mixed_rates_and_lengths_matches_the_oracle():
    cases = [(48000, 1729, (0.5, 0.5, 0.45, 0.4, 0.35, 0.3), 96000),   # the U-room RIR: 2 s at 48 kHz
             (16000, 3, (1.2, 1.0, 0.9, 0.8, 0.6, 0.4), 16000),
             (8000, 81, (1.2, 0.0, 0.9, 0.05, 0.6, 2.5), 3001),
             (44100, 5, (2.0, 1.5, 1.2, 1.0, 0.8, 0.6), 4410),
             (16000, 3, (1.2, 1.0, 0.9, 0.8, 0.6, 0.4), 1)]
    specs, expect = [], []
    for fs, seed, rt60, n in cases:
        d = oracle.fdn_design(fs, seed, rt60)
        pre = int(np.max(d["delays"]) + np.sum(d["allpass"]))
        specs.append((d["delays"], d["absorptive"], d["tone"], n, pre))
        expect.append(oracle.fdn_impulse(d["delays"], d["absorptive"], pre + n, d["allpass"], d["tone"])[pre:])
    for got, want in zip(fdn_on_gpu(specs), expect):
        np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("name", RENDER_CASES)
def test_drop_in_matches_the_reference_render(golden, name):
    case = json.loads(str(golden[f"render_{name}_case"]))
    rt60 = dict(zip(bands.FREQUENCY_BANDS, case["rt60"]))
    out, comp, meta = late_reverb.render_parametric_fdn_late_reverb(
        golden["render_traced"], {"bin_duration_s": 0.01}, rt60, sim_config(), decay_profiles=case.get("profiles"))
    ref_out, ref_comp = golden[f"render_{name}_out"], golden[f"render_{name}_fdn"]
    assert out.dtype == np.float32 and comp.dtype == np.float32 and out.shape == ref_out.shape
    # one float32 rounding step of the largest sample, from the energy sums' order
    for got, want in ((out, ref_out), (comp, ref_comp)):
        np.testing.assert_allclose(got, want, rtol=2e-7, atol=2e-7 * float(np.abs(want).max()))
    assert np.mean(out == ref_out) > 0.5
    ref = json.loads(str(golden[f"render_{name}_meta"]))
    assert set(meta) == set(ref)
    for key in ("applied", "changed", "added", "model", "transition_by_band", "delay_samples", "preroll_samples",
                "allpass_delay_samples", "transition_start_s", "transition_end_s", "rt60_bands"):
        assert meta[key] == ref[key], key
    for key in ("scale_by_band", "anchor_power_by_band", "fdn_energy_by_band"):
        assert set(meta[key]) == set(ref[key])
        for band, value in ref[key].items():
            assert meta[key][band] == pytest.approx(value, rel=1e-7, abs=1e-12), (key, band)
    for key in ("traced_tail_energy", "fdn_tail_energy", "rendered_tail_energy"):
        assert meta[key] == pytest.approx(ref[key], rel=1e-9), key


def test_batch_results_equal_each_job_alone(golden):
    r = late_reverb.renderer()
    traced = torch.from_numpy(golden["render_traced"].astype(np.float64)).cuda()
    long = torch.from_numpy(np.random.default_rng(3).uniform(-1, 1, (6, 20000)) *
                            np.exp(-np.arange(20000) / 4000.0)).cuda()
    specs = [(traced, 8000, 1729, (1.2,) * 6, 0.3), (long, 16000, 5, (0.9, 0.8, 0.7, 0.6, 0.5, 0.4), 0.8),
             (traced, 8000, 7, (1.2, 0.9, 0.0, 0.05, 0.6, 0.4), 0.2)]

    def jobs():
        return [late_reverb.LateReverbJob(t, torch.empty(t.shape, dtype=torch.float32, device="cuda"),
                                          torch.empty(t.shape, dtype=torch.float32, device="cuda"), fs, seed, rt60,
                                          0.01, trans) for t, fs, seed, rt60, trans in specs]

    together = jobs()
    stats_all, _, _ = r.render(together)
    alone = []
    for j in jobs():
        st, _, _ = r.render([j])
        alone.append((j, st))
    torch.cuda.synchronize()
    for k, (j, st) in enumerate(alone):
        assert torch.equal(j.out, together[k].out) and torch.equal(j.component, together[k].component)
        assert torch.equal(st[0], stats_all[k])


def test_reference_on_off_test_holds():
    """tests/test_steam_audio_parity.py:458-490 on the GPU renderer."""
    fs, n = 8000, 12000
    rng = np.random.default_rng(81)
    env = np.exp(-3.0 * np.log(10.0) * (np.arange(n) / fs) / 1.2)
    traced = np.vstack([rng.uniform(-1.0, 1.0, n) * env for _ in range(6)])
    rt60 = {b: 1.2 for b in bands.FREQUENCY_BANDS}
    cfg = sim_config(fs=fs, hybrid_transition_s=0.5)
    enabled, fdn, meta = late_reverb.render_parametric_fdn_late_reverb(traced, {"bin_duration_s": 0.01}, rt60, cfg)
    disabled, disabled_fdn, disabled_meta = late_reverb.render_parametric_fdn_late_reverb(
        traced, {"bin_duration_s": 0.01}, rt60, sim_config(fs=fs, hybrid_transition_s=0.5, late_tail=False))
    start = int(meta["transition_start_s"] * fs)
    assert meta["applied"] is True and meta["added"] is True and meta["delay_line_count"] == 16
    assert meta["fdn_tail_energy"] > 0.0 and disabled_meta["applied"] is False
    np.testing.assert_allclose(disabled, traced, rtol=1e-6, atol=1e-7)
    assert not np.any(disabled_fdn)
    assert float(np.sum(np.square(enabled[:, start:] - disabled[:, start:]))) > 1e-6
    assert float(np.sum(np.square(fdn[:, start:]))) > 1e-6
    # early part untouched (benchmark.py:370-390, pre-transition delta <= 1e-7)
    assert float(np.max(np.abs(enabled[:, :start] - disabled[:, :start]))) <= 1e-7


def test_reference_rt60_tracking_test_holds():
    """tests/test_steam_audio_parity.py:493-518: the hybrid IR's per-band RT60 within 12 % of the target."""
    fs, n, target = 16000, 32000, 1.2
    rng = np.random.default_rng(83)
    env = np.exp(-3.0 * np.log(10.0) * (np.arange(n) / fs) / target)
    traced = np.vstack([rng.uniform(-1.0, 1.0, n) * env for _ in range(6)])
    cfg = sim_config(fs=fs, hybrid_transition_s=0.5)
    rendered, _, meta = late_reverb.render_parametric_fdn_late_reverb(
        traced, {"bin_duration_s": 0.01}, {b: target for b in bands.FREQUENCY_BANDS}, cfg)
    assert meta["transition_start_s"] > 0.0
    bs = int(round(0.01 * fs))
    for band in range(6):
        sq = np.square(rendered[band].astype(np.float64))
        energy = np.add.reduceat(sq, np.arange(0, n, bs))
        assert metrics.schroeder_rt60(energy, bs / fs) == pytest.approx(target, rel=0.12)


def test_reference_breakpoint_test_holds():
    """tests/test_steam_audio_parity.py:521-560: a fitted breakpoint moves that band's crossfade."""
    fs, n = 8000, 12000
    rng = np.random.default_rng(89)
    traced = rng.uniform(-1.0, 1.0, (6, n)) * np.exp(-5.0 * np.arange(n) / fs)[None, :]
    _, _, meta = late_reverb.render_parametric_fdn_late_reverb(
        traced, {"bin_duration_s": 0.01}, {b: 1.0 for b in bands.FREQUENCY_BANDS},
        sim_config(fs=fs, hybrid_transition_s=1.0),
        decay_profiles={"125": {"model": "double_slope", "transition_time_s": 0.4,
                                "selected_target_source": "fitted_late_slope"}})
    assert meta["transition_by_band"]["125"] == {"start_s": 0.3, "end_s": 0.4, "model": "coupled_space_breakpoint",
                                                 "anchor_s": 0.4}
    assert meta["transition_by_band"]["250"] == {"start_s": 0.75, "end_s": 1.0,
                                                 "model": "configured_hybrid_transition", "anchor_s": 0.75}


def test_full_length_tail_matches_the_oracle():
    """A 48 kHz, 2 s RIR (the U-room length): the whole drop-in against the oracle's restatement."""
    fs, n = 48000, 96000
    rng = np.random.default_rng(5)
    env = np.exp(-3.0 * np.log(10.0) * (np.arange(n) / fs) / 0.6)
    traced = np.vstack([rng.uniform(-1.0, 1.0, n) * env for _ in range(6)]).astype(np.float32)
    rt60 = dict(zip(bands.FREQUENCY_BANDS, (0.7, 0.65, 0.6, 0.55, 0.5, 0.4)))
    cfg = sim_config(fs=fs, seed=1729, hybrid_transition_s=1.0)
    out, comp, meta = late_reverb.render_parametric_fdn_late_reverb(traced, {"bin_duration_s": 0.001}, rt60, cfg)
    ref_out, ref_comp, info = oracle.late_reverb(traced, 0.001, rt60, fs=fs, seed=1729, transition_s=1.0,
                                                 overlap_fraction=0.25)
    for got, want in ((out, ref_out), (comp, ref_comp)):
        np.testing.assert_allclose(got, want, rtol=2e-7, atol=2e-7 * float(np.abs(want).max()))
    for b, band in enumerate(bands.FREQUENCY_BANDS):
        assert meta["scale_by_band"][band] == pytest.approx(info["scales"][b], rel=1e-7)


def test_batched_late_tails_equal_the_drop_in_per_job():
    """RIRRenderer.late_tails over a mixed plan (16 and 48 kHz) equals render_parametric_fdn_late_reverb on
    each job's band IRs, with the RT60s estimated from its echogram, bit for bit."""
    from acoustic_agent_b200 import batching, scene, workloads
    ws = [workloads.shoebox(1729, rays=20000, bounces=50), workloads.u_furnished(1729, rays=20000)]
    specs, jobs = batching.workload_jobs(ws)
    jobs = jobs[:4]   # the shoebox RIR and three U-room channels
    renderer = batching.RIRRenderer(0)
    plan = renderer.plan([scene.compile_scene(s) for s in specs], jobs)
    renderer.launch(plan)
    tails = renderer.late_tails(plan)
    torch.cuda.synchronize()
    band_irs = renderer.results(plan)
    # the shoebox's traced energy gives RT60s; the U room's stays under the estimator's 1e-4 floor, so its
    # tails take the reference's zero-RT60 path (design at 0.1 s, FDN bands left unscaled)
    assert (tails.rt60[0] > 0).all()
    for k, j in enumerate(plan.jobs):
        rt60 = dict(zip(bands.FREQUENCY_BANDS, tails.rt60[k]))
        cfg = sim_config(fs=j.fs, seed=int(j.spec.seed), hybrid_transition_s=1.0, hybrid_overlap_fraction=0.25,
                         rt_bin_duration_s=j.spec.bin_duration)
        out, comp, _ = late_reverb.render_parametric_fdn_late_reverb(band_irs[k], {"bin_duration_s": j.spec.bin_duration},
                                                                     rt60, cfg)
        np.testing.assert_array_equal(tails.irs[k].cpu().numpy(), out)
        n = out.size
        start = sum(t.numel() for t in plan.irs[:k])
        np.testing.assert_array_equal(tails.component[start:start + n].cpu().numpy().reshape(out.shape), comp)
    for s in plan.scenes:
        s.close()
