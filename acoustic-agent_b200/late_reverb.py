"""Parametric FDN late reverberation on the GPU.

Drop-in for Acoustic Agent's ``_render_parametric_fdn_late_reverb``
(acoustic_agent/steam_rt.py:2500-2640): the traced band IRs are crossfaded
into a sixteen-line Hadamard feedback delay network whose per-band decay
follows the target RT60s.  The host side here mirrors the reference's
interface and does the small design work in float64 with the reference's
formulas, so the coefficients are bit-identical:

* delay lengths         steam_rt.py:2330-2340  ``_steam_fdn_delays``
* RBJ shelf / peaking   steam_rt.py:2343-2398
* six-band EQ cascade   steam_rt.py:2401-2416  (and its response matrix, :2419-2435)
* compensated EQ        steam_rt.py:2438-2452
* line / tone filters   steam_rt.py:2455-2470
* crossfade windows     steam_rt.py:2508-2541

The signal work runs in ``libacoustic_rt.so``: ``ac_fdn_impulse`` (the network,
bit-identical to the reference's float64 kernel) and ``ac_late_tail``
(band split, tail-power measurement, scaling and crossfade).  There is no CPU
path: without the library or a CUDA device the calls raise.
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass
from typing import Any, Mapping, Sequence

import numpy as np
import torch

from acoustic_agent_b200 import _lib, bands, runtime

NUM_LINES = _lib.AC_FDN_LINES
PRIMES = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53)
ALLPASS_DELAYS = (225, 341, 441, 556)   # steam_rt.py:2573
MODEL = "steam_style_16_line_hadamard_fdn"
CALIBRATION = ("steady-state pre-rolled feedback-loop multiband absorption, traced cutoff power, "
               "duration-integrated energy normalization, and equal-power hybrid crossfade")


# ---- design (host, float64) ------------------------------------------------

def line_delays(fs: int, seed: int) -> np.ndarray:
    """Sixteen prime-power delay lengths near 0.15 s / 16, jittered by a seeded 0-100 samples."""
    nominal = max(1, int(0.15 * 10.0 * max(int(fs), 1) / len(PRIMES)))
    jitter = np.random.default_rng(int(seed) + 1701).integers(0, 101, size=len(PRIMES))
    out = np.empty(len(PRIMES), dtype=np.int64)
    for k, prime in enumerate(PRIMES):
        want = max(1, nominal + int(jitter[k]))
        exponent = max(1, int(round(math.log(want) / math.log(int(prime)))))
        out[k] = max(1, int(prime) ** exponent)
    return out


def _rbj_terms(freq: float, gain: float, fs: int, q: float) -> tuple[float, float, float, float]:
    w0 = 2.0 * math.pi * float(freq) / max(float(fs), 1.0)
    cw, sw = math.cos(w0), math.sin(w0)
    return cw, sw / (2.0 * q), math.sqrt(max(float(gain), 1e-6)), sw


def low_shelf(cutoff: float, gain: float, fs: int) -> tuple[float, ...]:
    cw, alpha, A, _ = _rbj_terms(cutoff, gain, fs, 0.707)
    r = math.sqrt(A)
    a0 = (A + 1.0) + (A - 1.0) * cw + 2.0 * r * alpha
    return (A * ((A + 1.0) - (A - 1.0) * cw + 2.0 * r * alpha) / a0,
            2.0 * A * ((A - 1.0) - (A + 1.0) * cw) / a0,
            A * ((A + 1.0) - (A - 1.0) * cw - 2.0 * r * alpha) / a0,
            -2.0 * ((A - 1.0) + (A + 1.0) * cw) / a0,
            ((A + 1.0) + (A - 1.0) * cw - 2.0 * r * alpha) / a0)


def high_shelf(cutoff: float, gain: float, fs: int) -> tuple[float, ...]:
    cw, alpha, A, _ = _rbj_terms(cutoff, gain, fs, 0.707)
    r = math.sqrt(A)
    a0 = (A + 1.0) - (A - 1.0) * cw + 2.0 * r * alpha
    return (A * ((A + 1.0) + (A - 1.0) * cw + 2.0 * r * alpha) / a0,
            -2.0 * A * ((A - 1.0) + (A + 1.0) * cw) / a0,
            A * ((A + 1.0) + (A - 1.0) * cw - 2.0 * r * alpha) / a0,
            2.0 * ((A - 1.0) - (A + 1.0) * cw) / a0,
            ((A + 1.0) - (A - 1.0) * cw - 2.0 * r * alpha) / a0)


def peaking(low: float, high: float, gain: float, fs: int) -> tuple[float, ...]:
    centre = math.sqrt(max(float(low) * float(high), 1e-12))
    w0 = 2.0 * math.pi * centre / max(float(fs), 1.0)
    cw, sw = math.cos(w0), math.sin(w0)
    alpha = sw * ((float(high) - float(low)) / centre) / 2.0
    A = math.sqrt(max(float(gain), 1e-6))
    a0 = 1.0 + alpha / A
    return ((1.0 + alpha * A) / a0, -2.0 * cw / a0, (1.0 - alpha * A) / a0, -2.0 * cw / a0, (1.0 - alpha / A) / a0)


def eq_cascade(gains: Sequence[float], fs: int) -> np.ndarray:
    """[6, 5] sections: low shelf at the first crossover, peaking filters between crossovers, high shelf."""
    g = np.asarray(gains, dtype=np.float64).reshape(6)
    nyquist = max(1.0, 0.5 * float(fs))
    edges = bands.band_edges(fs)
    rows = np.empty((6, 5), dtype=np.float64)
    for b, (lo, hi) in enumerate(edges):
        if b == 0:
            rows[b] = low_shelf(float(np.clip(hi, 1e-3, nyquist * 0.999)), g[b], fs)
        elif b == 5:
            rows[b] = high_shelf(float(np.clip(lo, 1e-3, nyquist * 0.999)), g[b], fs)
        else:
            lower = float(np.clip(lo, 1e-3, nyquist * 0.998))
            rows[b] = peaking(lower, float(np.clip(hi, lower + 1e-3, nyquist * 0.999)), g[b], fs)
    return rows


_RESPONSE: dict[int, np.ndarray] = {}


def eq_response(fs: int) -> np.ndarray:
    """Log-magnitude of the cascade at the band centres per unit log-gain of each section (cached per rate)."""
    fs = int(fs)
    if fs not in _RESPONSE:
        centres = np.minimum(np.asarray([float(b) for b in bands.FREQUENCY_BANDS], dtype=np.float64),
                             0.9 * 0.5 * max(float(fs), 1.0))
        z = np.exp(-2.0j * math.pi * centres / max(float(fs), 1.0))
        probe = 0.5
        m = np.empty((6, 6), dtype=np.float64)
        for k in range(6):
            g = np.ones(6, dtype=np.float64)
            g[k] = probe
            h = np.ones(6, dtype=np.complex128)
            for c in eq_cascade(g, fs):
                h *= (c[0] + c[1] * z + c[2] * z * z) / (1.0 + c[3] * z + c[4] * z * z)
            m[:, k] = np.log(np.maximum(np.abs(h), 1e-12)) / math.log(probe)
        _RESPONSE[fs] = m
    return _RESPONSE[fs]


def compensated_cascade(gains: Sequence[float], fs: int) -> np.ndarray:
    """Section gains solved so the whole cascade reaches each band's target (clipped to [1e-3, 4])."""
    want = np.clip(np.asarray(gains, dtype=np.float64).reshape(6), 1e-3, 0.999999)
    m = eq_response(fs)
    try:
        logs = np.linalg.solve(m, np.log(want))
    except np.linalg.LinAlgError:
        logs = np.linalg.pinv(m) @ np.log(want)
    return eq_cascade(np.clip(np.exp(logs), 1e-3, 4.0), fs)


@dataclass(frozen=True)
class FdnDesign:
    delays: np.ndarray        # [16] int64
    absorptive: np.ndarray    # [16, 6, 5]
    tone: np.ndarray          # [6, 5]
    allpass: tuple[int, ...]

    @property
    def preroll(self) -> int:
        return int(np.max(self.delays) + sum(self.allpass))


def design(fs: int, seed: int, rt60: Sequence[float]) -> FdnDesign:
    """Delays plus per-line absorptive and output tone filters for six target RT60s."""
    delays = line_delays(fs, seed)
    t60 = np.asarray([max(0.1, float(v or 0.0)) for v in rt60], dtype=np.float64)
    absorptive = np.empty((delays.size, 6, 5), dtype=np.float64)
    for line, d in enumerate(np.asarray(delays, dtype=np.float64)):
        g = np.maximum(np.exp(-(6.91 * d) / (t60 * max(float(fs), 1.0))), 1e-3)
        absorptive[line] = compensated_cascade(g, fs)
    tone = np.sqrt(1.0 / t60)
    tone /= max(float(np.max(tone)), 1e-12)
    return FdnDesign(delays, absorptive, eq_cascade(tone, fs), ALLPASS_DELAYS)


def _cascade_many(gains: np.ndarray, fs: int) -> np.ndarray:
    """eq_cascade for many gain rows at once: [M, 6] -> [M, 6, 5], the same operations element by element."""
    g = np.asarray(gains, dtype=np.float64).reshape(-1, 6)
    nyquist = max(1.0, 0.5 * float(fs))
    out = np.empty((g.shape[0], 6, 5), dtype=np.float64)
    for b, (lo, hi) in enumerate(bands.band_edges(fs)):
        A = np.sqrt(np.maximum(g[:, b], 1e-6))
        if b == 0 or b == 5:
            cutoff = float(np.clip(hi if b == 0 else lo, 1e-3, nyquist * 0.999))
            cw, alpha, _, _ = _rbj_terms(cutoff, 1.0, fs, 0.707)
            r = np.sqrt(A)
            if b == 0:
                a0 = (A + 1.0) + (A - 1.0) * cw + 2.0 * r * alpha
                rows = (A * ((A + 1.0) - (A - 1.0) * cw + 2.0 * r * alpha) / a0,
                        2.0 * A * ((A - 1.0) - (A + 1.0) * cw) / a0,
                        A * ((A + 1.0) - (A - 1.0) * cw - 2.0 * r * alpha) / a0,
                        -2.0 * ((A - 1.0) + (A + 1.0) * cw) / a0,
                        ((A + 1.0) + (A - 1.0) * cw - 2.0 * r * alpha) / a0)
            else:
                a0 = (A + 1.0) - (A - 1.0) * cw + 2.0 * r * alpha
                rows = (A * ((A + 1.0) + (A - 1.0) * cw + 2.0 * r * alpha) / a0,
                        -2.0 * A * ((A - 1.0) + (A + 1.0) * cw) / a0,
                        A * ((A + 1.0) + (A - 1.0) * cw - 2.0 * r * alpha) / a0,
                        2.0 * ((A - 1.0) - (A + 1.0) * cw) / a0,
                        ((A + 1.0) - (A - 1.0) * cw - 2.0 * r * alpha) / a0)
        else:
            lower = float(np.clip(lo, 1e-3, nyquist * 0.998))
            upper = float(np.clip(hi, lower + 1e-3, nyquist * 0.999))
            centre = math.sqrt(max(lower * upper, 1e-12))
            w0 = 2.0 * math.pi * centre / max(float(fs), 1.0)
            cw, sw = math.cos(w0), math.sin(w0)
            alpha = sw * ((upper - lower) / centre) / 2.0
            a0 = 1.0 + alpha / A
            rows = ((1.0 + alpha * A) / a0, -2.0 * cw / a0, (1.0 - alpha * A) / a0, -2.0 * cw / a0,
                    (1.0 - alpha / A) / a0)
        out[:, b] = np.stack(rows, axis=-1)
    return out


def design_many(fs: int, seed: int, rt60s: np.ndarray) -> list[FdnDesign]:
    """design() for many RT60 rows of one sample rate and seed, with the per-line solves batched."""
    t60 = np.maximum(0.1, np.nan_to_num(np.asarray(rt60s, dtype=np.float64).reshape(-1, 6)))
    if t60.shape[0] == 0:
        return []
    delays = line_delays(fs, seed)
    d = np.asarray(delays, dtype=np.float64)
    gains = np.maximum(np.exp(-(6.91 * d)[None, :, None] / (t60[:, None, :] * max(float(fs), 1.0))), 1e-3)
    want = np.clip(gains.reshape(-1, 6), 1e-3, 0.999999)
    m = eq_response(fs)
    logs = np.linalg.solve(np.broadcast_to(m, (want.shape[0], 6, 6)), np.log(want)[..., None])[..., 0]
    absorptive = _cascade_many(np.clip(np.exp(logs), 1e-3, 4.0), fs).reshape(t60.shape[0], delays.size, 6, 5)
    tone_gains = np.sqrt(1.0 / t60)
    tone_gains /= np.maximum(np.max(tone_gains, axis=1, keepdims=True), 1e-12)
    tones = _cascade_many(tone_gains, fs)
    return [FdnDesign(delays, absorptive[k], tones[k], ALLPASS_DELAYS) for k in range(t60.shape[0])]


_Y00 = 1.0 / math.sqrt(4.0 * math.pi)   # steam_rt.py:37-38


def estimate_reverb_times(echogram: np.ndarray, bin_duration_s: float, speed_of_sound: float) -> list[float]:
    """The reference's traced RT60 per band (steam_rt.py:2727-2742): the Schroeder fit of Y00 * E, weighted
    by the band's air absorption over the bin start times (:2196-2202), with a 1e-4 energy floor."""
    from acoustic_agent_b200 import metrics
    e = np.asarray(echogram)
    times = float(bin_duration_s) * np.arange(e.shape[1], dtype=np.float64)
    distances = np.maximum(times, 0.0) * max(0.0, float(speed_of_sound))
    out = []
    for b, coeff in enumerate(bands.AIR_ABSORPTION_NP_PER_M):
        weights = np.exp(-2.0 * max(0.0, float(coeff)) * distances)
        out.append(metrics.schroeder_rt60((_Y00 * e[b]) * weights, bin_duration_s, min_total_energy=1e-4))
    return out


# ---- crossfade windows -----------------------------------------------------

@dataclass
class Windows:
    start: list[int]
    end: list[int]
    model: list[str]
    transition_s: float
    overlap: float
    start_s: float

    def anchor(self, band: int) -> int:
        return self.end[band] if self.model[band] == "coupled_space_breakpoint" else self.start[band]


def windows(num_samples: int, fs: int, transition_s: float, overlap_fraction: float,
            decay_profiles: Mapping[str, Any] | None = None) -> Windows:
    N = int(num_samples)
    fs = max(1, int(fs))
    duration = N / fs
    trans = min(max(1.0 / fs, float(transition_s)), max(1.0 / fs, (N - 1) / fs))
    overlap = float(np.clip(overlap_fraction, 0.0, 0.95))
    start_s = (1.0 - overlap) * trans
    s0 = min(N, max(0, int(math.floor(start_s * fs))))
    e0 = min(N, max(s0 + 1, int(math.ceil(trans * fs))))
    w = Windows([s0] * 6, [e0] * 6, ["configured_hybrid_transition"] * 6, trans, overlap, start_s)
    profiles = decay_profiles if isinstance(decay_profiles, Mapping) else {}
    for b, band in enumerate(bands.FREQUENCY_BANDS):
        prof = profiles.get(band)
        if not isinstance(prof, Mapping):
            continue
        breakpoint = float(prof.get("transition_time_s", 0.0) or 0.0)
        if str(prof.get("selected_target_source", "")) == "fitted_late_slope" and 0.0 < breakpoint < duration:
            w.start[b] = min(N - 1, max(0, int(math.floor((1.0 - overlap) * breakpoint * fs))))
            w.end[b] = min(N, max(w.start[b] + 1, int(math.ceil(breakpoint * fs))))
            w.model[b] = "coupled_space_breakpoint"
    return w


# ---- the GPU renderer --------------------------------------------------------

@dataclass
class LateReverbJob:
    """One RIR's hybrid tail: traced band signals in, crossfaded band signals out (all on one device)."""

    traced: torch.Tensor          # [6, N] float64
    out: torch.Tensor             # [6, N] float32
    component: torch.Tensor       # [6, N] float32, the FDN part of `out`
    fs: int
    seed: int
    rt60: Sequence[float]         # six target RT60s (s); <= 0 keeps that band's FDN unscaled
    bin_duration_s: float
    transition_s: float = 1.0
    overlap_fraction: float = 0.25
    decay_profiles: Mapping[str, Any] | None = None


class LateReverbRenderer:
    """Renders batches of hybrid late tails: one FDN launch and one band/mix launch pair per batch."""

    def __init__(self, device: int | torch.device = 0) -> None:
        self.device = torch.device("cuda", device) if isinstance(device, int) else torch.device(device)
        self.fdn_ws = runtime.FdnWorkspace(self.device)
        self.tail_ws = runtime.LateTailWorkspace(self.device)
        self._designs: dict[tuple, FdnDesign] = {}

    def design(self, fs: int, seed: int, rt60: Sequence[float]) -> FdnDesign:
        key = (int(fs), int(seed), tuple(float(v or 0.0) for v in rt60))
        if key not in self._designs:
            if len(self._designs) > 1024:
                self._designs.clear()
            self._designs[key] = design(fs, seed, rt60)
        return self._designs[key]

    def render(self, jobs: Sequence[LateReverbJob], *, stream: torch.cuda.Stream | None = None,
               fdn_events: tuple[torch.cuda.Event, torch.cuda.Event] | None = None,
               designs: Sequence[FdnDesign] | None = None
               ) -> tuple[torch.Tensor, list[FdnDesign], list[Windows]]:
        """Enqueue every job on `stream`; returns the [J, 6, AC_LATE_STATS] float64 stats tensor, the designs
        and the windows.  Jobs whose tail starts outside the signal must not be passed.  `fdn_events`, if
        given, are recorded around the FDN launch (to time the network alone); `designs`, if given, are
        the jobs' FDN designs (from design_many), else they are made here."""
        J = len(jobs)
        stats = torch.zeros(max(J, 1), 6, _lib.AC_LATE_STATS, dtype=torch.float64, device=self.device)
        if J == 0:
            return stats[:0], [], []
        lengths = [int(j.traced.shape[1]) for j in jobs]
        raw = torch.empty(sum(lengths), dtype=torch.float64, device=self.device)
        cfg = runtime.synth_batch_config([j.fs for j in jobs])
        rate_index = {int(cfg.sample_rates[k]): k for k in range(cfg.num_rates)}
        fdn_jobs = (_lib.ACFdnJob * J)()
        tail_jobs = (_lib.ACLateTailJob * J)()
        given = list(designs) if designs is not None else None
        if given is not None and len(given) != J:
            raise ValueError("one design per job")
        designs, wins = [], []
        offset = 0
        for k, job in enumerate(jobs):
            N = lengths[k]
            for t, dtype in ((job.traced, torch.float64), (job.out, torch.float32), (job.component, torch.float32)):
                if t.dtype != dtype or not t.is_contiguous() or tuple(t.shape) != (6, N) or t.device != self.device:
                    raise ValueError(f"late reverb job {k}: expected contiguous [6, {N}] {dtype} on {self.device}")
            fs = max(1, int(job.fs))
            d = given[k] if given is not None else self.design(fs, job.seed, job.rt60)
            w = windows(N, fs, job.transition_s, job.overlap_fraction, job.decay_profiles)
            if min(w.start) >= N:
                raise ValueError(f"late reverb job {k}: the tail starts after the signal ends")
            designs.append(d)
            wins.append(w)
            f = fdn_jobs[k]
            ctypes.memmove(ctypes.addressof(f.absorptive), np.ascontiguousarray(d.absorptive).ctypes.data,
                           ctypes.sizeof(f.absorptive))
            ctypes.memmove(ctypes.addressof(f.tone), np.ascontiguousarray(d.tone).ctypes.data, ctypes.sizeof(f.tone))
            f.delays[:] = [int(v) for v in d.delays]
            f.allpass_delays[:] = list(d.allpass)
            f.num_samples = N
            f.preroll = d.preroll
            f.out = raw.data_ptr() + 8 * offset
            t = tail_jobs[k]
            t.traced = job.traced.data_ptr()
            t.fdn = raw.data_ptr() + 8 * offset
            t.out = job.out.data_ptr()
            t.fdn_component = job.component.data_ptr()
            t.stats = stats.data_ptr() + k * 6 * _lib.AC_LATE_STATS * 8
            t.rt60[:] = [float(v or 0.0) for v in job.rt60]
            t.start[:] = w.start
            t.end[:] = w.end
            t.anchor[:] = [w.anchor(b) for b in range(6)]
            t.changed_from = min(w.start)
            t.num_samples = N
            t.bin_samples = max(1, int(round(float(job.bin_duration_s) * fs)))
            t.rate_index = rate_index[fs]
            offset += N
        launch_stream = stream if stream is not None else torch.cuda.current_stream(self.device)
        if fdn_events is not None:
            fdn_events[0].record(launch_stream)
        runtime.fdn_impulse(fdn_jobs, J, self.fdn_ws, stream=stream)
        if fdn_events is not None:
            fdn_events[1].record(launch_stream)
        runtime.late_tail(tail_jobs, J, cfg, self.tail_ws, stream=stream)
        # keep the FDN scratch alive until the stream has used it
        raw.record_stream(launch_stream)
        return stats, designs, wins


@dataclass
class BatchTails:
    """Hybrid band IRs of a batch: every job's traced band IRs crossfaded into its FDN late tail."""

    out: torch.Tensor             # float32, the jobs' [6, N] hybrid band IRs back to back
    component: torch.Tensor       # float32, the FDN part of `out`, same layout
    irs: list[torch.Tensor]       # per job: its [6, N] view of `out`
    rt60: np.ndarray              # [J, 6] target RT60s estimated from the jobs' echograms
    stats: torch.Tensor           # [J, 6, AC_LATE_STATS] float64 (zeros for a job without a tail)
    host_seconds: float           # RT60 estimates, designs and job tables on the host


def batch_late_tails(renderer: LateReverbRenderer, band_irs: Sequence[torch.Tensor], echograms: Sequence[np.ndarray],
                     fs: Sequence[int], seeds: Sequence[int], bin_durations: Sequence[float],
                     speeds: Sequence[float], *, transition_s: float = 1.0, overlap_fraction: float = 0.25,
                     stream: torch.cuda.Stream | None = None) -> BatchTails:
    """Late tails of many RIRs, as the reference's renderer makes one (steam_rt.py:1014-1035, single room).

    `band_irs` are the jobs' float32 [6, N] device band IRs (contiguous and back to back in one buffer, in
    job order), `echograms` their [6, bins] host echograms.  Per job: the six target RT60s from the
    echogram (estimate_reverb_times), an FDN designed for them (design_many: the same numbers as the
    per-call design) and the hybrid tail; all FDN impulses go in one ac_fdn_impulse launch and all tails
    in one ac_late_tail, enqueued on `stream` after whatever produced `band_irs` there.  Each job's result
    equals render_parametric_fdn_late_reverb on its band IRs.  The coupled-space breakpoint model of
    multi-room renders is not applied.
    """
    t0 = time.perf_counter()
    J = len(band_irs)
    stream = stream if stream is not None else torch.cuda.current_stream(renderer.device)
    total = sum(t.numel() for t in band_irs)
    base = band_irs[0] if J else None
    if J and any(t.data_ptr() != base.data_ptr() + 4 * sum(u.numel() for u in band_irs[:k])
                 for k, t in enumerate(band_irs)):
        raise ValueError("band_irs must lie back to back in one buffer, in job order")
    flat = torch.as_strided(base, (total,), (1,)) if J else torch.empty(0, device=renderer.device)
    with torch.cuda.stream(stream):
        traced = flat.to(torch.float64)
        out = torch.empty_like(flat)
        component = torch.zeros_like(flat)
    rt60 = np.zeros((J, 6), dtype=np.float64)
    for k in range(J):
        rt60[k] = estimate_reverb_times(echograms[k], bin_durations[k], speeds[k])
    designs: list[Any] = [None] * J
    groups: dict[tuple[int, int], list[int]] = {}
    for k in range(J):
        groups.setdefault((max(1, int(fs[k])), int(seeds[k])), []).append(k)
    for (rate, seed), members in groups.items():
        for k, d in zip(members, design_many(rate, seed, rt60[members])):
            designs[k] = d
    views, jobs, chosen = [], [], []
    off = 0
    for k, ir in enumerate(band_irs):
        n = ir.numel()
        shape = tuple(ir.shape)
        views.append(out[off:off + n].view(shape))
        w = windows(shape[1], fs[k], transition_s, overlap_fraction)
        if min(w.start) >= shape[1]:
            with torch.cuda.stream(stream):
                views[-1].copy_(ir)   # no tail fits: the traced band IRs stand (steam_rt.py:2542-2552)
        else:
            jobs.append(LateReverbJob(traced[off:off + n].view(shape), views[-1],
                                      component[off:off + n].view(shape), int(fs[k]), int(seeds[k]), rt60[k],
                                      bin_durations[k], transition_s, overlap_fraction))
            chosen.append(k)
        off += n
    host_seconds = time.perf_counter() - t0
    stats = torch.zeros(J, 6, _lib.AC_LATE_STATS, dtype=torch.float64, device=renderer.device)
    if jobs:
        got, _, _ = renderer.render(jobs, stream=stream, designs=[designs[k] for k in chosen])
        with torch.cuda.stream(stream):
            stats[chosen] = got
    traced.record_stream(stream)
    return BatchTails(out, component, views, rt60, stats, host_seconds)


def metadata(stats: np.ndarray, d: FdnDesign, w: Windows, fs: int, rt60_bands: Mapping[str, float]) -> dict[str, Any]:
    """The reference's late-tail metadata dict (steam_rt.py:2618-2640) from one job's [6, AC_LATE_STATS] stats."""
    rt60 = [float(rt60_bands.get(b, 0.0) or 0.0) for b in bands.FREQUENCY_BANDS]
    rt60_used = {b: round(v, 4) for b, v in zip(bands.FREQUENCY_BANDS, rt60) if v > 0.0}
    transition_by_band: dict[str, dict[str, Any]] = {}
    scales, powers, fdn_by_band = {}, {}, {}
    for b, band in enumerate(bands.FREQUENCY_BANDS):
        transition_by_band[band] = {"start_s": round(float(w.start[b]) / fs, 6), "end_s": round(float(w.end[b]) / fs, 6),
                                    "model": w.model[b]}
        if rt60[b] <= 0.0:
            continue
        scales[band] = round(float(stats[b, _lib.AC_LATE_SCALE]), 8)
        powers[band] = round(float(stats[b, _lib.AC_LATE_POWER]), 14)
        transition_by_band[band]["anchor_s"] = round(float(w.anchor(b)) / fs, 6)
        fdn_by_band[band] = round(float(stats[b, _lib.AC_LATE_FDN_ENERGY]), 12)
    fdn_energy = float(np.sum(stats[:, _lib.AC_LATE_COMPONENT]))
    return {
        "applied": bool(rt60_used and fdn_energy > 1e-18),
        "changed": bool(np.any(stats[:, _lib.AC_LATE_CHANGED] > 0.0)),
        "added": bool(fdn_energy > 1e-18),
        "model": MODEL,
        "rt60_source": "steam_audio_reverb_estimator_from_traced_energy_field",
        "calibration": CALIBRATION,
        "transition_start_s": round(float(min(w.start)) / fs, 6),
        "transition_end_s": round(float(max(w.end)) / fs, 6),
        "configured_transition_end_s": round(w.transition_s, 6),
        "transition_by_band": transition_by_band,
        "overlap_fraction": w.overlap,
        "delay_line_count": int(d.delays.size),
        "delay_samples": [int(v) for v in d.delays],
        "allpass_delay_samples": [int(v) for v in d.allpass],
        "preroll_samples": d.preroll,
        "traced_tail_energy": round(float(np.sum(stats[:, _lib.AC_LATE_TRACED_TAIL])), 12),
        "fdn_tail_energy": round(fdn_energy, 12),
        "rendered_tail_energy": round(float(np.sum(stats[:, _lib.AC_LATE_RENDERED_TAIL])), 12),
        "anchor_power_by_band": powers,
        "scale_by_band": scales,
        "fdn_energy_by_band": fdn_by_band,
        "rt60_bands": rt60_used,
    }


_RENDERERS: dict[int, LateReverbRenderer] = {}


def renderer(device: int | None = None) -> LateReverbRenderer:
    if not torch.cuda.is_available():
        raise _lib.BackendError(_lib.AC_ERR_UNSUPPORTED, "the late-reverb renderer needs a CUDA device")
    dev = torch.cuda.current_device() if device is None else int(device)
    if dev not in _RENDERERS:
        _RENDERERS[dev] = LateReverbRenderer(dev)
    return _RENDERERS[dev]


def render_parametric_fdn_late_reverb(traced_band_irs: Any, field: Mapping[str, Any], rt60_bands: Mapping[str, float],
                                      config: Any, *, decay_profiles: Mapping[str, Any] | None = None,
                                      device: int | None = None) -> tuple[np.ndarray, np.ndarray, dict[str, Any]]:
    """Same arguments, results and errors as steam_rt.py:2500 ``_render_parametric_fdn_late_reverb``."""
    traced = np.asarray(traced_band_irs, dtype=np.float64)
    if traced.ndim != 2 or traced.shape[0] != 6:
        raise ValueError(f"expected 6 traced band IRs, got {traced.shape}")
    fs = max(1, int(config.fs))
    N = int(traced.shape[1])
    w = windows(N, fs, config.hybrid_transition_s, config.hybrid_overlap_fraction, decay_profiles)
    if not config.late_tail or min(w.start) >= N:
        return traced.astype(np.float32), np.zeros_like(traced, dtype=np.float32), {
            "applied": False,
            "added": False,
            "reason": "disabled" if not config.late_tail else "tail_start_outside_rir",
            "model": MODEL,
            "transition_start_s": round(w.start_s, 6),
            "transition_end_s": round(w.transition_s, 6),
            "overlap_fraction": w.overlap,
        }
    r = renderer(device)
    stream = torch.cuda.current_stream(r.device)
    traced_dev = torch.from_numpy(np.ascontiguousarray(traced)).pin_memory().to(r.device, non_blocking=True)
    out = torch.empty(6, N, dtype=torch.float32, device=r.device)
    comp = torch.empty(6, N, dtype=torch.float32, device=r.device)
    bin_dur = float(field.get("bin_duration_s", config.rt_bin_duration_s))
    rt60 = [float(rt60_bands.get(b, 0.0) or 0.0) for b in bands.FREQUENCY_BANDS]
    job = LateReverbJob(traced_dev, out, comp, fs, int(config.seed), rt60, bin_dur, float(config.hybrid_transition_s),
                        float(config.hybrid_overlap_fraction), decay_profiles)
    stats, designs, wins = r.render([job], stream=stream)
    host = [out.to("cpu", non_blocking=True), comp.to("cpu", non_blocking=True), stats.to("cpu", non_blocking=True)]
    stream.synchronize()
    out_np, comp_np, stats_np = (t.numpy() for t in host)
    return out_np, comp_np, metadata(stats_np[0], designs[0], wins[0], fs, rt60_bands)
