"""Host-side constants of the echogram -> band-IR synthesis.

* crossover low-pass sections: acoustic_agent/steam_rt.py:4123-4127 (band
  edges) and :4154-4170 (eight-pole low-pass as four biquads, Q from the
  Butterworth pole angles).  Computed with Python floats exactly as the
  reference does, so the GPU filters use bit-identical coefficients.
* air absorption per band: acoustic_agent/acoustics.py:12-22.
* per-bin air gains: steam_rt.py:2190-2193 ``_air_absorption_amplitude``.
"""
from __future__ import annotations

import math

import numpy as np

FREQUENCY_BANDS = ("125", "250", "500", "1000", "2000", "4000")
AIR_ABSORPTION_NP_PER_M = (0.0, 0.00011513, 0.00034539, 0.00057565, 0.0011513, 0.0034539)
INNER_CROSSOVERS = (176.78, 353.55, 707.11, 1414.2, 2828.4)


def band_edges(fs: int) -> list[tuple[float, float]]:
    nyquist = fs * 0.5
    bounds = [0.0, *INNER_CROSSOVERS, nyquist]
    return [(bounds[i], bounds[i + 1]) for i in range(6)]


def lowpass_sections(cutoff_hz: float, fs: int) -> list[tuple[float, float, float, float, float]]:
    """Four biquad sections (b0, b1, b2, a1, a2) of the eight-pole low-pass at cutoff_hz."""
    sampling_rate = max(1, int(fs))
    nyquist = 0.5 * sampling_rate
    cutoff = float(np.clip(float(cutoff_hz), 1e-3, nyquist * 0.999))
    order = 8
    out = []
    for section in range(order // 2):
        section_q = 1.0 / (2.0 * math.cos((2.0 * section + 1.0) * math.pi / (2.0 * order)))
        w0 = 2.0 * math.pi * cutoff / sampling_rate
        cw0, sw0 = math.cos(w0), math.sin(w0)
        alpha = sw0 / (2.0 * section_q)
        a0 = 1.0 + alpha
        b0 = ((1.0 - cw0) / 2.0) / a0
        b1 = (1.0 - cw0) / a0
        b2 = b0
        a1 = (-2.0 * cw0) / a0
        a2 = (1.0 - alpha) / a0
        out.append((b0, b1, b2, a1, a2))
    return out


def crossover_table(fs: int) -> np.ndarray:
    """[5 cutoffs, 4 sections, 5 coefficients] float64 for the five inner crossovers."""
    crossovers = [edge[1] for edge in band_edges(fs)[:-1]]
    return np.asarray([lowpass_sections(c, fs) for c in crossovers], dtype=np.float64)


def samples_per_bin(bin_duration_s: float, fs: int) -> int:
    return max(1, int(math.ceil(float(bin_duration_s) * int(fs))))


def air_gain_table(num_bins: int, spb: int, fs: int, direct_delay_s: float, c: float) -> np.ndarray:
    """[6, bins] amplitude gains exp(-alpha * c * t) at each bin centre, with math.exp like the reference."""
    direct = max(0.0, float(direct_delay_s))
    out = np.empty((6, num_bins), dtype=np.float64)
    speed = max(0.0, float(c))
    for band, coeff in enumerate(AIR_ABSORPTION_NP_PER_M):
        alpha = max(0.0, float(coeff))
        for b in range(num_bins):
            path_time_s = direct + (b + 0.5) * spb / int(fs)
            out[band, b] = math.exp(-alpha * (max(0.0, path_time_s) * speed))
    return out
