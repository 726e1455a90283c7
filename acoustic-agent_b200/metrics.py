"""Room-acoustic decay metrics on six-band echograms.

Used to compare a trace with the float64 oracle when ray-by-ray identity is
not expected (float32 arithmetic, or a different random stream):

* EDC: Schroeder backward integral of bin energies, in dB re the total
  (the reference's decay fits start from the same integral,
  steam_rt.py:2727-2792 ``_schroeder_fit_rt60``);
* T30: decay time from a least-squares line over -5 .. -35 dB, times 2;
* EDT: same over 0 .. -10 dB, times 6;
* C50: early-to-late energy ratio at 50 ms after the first arrival bin;
* the reference's own traced RT60 fit (``schroeder_rt60``).
"""
from __future__ import annotations

import numpy as np


def edc_db(echogram: np.ndarray) -> np.ndarray:
    """[bands, bins] energy decay curve in dB (0 dB at t=0; -inf after the last energy)."""
    e = np.clip(np.asarray(echogram, dtype=np.float64), 0.0, None)
    tail = np.cumsum(e[:, ::-1], axis=1)[:, ::-1]
    total = tail[:, :1]
    with np.errstate(divide="ignore", invalid="ignore"):
        return 10.0 * np.log10(np.where(total > 0, tail / np.where(total > 0, total, 1.0), 0.0))


def edc_error_db(a: np.ndarray, b: np.ndarray, range_db: float = 30.0) -> np.ndarray:
    """Per-band max |EDC_a - EDC_b| over the bins where EDC_b >= -range_db."""
    ea, eb = edc_db(a), edc_db(b)
    out = np.zeros(ea.shape[0])
    for band in range(ea.shape[0]):
        mask = eb[band] >= -range_db
        if np.any(mask):
            out[band] = float(np.max(np.abs(ea[band, mask] - eb[band, mask])))
    return out


def schroeder_rt60(energy: np.ndarray, bin_dur: float, *, min_total_energy: float = 1e-12) -> float:
    """The reference's traced RT60 of one band (steam_rt.py:3052-3067): least-squares line through the
    Schroeder curve between -5 and -25 dB, bins timed at their start, extrapolated to -60 dB."""
    e = np.asarray(energy, dtype=np.float64)
    total = float(np.sum(e))
    if total < float(min_total_energy):
        return 0.0
    edc = np.cumsum(e[::-1])[::-1]
    db = 10.0 * np.log10(np.clip(edc / total, 1e-12, None))
    x = float(bin_dur) * np.arange(edc.size, dtype=np.float64)
    fit = (db <= -5.0) & (db >= -25.0)
    if int(np.count_nonzero(fit)) < 2:
        return 0.0
    xs, ys = x[fit], db[fit]
    n = xs.size
    denom = n * np.sum(xs * xs) - np.sum(xs) ** 2
    numer = n * np.sum(xs * ys) - np.sum(xs) * np.sum(ys)
    slope = numer / denom if abs(denom) > 1e-12 else 0.0
    return float(max(0.0, -60.0 / slope)) if slope < -1e-9 else 0.0


def _decay_time(edc: np.ndarray, bin_dur: float, hi_db: float, lo_db: float, factor: float) -> float:
    t = (np.arange(edc.shape[0]) + 0.5) * bin_dur
    mask = (edc <= hi_db) & (edc >= lo_db) & np.isfinite(edc)
    if np.count_nonzero(mask) < 2:
        return 0.0
    slope = np.polyfit(t[mask], edc[mask], 1)[0]
    return float(factor * (-10.0 / slope)) if slope < 0 else 0.0


def t30(echogram: np.ndarray, bin_dur: float) -> np.ndarray:
    e = edc_db(echogram)
    return np.asarray([_decay_time(e[b], bin_dur, -5.0, -35.0, 6.0) for b in range(e.shape[0])])


def edt(echogram: np.ndarray, bin_dur: float) -> np.ndarray:
    e = edc_db(echogram)
    return np.asarray([_decay_time(e[b], bin_dur, 0.0, -10.0, 6.0) for b in range(e.shape[0])])


def c50(echogram: np.ndarray, bin_dur: float) -> np.ndarray:
    e = np.clip(np.asarray(echogram, dtype=np.float64), 0.0, None)
    k = max(1, int(round(0.05 / bin_dur)))
    early = np.sum(e[:, :k], axis=1)
    late = np.sum(e[:, k:], axis=1)
    with np.errstate(divide="ignore"):
        return 10.0 * np.log10(np.where(late > 0, early / np.where(late > 0, late, 1.0), np.inf))


def parity(ours: np.ndarray, ref: np.ndarray, bin_dur: float) -> dict:
    """Worst band of each decay statistic of `ours` against `ref` ([bands, bins] echograms):

    * ``edc_err_db_max``: max |EDC difference| over the first 30 dB of the reference's decay;
    * ``t30_rel``, ``edt_rel``: max relative difference of T30 and EDT;
    * ``c50_rel``: max relative difference of the early-to-late energy ratio (the linear C50),
      ``c50_db``: the same difference in dB;
    * ``band_energy_rel``: max relative difference of a band's total energy.

    Bands whose reference energy is zero are skipped.
    """
    a = np.asarray(ours, dtype=np.float64)
    b = np.asarray(ref, dtype=np.float64)
    live = np.sum(b, axis=1) > 0.0
    if not np.any(live):
        return {"edc_err_db_max": 0.0, "t30_rel": 0.0, "edt_rel": 0.0, "c50_rel": 0.0, "c50_db": 0.0,
                "band_energy_rel": 0.0}
    a, b = a[live], b[live]

    def rel(x, y):
        x, y = np.asarray(x, dtype=np.float64), np.asarray(y, dtype=np.float64)
        with np.errstate(divide="ignore", invalid="ignore"):
            r = np.where(x == y, 0.0, np.where((y != 0.0) & np.isfinite(y), np.abs(x - y) / np.abs(y), np.inf))
        return float(np.max(r))

    def c50_db_diff(x, y):
        # equal values (a band with no late energy has +inf in both) differ by 0
        with np.errstate(invalid="ignore"):
            d = np.where(x == y, 0.0, np.abs(x - y))
        return float(np.max(d))

    ca, cb = c50(a, bin_dur), c50(b, bin_dur)
    return {
        "edc_err_db_max": float(np.max(edc_error_db(a, b))),
        "t30_rel": rel(t30(a, bin_dur), t30(b, bin_dur)),
        "edt_rel": rel(edt(a, bin_dur), edt(b, bin_dur)),
        "c50_rel": rel(10.0 ** (ca / 10.0), 10.0 ** (cb / 10.0)),
        "c50_db": c50_db_diff(ca, cb),
        "band_energy_rel": rel(np.sum(a, axis=1), np.sum(b, axis=1)),
    }
