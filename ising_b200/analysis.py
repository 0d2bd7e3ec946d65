"""Time-series statistics for Monte Carlo observables (host-side, numpy).

tau_int uses Sokal's automatic windowing (window W = smallest t with t >= c*tau(t), c = 5);
binning_error uses the standard blocking estimate.  Effective samples: N / (2 tau_int).
"""
from __future__ import annotations

import numpy as np


def autocorrelation(x: np.ndarray) -> np.ndarray:
    x = np.asarray(x, dtype=np.float64)
    n = len(x)
    d = x - x.mean()
    f = np.fft.rfft(d, n=2 * n)
    acf = np.fft.irfft(f * np.conj(f))[:n] / n
    return acf / acf[0] if acf[0] > 0 else np.zeros(n)


def tau_int(x, c: float = 5.0) -> float:
    """Integrated autocorrelation time with Sokal's automatic window."""
    x = np.asarray(x, dtype=np.float64)
    if len(x) < 4 or np.var(x) == 0.0:
        return 0.5
    rho = autocorrelation(x)
    tau = 0.5
    for t in range(1, len(x)):
        tau += rho[t]
        if t >= c * tau:
            break
    return max(tau, 0.5)


def ess(x, c: float = 5.0) -> float:
    return len(x) / (2.0 * tau_int(x, c))


def binning_error(x, min_bins: int = 16) -> float:
    """Standard error of the mean from the plateau of blocked variances."""
    x = np.asarray(x, dtype=np.float64)
    n = len(x)
    best = x.std(ddof=1) / np.sqrt(n) if n > 1 else 0.0
    b = 1
    while n // b >= min_bins:
        m = n // b
        blocks = x[: m * b].reshape(m, b).mean(axis=1)
        err = blocks.std(ddof=1) / np.sqrt(m)
        best = max(best, err)
        b *= 2
    return best


def specific_heat(e, beta: float, n_sites: int):
    """C_v = beta^2 N (<e^2> - <e>^2) with e the energy per site."""
    e = np.asarray(e) / n_sites
    return beta * beta * n_sites * (np.mean(e * e) - np.mean(e) ** 2)


def susceptibility(m_abs, beta: float, n_sites: int):
    """chi = beta N (<m^2> - <|m|>^2) with m the magnetisation per site."""
    m = np.asarray(m_abs)
    return beta * n_sites * (np.mean(m * m) - np.mean(m) ** 2)
