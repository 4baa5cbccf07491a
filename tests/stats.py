"""Binned mean / error of a Markov-chain time series (test helper)."""
import numpy as np


def binned_mean_err(x, nbins: int = 20):
    """Mean and its standard error from `nbins` equal bins (bins longer than the
    integrated autocorrelation time make the bin means independent)."""
    x = np.asarray(x, float)
    n = (x.size // nbins) * nbins
    b = x[:n].reshape(nbins, -1).mean(axis=1)
    return b.mean(), b.std(ddof=1) / np.sqrt(nbins)


def tau_int(x, wmax: int = 200) -> float:
    """Integrated autocorrelation time with a self-consistent window (Madras-Sokal, c = 6)."""
    x = np.asarray(x, float) - np.mean(x)
    n = x.size
    var = np.dot(x, x) / n
    if var == 0:
        return 0.5
    tau = 0.5
    for w in range(1, min(wmax, n // 2)):
        rho = np.dot(x[:-w], x[w:]) / (n - w) / var
        tau += rho
        if w >= 6 * tau:
            break
    return max(tau, 0.5)


def z_score(a, b, nbins: int = 20) -> float:
    ma, ea = binned_mean_err(a, nbins)
    mb, eb = binned_mean_err(b, nbins)
    return abs(ma - mb) / np.hypot(ea, eb)
