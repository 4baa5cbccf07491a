"""Binned mean / error of Markov-chain time series (test helper)."""
import math

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


def bin_length(taus, factor: float = 10.0) -> int:
    """Bin length of at least `factor` times the largest integrated autocorrelation time."""
    return int(math.ceil(factor * max(taus)))


def chain_bins(x, length: int) -> np.ndarray:
    """Means of consecutive bins of `length` samples (a trailing partial bin is dropped)."""
    x = np.asarray(x, float)
    n = (x.size // length) * length
    return x[:n].reshape(-1, length).mean(axis=1)


def pooled_mean_err(bins_per_chain):
    """Mean and standard error from the bin means of several independent chains, pooled:
    with bins much longer than the autocorrelation time every bin mean is an independent
    sample of the same distribution."""
    b = np.concatenate([np.asarray(c, float) for c in bins_per_chain])
    return float(b.mean()), float(b.std(ddof=1) / np.sqrt(b.size)), int(b.size)


def chains_summary(series, factor: float = 10.0, length: int = 0) -> dict:
    """tau_int of each chain, the common bin length (>= factor * the largest tau_int, or
    `length` if that is longer), the bin means of each chain, and the pooled mean and error."""
    taus = [tau_int(x) for x in series]
    length = max(length, bin_length(taus, factor))
    bins = [chain_bins(x, length) for x in series]
    mean, err, nb = pooled_mean_err(bins)
    return {"tau_int": taus, "bin_length": length, "bins": bins, "mean": mean, "err": err, "n_bins": nb}


def between_chain_err(bins_per_chain) -> float:
    """Standard error of the grand mean from the scatter of the chain means (every chain has
    bins of the same length).  Unlike the pooled-bin error it also sees modes slower than one
    chain's length, such as metastable states a chain starts in and keeps."""
    m = np.array([np.mean(c) for c in bins_per_chain])
    return float(m.std(ddof=1) / np.sqrt(m.size))


def chains_estimate(bins_per_chain):
    """Mean and the larger of the pooled-bin and between-chain errors."""
    mean, err, nb = pooled_mean_err(bins_per_chain)
    return mean, max(err, between_chain_err(bins_per_chain)), nb
