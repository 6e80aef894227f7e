"""Validation helpers on the host (src/validate.jl, src/analytical.jl).

compare_moments(x, y)      the reference's convention for two sample sets: relative error
                           |a - b| / max(|a|, |b|, 1e-10) of the means and of the
                           (unbiased) variances, and pass = both < rtol (validate.jl:70-77).
moment_errors(X, Y)        the same per column (gene) of two cells x genes matrices, plus
                           the Fano factor var / mean under the same convention.
ks_statistic(x, y)         two-sample Kolmogorov-Smirnov statistic with the tie order of the
                           reference's merge walk (validate.jl:14-41); ks_critical_value
                           its asymptotic critical value (validate.jl:51-61).
telegraph_pmf / _mean / _variance / _fano
                           the telegraph model's steady-state mRNA distribution and moments
                           (analytical.jl:35-119), for comparing histograms of the device
                           results (DeviceRun.histogram).
The device-side reductions are DeviceRun.moments / histogram and api.ks_statistic_device.
"""
from __future__ import annotations

from typing import Dict, Optional

import numpy as np


def _relerr(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.abs(a - b) / np.maximum(np.maximum(np.abs(a), np.abs(b)), 1e-10)


def compare_moments(x, y, rtol: float = 0.05):
    """(mean_relerr, var_relerr, pass) of two sample vectors (validate.jl:70-77)."""
    x = np.asarray(x, dtype=np.float64).reshape(-1)
    y = np.asarray(y, dtype=np.float64).reshape(-1)
    mean_err = float(_relerr(x.mean(), y.mean()))
    var_err = float(_relerr(x.var(ddof=1), y.var(ddof=1)))
    return mean_err, var_err, bool(mean_err < rtol and var_err < rtol)


def column_moments(X) -> Dict[str, np.ndarray]:
    """Per-column mean, unbiased variance and Fano factor (var / mean; 0 where mean is 0)."""
    Xd = np.asarray(X, dtype=np.float64)
    mean = Xd.mean(0)
    var = Xd.var(0, ddof=1) if Xd.shape[0] > 1 else np.zeros(Xd.shape[1])
    fano = np.divide(var, mean, out=np.zeros_like(var), where=mean != 0)
    return {"mean": mean, "var": var, "fano": fano}


def moment_errors(X, Y) -> Dict[str, np.ndarray]:
    """Per-column relative errors of mean, variance and Fano factor between two cells x genes
    matrices, each |a - b| / max(|a|, |b|, 1e-10) as compare_moments does."""
    a, b = column_moments(X), column_moments(Y)
    return {k: _relerr(a[k], b[k]) for k in ("mean", "var", "fano")}


def max_moment_error(X, Y) -> float:
    """Largest per-column mean / variance / Fano error between two matrices."""
    e = moment_errors(X, Y)
    return float(max(e[k].max() for k in e))


def ks_statistic(x, y) -> float:
    """Largest |ecdf_x - ecdf_y| over the steps of the merge walk of validate.jl:14-41, which
    takes the x sample first on ties: after the i-th x it has taken the y's below x_i, after
    the j-th y the x's up to y_j."""
    sx = np.sort(np.asarray(x, dtype=np.float64).reshape(-1))
    sy = np.sort(np.asarray(y, dtype=np.float64).reshape(-1))
    nx, ny = len(sx), len(sy)
    ex = np.arange(1, nx + 1) / nx - np.searchsorted(sy, sx, side="left") / ny
    ey = np.searchsorted(sx, sy, side="right") / nx - np.arange(1, ny + 1) / ny
    return float(max(np.abs(ex).max(initial=0.0), np.abs(ey).max(initial=0.0)))


def ks_critical_value(n1: int, n2: int, alpha: float = 0.05) -> float:
    """Asymptotic two-sample critical value c(alpha) sqrt((n1 + n2) / (n1 n2)) (validate.jl:51-61)."""
    c = 1.63 if alpha <= 0.01 else 1.36 if alpha <= 0.05 else 1.22
    return c * float(np.sqrt((n1 + n2) / (n1 * n2)))


def telegraph_logpmf(n: int, a: float, b: float, c: float) -> float:
    """log P(n) of the telegraph model with dimensionless rates a (on), b (off), c
    (transcription), all over the mRNA decay rate (analytical.jl:35-52)."""
    from scipy.special import gammaln, hyp1f1
    lp = (-c + n * np.log(c) - gammaln(n + 1) + gammaln(a + n) - gammaln(a) - gammaln(a + b + n)
          + gammaln(a + b))
    return float(lp + np.log(hyp1f1(b, a + b + n, c)))


def telegraph_pmf(n: int, a: float, b: float, c: float) -> float:
    return float(np.exp(telegraph_logpmf(n, a, b, c)))


def telegraph_mean(a: float, b: float, c: float) -> float:
    return a * c / (a + b)


def telegraph_variance(a: float, b: float, c: float) -> float:
    mu = telegraph_mean(a, b, c)
    return mu + a * b * c * c / ((a + b) ** 2 * (a + b + 1))


def telegraph_fano(a: float, b: float, c: float) -> float:
    return 1.0 + b * c / ((a + b) * (a + b + 1))


def telegraph_distribution(a: float, b: float, c: float, nmax: Optional[int] = None,
                           tol: float = 1e-12) -> np.ndarray:
    """P(0), ..., P(nmax) of the telegraph model (analytical.jl:71-95): nmax defaults to
    max(ceil(mean + 10 sd), 100); the vector is cut after the last n with P(n) > tol x max P
    and normalised."""
    if nmax is None:
        mu = telegraph_mean(a, b, c)
        sd = float(np.sqrt(telegraph_variance(a, b, c)))
        nmax = max(int(np.ceil(mu + 10.0 * sd)), 100)
    logp = np.array([telegraph_logpmf(n, a, b, c) for n in range(nmax + 1)])
    top = logp.max()
    keep = np.nonzero(logp > np.log(tol) + top)[0]
    if len(keep):
        logp = logp[: keep[-1] + 1]
    p = np.exp(logp - top)
    return p / p.sum()


def empirical_pmf(samples, nmax: int) -> np.ndarray:
    """Fraction of the samples at each n = 0..nmax after rounding max(x, 0) half to even;
    samples above nmax count in the total only (experiments/validate_telegraph.jl:80-89)."""
    s = np.rint(np.maximum(np.asarray(samples, dtype=np.float64).reshape(-1), 0.0)).astype(np.int64)
    counts = np.bincount(s[s <= nmax], minlength=nmax + 1)[: nmax + 1]
    return counts / len(s)


def l1_distance(p_empirical, p_exact) -> float:
    """Sum of |p_empirical - p_exact| over the common support plus the tail mass of the longer
    vector (experiments/validate_telegraph.jl:91-106)."""
    pe, px = np.asarray(p_empirical, np.float64), np.asarray(p_exact, np.float64)
    n = min(len(pe), len(px))
    return float(np.abs(pe[:n] - px[:n]).sum() + np.abs(pe[n:]).sum() + np.abs(px[n:]).sum())


def ks_vs_exact(samples, p_exact) -> float:
    """Largest |ecdf - F| at each sorted sample (rounded as in empirical_pmf), taken after
    and just before the sample's step, F the exact CDF at min(sample, len - 1)
    (experiments/validate_telegraph.jl:108-125).  On integer samples the term before a step
    compares F(n) with the ECDF below n, so the statistic is at least about max_n P(n)
    whatever the samples (the first sample alone gives P(0) when it is 0): l1_distance is
    the measure that shrinks with agreement."""
    cdf = np.cumsum(np.asarray(p_exact, np.float64))
    s = np.sort(np.rint(np.maximum(np.asarray(samples, dtype=np.float64).reshape(-1), 0.0)).astype(np.int64))
    n = len(s)
    F = cdf[np.minimum(s, len(cdf) - 1)]
    i = np.arange(1, n + 1)
    return float(max(np.abs(i / n - F).max(initial=0.0), np.abs((i - 1) / n - F).max(initial=0.0)))


def pmf_comparison_from_histogram(hist, p_exact) -> dict:
    """l1_distance(empirical_pmf) and ks_vs_exact from counts of the rounded samples at
    0..L-1 and of all samples >= L in hist[L] (L = len(p_exact); nbins = L + 1), the same
    values as from the samples themselves: samples at or above L - 1 all meet F[L - 1], so
    the walk over sorted samples needs only the cumulative counts."""
    h = np.asarray(hist, dtype=np.float64)
    L = len(p_exact)
    if len(h) != L + 1:
        raise ValueError("the histogram needs len(p_exact) + 1 bins")
    n = h.sum()
    cdf = np.cumsum(np.asarray(p_exact, np.float64))
    C = np.cumsum(h)
    prev = np.concatenate([[0.0], C[:-1]])
    F = cdf[np.minimum(np.arange(L + 1), L - 1)]
    occ = h > 0
    ks = float(max(np.abs(C[occ] / n - F[occ]).max(initial=0.0), np.abs(prev[occ] / n - F[occ]).max(initial=0.0)))
    return {"l1": l1_distance(h[:L] / n, p_exact), "ks": ks, "n": int(n)}
