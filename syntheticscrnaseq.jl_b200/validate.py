"""Moment comparisons of simulated count matrices (src/validate.jl:70-77).

compare_moments(x, y)      the reference's convention for two sample sets: relative error
                           |a - b| / max(|a|, |b|, 1e-10) of the means and of the
                           (unbiased) variances, and pass = both < rtol.
moment_errors(X, Y)        the same per column (gene) of two cells x genes matrices, plus
                           the Fano factor var / mean under the same convention.
"""
from __future__ import annotations

from typing import Dict

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
