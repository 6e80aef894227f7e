"""Moment error of the GPU path against the FP64 oracle on the same Philox increments, at
the benchmark workloads' own sizes: the accuracy the throughput metric is quoted at.

Convention (src/validate.jl:70-77, compare_moments): per gene, |a - b| / max(|a|, |b|, 1e-10)
of the mean and of the unbiased variance across cells, and the same for the Fano factor
var / mean, for mRNA and protein.  Bars:
  register path (FP32 state): every gene's mean, variance and Fano within 1 %
    - plain CLE, G=5 mixed regulation, 5,000 cells, dt=0.01, T=50 (5,000 steps)
    - telegraph CLE, G=10 bursty genes, 20,000 cells, dt=0.01, T=50 (5,000 steps)
  tensor-core path, dense G=2000 (10 % of A nonzero, 40 + 40 cooperative / redundant edges),
  dt=0.005, on 256 cells x 400 steps (the oracle's dense contraction costs ~1 ms per
  cell-step): every gene's mean, variance and Fano within 1 % with BF16 contraction inputs
  (measured on a B200: largest error 9e-4) and with FP16 inputs (1.4e-4).
Measured for the register path: 1.8e-7 (plain) and 2.4e-7 (telegraph).
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_FP32 = 0.01
TOL_BF16 = 0.01
TOL_F16 = 0.01
THREADS = os.cpu_count() or 1


def _both(orc_out):
    """Oracle [G, N] M and P as a cells x 2G matrix (the GPU readout 'both')."""
    return np.hstack([orc_out["M"].T, orc_out["P"].T])


def _check(pkg, got, want, tol, label):
    errs = pkg.moment_errors(got, want)
    worst = {k: float(v.max()) for k, v in errs.items()}
    assert max(worst.values()) <= tol, (label, worst)
    return worst


def test_plain_workload_moments(pkg, orc):
    wl = pkg.config0()
    got = pkg.simulate(wl.net, pkg.CLE(wl.dt), wl.kin, cell_num=wl.cell_num, T=wl.T, readout="both", seed=10)
    want = orc.simulate(wl.net, wl.kin, dt=wl.dt, T=wl.T, cell_num=wl.cell_num, seed=10, nthreads=THREADS)
    _check(pkg, got, _both(want), TOL_FP32, "plain G=5")


def test_telegraph_workload_moments(pkg, orc):
    wl = pkg.config1()
    got = pkg.simulate(wl.net, pkg.CLE(wl.dt), wl.kin, cell_num=wl.cell_num, T=wl.T, readout="both", seed=11)
    want = orc.simulate(wl.net, wl.kin, dt=wl.dt, T=wl.T, cell_num=wl.cell_num, seed=11, nthreads=THREADS)
    _check(pkg, got, _both(want), TOL_FP32, "telegraph G=10")


@pytest.mark.parametrize("precision,tol", [("fp32", TOL_BF16), ("fp32_f16", TOL_F16)])
def test_dense_workload_moments(pkg, orc, precision, tol):
    wl = pkg.config2()
    N, steps = 256, 400
    got = pkg.simulate(wl.net, pkg.CLE(wl.dt), wl.kin, cell_num=N, n_steps=steps, readout="both", seed=12,
                       path="tensor", precision=precision)
    want = orc.simulate(wl.net, wl.kin, dt=wl.dt, cell_num=N, n_steps=steps, seed=12, nthreads=THREADS)
    _check(pkg, got, _both(want), tol, f"dense G=2000 {precision}")
