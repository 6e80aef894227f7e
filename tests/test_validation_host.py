"""Host-side validation helpers against literal restatements of the reference's algorithms:
the two-sample KS merge walk (src/validate.jl:14-41), the telegraph distribution
(src/analytical.jl:35-119) and the 10x Matrix Market reader (experiments/compare_real_scrnaseq.jl:69-93)."""
import numpy as np
import pytest


def _ks_walk(x, y):
    """validate.jl:14-41 step by step."""
    sx, sy = sorted(x), sorted(y)
    nx, ny = len(sx), len(sy)
    ix = iy = 0
    d = ex = ey = 0.0
    while ix < nx or iy < ny:
        if ix >= nx:
            ey += 1.0 / ny
            iy += 1
        elif iy >= ny:
            ex += 1.0 / nx
            ix += 1
        elif sx[ix] <= sy[iy]:
            ex += 1.0 / nx
            ix += 1
        else:
            ey += 1.0 / ny
            iy += 1
        d = max(d, abs(ex - ey))
    return d


@pytest.mark.parametrize("seed", range(6))
def test_ks_statistic_matches_the_merge_walk(pkg, seed):
    rng = np.random.default_rng(seed)
    nx, ny = int(rng.integers(1, 300)), int(rng.integers(1, 300))
    if seed % 2:  # integer data: many ties
        x, y = rng.poisson(3.0, nx).astype(float), rng.poisson(3.5, ny).astype(float)
    else:
        x, y = rng.normal(0, 1, nx), rng.normal(0.2, 1.1, ny)
    assert abs(pkg.ks_statistic(x, y) - _ks_walk(list(x), list(y))) < 1e-12


def test_ks_ties_and_critical_value(pkg):
    assert pkg.ks_statistic([1, 1], [1, 1]) == 1.0  # the walk takes both x before the equal y's
    assert abs(pkg.ks_critical_value(100, 100) - 1.36 * np.sqrt(0.02)) < 1e-15
    assert pkg.ks_critical_value(10, 10, alpha=0.01) > pkg.ks_critical_value(10, 10, alpha=0.1)


@pytest.mark.parametrize("a,b,c", [(0.5, 2.0, 20.0), (1.0, 1.0, 10.0), (0.3, 3.0, 40.0)])
def test_telegraph_distribution(pkg, a, b, c):
    n = np.arange(0, 400)
    p = np.array([pkg.telegraph_pmf(int(k), a, b, c) for k in n])
    assert abs(p.sum() - 1.0) < 1e-9
    mean = (n * p).sum()
    var = (n * n * p).sum() - mean * mean
    assert abs(mean - pkg.telegraph_mean(a, b, c)) < 1e-8 * c
    assert abs(var - pkg.telegraph_variance(a, b, c)) < 1e-7 * c * c
    assert abs(var / mean - pkg.telegraph_fano(a, b, c)) < 1e-8 * c


def test_read_10x_mtx(pkg, tmp_path):
    path = tmp_path / "matrix.mtx"
    path.write_text("%%MatrixMarket matrix coordinate integer general\n% comment\n3 4 4\n1 1 5\n3 1 2\n2 3 7\n3 4 1\n")
    X = pkg.read_10x_mtx(str(path))
    want = np.zeros((3, 4), dtype=np.int64)
    want[0, 0], want[2, 0], want[1, 2], want[2, 3] = 5, 2, 7, 1
    assert np.array_equal(X, want)
    bad = tmp_path / "bad.mtx"
    bad.write_text("%%MatrixMarket matrix coordinate integer general\n2 2 3\n1 1 1\n")
    with pytest.raises(ValueError):
        pkg.read_10x_mtx(str(bad))


def _ks_vs_exact_loop(samples, p_exact):
    """experiments/validate_telegraph.jl:108-125 as a plain loop (1-based CDF index)."""
    cdf = np.cumsum(p_exact)
    s = sorted(int(np.rint(max(x, 0.0))) for x in samples)
    n, d = len(s), 0.0
    for i, v in enumerate(s, start=1):
        idx = min(v + 1, len(cdf))
        F = cdf[idx - 1] if idx > 0 else 0.0
        d = max(d, abs(i / n - F), abs((i - 1) / n - F))
    return d


def _l1_loop(pe, px):
    """experiments/validate_telegraph.jl:91-106 as a plain loop."""
    m = min(len(pe), len(px))
    return sum(abs(pe[i] - px[i]) for i in range(m)) + sum(abs(x) for x in pe[m:]) + sum(abs(x) for x in px[m:])


@pytest.mark.parametrize("a,b,c", [(50.0, 50.0, 40.0), (2.0, 5.0, 70.0), (0.2, 0.3, 50.0)])
def test_telegraph_distribution_vector(pkg, a, b, c):
    """analytical.jl:71-95: normalised, truncated where P(n) < 1e-12 max P, equal to the PMF."""
    p = pkg.telegraph_distribution(a, b, c)
    assert abs(p.sum() - 1.0) < 1e-12 and p[-1] > 1e-12 * p.max() * 0.999
    q = np.array([pkg.telegraph_pmf(n, a, b, c) for n in range(len(p))])
    assert np.allclose(p, q / q.sum(), rtol=1e-10, atol=1e-300)
    assert len(pkg.telegraph_distribution(a, b, c, nmax=30)) <= 31


def test_pmf_comparisons_match_the_reference_loops(pkg):
    rng = np.random.default_rng(5)
    p_exact = pkg.telegraph_distribution(2.0, 5.0, 70.0)
    L = len(p_exact)
    # samples as a simulator reads them out: non-negative reals, some negative, some beyond L,
    # some exactly at half-integers (rounded half to even)
    x = np.concatenate([rng.negative_binomial(3, 0.13, 3000).astype(np.float64) + rng.uniform(-0.5, 0.5, 3000),
                        [-2.0, 0.5, 1.5, 2.5, L - 1.0, L + 0.0, L + 7.3, 3 * L]])
    pe = pkg.empirical_pmf(x, L - 1)
    assert abs(pkg.l1_distance(pe, p_exact) - _l1_loop(list(pe), list(p_exact))) < 1e-12
    assert abs(pkg.l1_distance(pe[:10], p_exact) - _l1_loop(list(pe[:10]), list(p_exact))) < 1e-12
    ks = pkg.ks_vs_exact(x, p_exact)
    assert abs(ks - _ks_vs_exact_loop(x, p_exact)) < 1e-12
    # the device path: counts of rint(x) clamped to [0, L] (the histogram kernel's rule)
    hist = np.bincount(np.clip(np.rint(x), 0, L).astype(np.int64), minlength=L + 1)
    r = pkg.pmf_comparison_from_histogram(hist, p_exact)
    assert r["n"] == len(x)
    assert abs(r["ks"] - ks) < 1e-12 and abs(r["l1"] - pkg.l1_distance(pe, p_exact)) < 1e-12
