"""Pins the CPU oracle before it is trusted as the checker.

The reference has no golden vectors; its CLE tests are closed-form moment checks
with tolerance bands.  Each test here re-runs one of them on the oracle with the
same parameters and bands (file:line of the reference test in each docstring),
plus the published Philox4x32-10 known-answer vectors.
"""
import math

import numpy as np
import pytest


def _relerr(obs, exact):
    return abs(obs - exact) / max(abs(exact), 1e-10)


PHILOX_KAT = [
    # (counter, key, expected) -- Salmon et al. known-answer vectors for Philox4x32-10
    ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
    ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
    ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
     [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
]


@pytest.mark.parametrize("ctr,key,want", PHILOX_KAT)
def test_philox_known_answers(orc, ctr, key, want):
    assert orc.philox(ctr, key).tolist() == want


def test_normals_are_standard(orc):
    z = np.array([orc.step_normals(3, 0, c, 1, g) for c in range(4000) for g in range(2)]).ravel()
    assert abs(z.mean()) < 0.03
    assert abs(z.var() - 1.0) < 0.04


def _one_gene(pkg, beta, **kin):
    net = pkg.GeneNetwork(1, [beta], np.zeros((1, 1)))
    return net, pkg.KineticParams(**kin)


def test_two_stage_moments(pkg, orc):
    """test/test_analytical_moments.jl:110-121 (CLE, dt=0.1, N=10000, T=500)."""
    beta, mu_m, mu_p, k_t = 2.0, 0.1, 0.2, 1.0
    net, kin = _one_gene(pkg, beta, k_t=k_t, K_d=50.0, n=2.0, mu_m=mu_m, mu_p=mu_p)
    r = orc.simulate(net, kin, dt=0.1, T=500.0, cell_num=10000, seed=42)
    m, p = r["M"][0], r["P"][0]
    assert _relerr(m.mean(), beta / mu_m) < 0.05
    assert _relerr(m.var(ddof=1), beta / mu_m) < 0.20
    assert _relerr(p.mean(), k_t * beta / (mu_m * mu_p)) < 0.05
    assert _relerr(p.var(ddof=1) / p.mean(), 1 + k_t / (mu_m + mu_p)) < 0.20


def test_two_gene_means(pkg, orc):
    """test/test_analytical_moments.jl:195-204 (two unregulated genes, CLE means < 5%)."""
    b1, b2, mu_m, mu_p, k_t = 2.0, 5.0, 0.1, 0.2, 1.0
    net = pkg.GeneNetwork(2, [b1, b2], np.zeros((2, 2)))
    kin = pkg.KineticParams(k_t=k_t, K_d=50.0, n=2.0, mu_m=mu_m, mu_p=mu_p)
    r = orc.simulate(net, kin, dt=0.1, T=500.0, cell_num=5000, seed=100)
    for g, b in enumerate((b1, b2)):
        assert _relerr(r["M"][g].mean(), b / mu_m) < 0.05
        assert _relerr(r["P"][g].mean(), k_t * b / (mu_m * mu_p)) < 0.05


def test_dilution_moments(pkg, orc):
    """test/test_analytical_moments.jl:306-314 (dilution 0.03)."""
    beta, mu_m, mu_p, k_t, mu = 2.0, 0.1, 0.2, 1.0, 0.03
    net, kin = _one_gene(pkg, beta, k_t=k_t, K_d=50.0, n=2.0, mu_m=mu_m, mu_p=mu_p, dilution=mu)
    r = orc.simulate(net, kin, dt=0.1, T=500.0, cell_num=10000, seed=42)
    m_exact = beta / (mu_m + mu)
    assert _relerr(r["M"][0].mean(), m_exact) < 0.05
    assert _relerr(r["P"][0].mean(), k_t * m_exact / (mu_p + mu)) < 0.05
    p = r["P"][0]
    assert _relerr(p.var(ddof=1) / p.mean(), 1 + k_t / (mu_m + mu_p + 2 * mu)) < 0.20


def test_high_count_fano(pkg, orc):
    """test/test_analytical_moments.jl:654-666 (beta=10, CLE Fano within 10%)."""
    net, kin = _one_gene(pkg, 10.0, k_t=1.0, K_d=50.0, n=2.0, mu_m=0.1, mu_p=0.2)
    r = orc.simulate(net, kin, dt=0.1, T=300.0, cell_num=10000, seed=42)
    p = r["P"][0]
    assert _relerr(p.var(ddof=1) / p.mean(), 1 + 1.0 / 0.3) < 0.10


def test_low_count_clamping(pkg, orc):
    """test/test_analytical_moments.jl:553-631: at <m> ~ 1 the CLE mean is biased by
    at most 25% and clamped zeros appear."""
    net, kin = _one_gene(pkg, 0.1, k_t=1.0, K_d=50.0, n=2.0, mu_m=0.1, mu_p=0.2)
    r = orc.simulate(net, kin, dt=0.05, T=500.0, cell_num=15000, seed=42)
    m = r["M"][0]
    assert _relerr(m.mean(), 1.0) < 0.25
    assert np.count_nonzero(m == 0.0) > 0


def test_telegraph_mean(pkg, orc):
    """Telegraph gating (tauleap_binomial.jl:64-137 semantics): the mRNA mean matches
    the exact telegraph mean k_on/(k_on+k_off) * beta/mu_m (src/analytical.jl:102)."""
    k_on, k_off, beta, mu_m = 0.5, 2.0, 20.0, 1.0
    net = pkg.GeneNetwork(1, [beta], np.zeros((1, 1)), k_on=[k_on], k_off=[k_off])
    kin = pkg.KineticParams(k_t=1.0, K_d=50.0, n=2.0, mu_m=mu_m, mu_p=0.2)
    r = orc.simulate(net, kin, dt=0.01, T=30.0, cell_num=8000, seed=5)
    a, b, c = k_on / mu_m, k_off / mu_m, beta / mu_m
    assert _relerr(r["M"][0].mean(), a * c / (a + b)) < 0.05
    frac_on = r["prom"][0].mean()
    assert abs(frac_on - k_on / (k_on + k_off)) < 0.02


def test_switch_waiting_time_is_geometric(orc):
    """A promoter switching at a step draws its next waiting time from the 18 spare bits
    of its normal words: over all 2^18 uniforms, P(K > k) = q^k (q = exp(-k_sw dt)) to
    within the grid spacing, i.e. the per-step Bernoulli switching of
    tauleap_binomial.jl:111-121."""
    rng = np.random.default_rng(1)
    for w0, w1 in rng.integers(0, 2**32, size=(50, 2), dtype=np.uint64):
        w0, w1 = int(w0), int(w1)
        want = ((((w0 & 511) << 9) | (w1 & 511)) + 1) / 2.0**18
        assert orc.switch_uniform(w0, w1) == np.float32(want)
    for rate, dt in ((0.5, 0.01), (7.0, 0.01), (2.0, 0.1)):
        inv = np.float32(-math.log(2.0) / (rate * dt))
        q = math.exp(-rate * dt)
        u = (np.arange(2**18, dtype=np.float64) + 1.0) / 2.0**18
        K = np.array([orc.geom_steps_u(x, inv) for x in u])
        assert K.min() >= 1
        mean_wait = 1.0 / (1.0 - q)
        for k in np.unique(np.linspace(0, 5 * mean_wait, 40).astype(int)):
            assert abs(np.mean(K > k) - q ** k) < 2.0**-16, (rate, dt, k)


def test_capture_bands(orc):
    """test/test_capture.jl:1-31 on the inverse-CDF capture sampler."""
    rng = np.random.default_rng(42)
    X = np.round(rng.random((5, 1000)) * 100)  # [G, N]
    eff = orc.capture_efficiency(1000, 0.1, 0.2, 1, seed=100)
    Y = orc.capture_counts(X, eff, seed=100)
    assert np.all(Y <= X) and np.all(Y >= 0)
    rates = Y / np.maximum(X, 1)
    assert abs(rates[X > 10].mean() - 0.1) < 0.05
    eff1 = orc.capture_efficiency(1000, 1.0, 0.01, 1, seed=200)
    Y1 = orc.capture_counts(X, eff1, seed=200)
    assert (Y1 / np.maximum(X, 1)).mean() > 0.95
    eff0 = orc.capture_efficiency(1000, 1e-10, 0.01, 1, seed=300)
    Y0 = orc.capture_counts(X, eff0, seed=300)
    assert Y0.sum() < X.sum() * 0.01


def test_capture_efficiency_lognormal(orc):
    """capture.jl:30-36: mean efficiency equals `efficiency` with the sigma^2/2 correction."""
    eff = orc.capture_efficiency(200000, 0.1, 0.5, 1, seed=9)
    assert abs(eff.mean() - 0.1) < 0.002
    eff_raw = orc.capture_efficiency(200000, 0.1, 0.5, 0, seed=9)
    assert abs(np.log(eff_raw).mean() - math.log(0.1)) < 0.01


def test_binomial_sampler_moments(orc):
    n, p = 700, 0.37
    xs = np.array([orc.binomial_invcdf(n, p, 1, 0, c, 0) for c in range(20000)])
    assert abs(xs.mean() - n * p) < 0.5
    assert abs(xs.var() / (n * p * (1 - p)) - 1) < 0.05
    hs = np.array([orc.binomial_half(301, 1, 0, c, 10, 0, 1) for c in range(20000)])
    assert abs(hs.mean() - 150.5) < 0.2
    assert abs(hs.var() / (301 * 0.25) - 1) < 0.05


def test_population_volume_law(pkg, orc):
    """test/test_analytical_moments.jl:366-421 volume law on the CLE population:
    <V> = V_div ln 2, <1/V> = 3/(2 V_div), median 2 V_div / 3, within 15%; mRNA
    correlates with volume (:423-430)."""
    net, kin = _one_gene(pkg, 2.0, k_t=1.0, K_d=50.0, n=2.0, mu_m=0.1, mu_p=0.2)
    pop = pkg.PopulationConfig(cell_num=5000, growth_rate=0.03, V_div=2.0, V_init=(1.0, 2.0),
                               div_check_interval=1)
    r = orc.simulate(net, kin, dt=0.1, T=500.0, cell_num=5000, seed=42, population=pop)
    V = r["V"]
    assert V.min() >= 1.0 * 0.99
    assert V.max() <= 2.0 * math.exp(0.03 * 0.1) * 1.01
    assert _relerr(V.mean(), 2.0 * math.log(2)) < 0.15
    assert _relerr((1 / V).mean(), 0.75) < 0.15
    assert _relerr(np.median(V), 4.0 / 3.0) < 0.15
    assert np.corrcoef(r["M"][0], V)[0, 1] > 0.1


@pytest.mark.parametrize("partition", ["halve", "binomial"])
def test_population_sanity(pkg, orc, partition):
    """test/test_growth_feedback.jl:40-51 and test_analytical_moments.jl:254-264."""
    net, kin = _one_gene(pkg, 2.0, k_t=1.0, K_d=50.0, n=2.0, mu_m=0.1, mu_p=0.2)
    pop = pkg.PopulationConfig(cell_num=2000, growth_rate=0.03, V_div=2.0, V_init=(0.8, 1.2),
                               div_check_interval=5, partition=partition)
    r = orc.simulate(net, kin, dt=0.1, T=200.0, cell_num=2000, seed=42, population=pop)
    P = r["P"][0]
    assert P.shape == (2000,)
    assert np.all(P >= 0) and np.all(np.isfinite(P)) and P.mean() > 0
    if partition == "binomial":
        # right after a division check the split counts are integers; the mean stays near
        # the dilution-free level scaled by the mean volume (transcription ~ V)
        assert P.mean() > 0.5 * 100


def test_regulated_network_runs(pkg, orc):
    net = pkg.sample_network(10, seed=3, bursty=True)
    r = orc.simulate(net, pkg.WORKLOAD_KINETICS, dt=0.01, T=5.0, cell_num=300, seed=1)
    assert np.all(np.isfinite(r["M"])) and np.all(r["M"] >= 0) and np.all(r["P"] >= 0)
