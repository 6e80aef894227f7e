"""GPU binomial tau-leap (ext/SyntheticscRNAseqCUDAExt.jl:215-399, population :531-663) against
the oracle's FP32 restatement, through the C ABI.

Unregulated networks (constitutive and telegraph genes, with and without a Moran population):
the kernel and the oracle run the same explicitly rounded FP32 operations on the same Philox
uniforms, so counts, promoter states, volumes and the concentration readout are bit-exact.
Regulated networks: the oracle's regulation is FP64 (cle.jl's contraction) and the kernel's
FP32, so a count can differ where a uniform falls within rounding of a Poisson CDF step;
fewer than 1 % of the final counts may differ and per-gene means agree within 1 %.
The kernel draws a thread unit's Poisson counts either in lock step or one after another
(SCRNA_TAU_LOCKSTEP=1 / 0 forces one; lock step by default), for units of gene pairs or
quads or single genes (SCRNA_TAU_GENES_PER_THREAD=2 / 4 / 1; pairs by default): every combination gives the same
bits, so the bit-exact cases run under several.
Beyond 128 genes the automatic path runs the tau-leap's tensor form, whose FP32 regulation
follows the register path's operations, so its counts are the register path's bit for bit.
Statistical pins of the reference: test/test_analytical_moments.jl:85-96 (means within 3 %,
variance and Fano within 15 % of the exact two-stage moments) and test/test_gpu_parity.jl:32-42.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _unregulated(pkg, G, bursty, seed):
    rng = np.random.default_rng(seed)
    kon = np.exp(rng.uniform(np.log(0.1), np.log(1.0), G)) if bursty else None
    koff = np.exp(rng.uniform(np.log(1.0), np.log(10.0), G)) if bursty else None
    return pkg.GeneNetwork(G, np.exp(rng.uniform(0.0, np.log(10.0), G)), np.zeros((G, G)), k_on=kon, k_off=koff)


def _tau_run(pkg, net, kin, **kw):
    run = pkg.DeviceRun(net, pkg.BinomialTauLeap(kw.pop("dt", 0.05)), kin, **kw)
    run.launch()
    return run


@pytest.fixture(params=[("0", "4"), ("1", "4"), ("1", "2"), ("1", "1")],
                ids=["serial-quads", "lockstep-quads", "lockstep-pairs", "lockstep-singles"])
def schedule(request, monkeypatch):
    monkeypatch.setenv("SCRNA_TAU_LOCKSTEP", request.param[0])
    monkeypatch.setenv("SCRNA_TAU_GENES_PER_THREAD", request.param[1])
    return request.param


@pytest.mark.parametrize("G,bursty", [(1, False), (4, False), (7, True), (13, True)])
def test_unregulated_trajectories_bit_exact(pkg, orc, G, bursty, schedule):
    net = _unregulated(pkg, G, bursty, seed=G)
    kin = pkg.KineticParams(k_t=3.0, K_d=10.0, n=2.0, mu_m=0.7, mu_p=0.3)
    N, steps = 300, 400
    got = _tau_run(pkg, net, kin, cell_num=N, T=0.0, n_steps=steps, seed=5, readout="both").read_raw()
    ref = orc.simulate(net, kin, dt=0.05, cell_num=N, n_steps=steps, seed=5, tauleap=True)
    assert np.array_equal(got["M"], ref["M"]) and np.array_equal(got["P"], ref["P"])
    assert np.array_equal(got["prom"], ref["prom"])
    assert np.all(got["M"] == np.round(got["M"])) and np.all(got["M"] >= 0)


@pytest.mark.parametrize("partition,exclude_mother", [("binomial", False), ("halve", True)])
def test_population_bit_exact(pkg, orc, partition, exclude_mother, schedule):
    net = _unregulated(pkg, 5, True, seed=9)
    kin = pkg.KineticParams(k_t=2.0, K_d=10.0, n=2.0, mu_m=0.8, mu_p=0.25, dilution=0.1)
    N, steps = 200, 350
    pop = pkg.PopulationConfig(cell_num=N, growth_rate=0.7, V_div=2.0, V_init=(1.0, 2.0), div_check_interval=10,
                               partition=partition, exclude_mother=exclude_mother)
    run = _tau_run(pkg, net, kin, cell_num=N, T=0.0, n_steps=steps, seed=8, readout="both", population=pop)
    got = run.read_raw()
    ref = orc.simulate(net, kin, dt=0.05, cell_num=N, n_steps=steps, seed=8, population=pop, tauleap=True)
    assert np.array_equal(got["V"], ref["V"])
    assert np.array_equal(got["M"], ref["M"]) and np.array_equal(got["P"], ref["P"])
    # readout: concentrations (ext:654-661)
    X = run.read()
    assert np.array_equal(X[:, :5], (ref["M"] / ref["V"]).T) and np.array_equal(X[:, 5:], (ref["P"] / ref["V"]).T)


def test_regulated_network_against_oracle(pkg, orc):
    net = pkg.sample_network(10, seed=1, bursty=True)
    assert net.cooperative or net.redundant
    kin = pkg.WORKLOAD_KINETICS
    N, steps = 2000, 300
    got = _tau_run(pkg, net, kin, cell_num=N, T=0.0, n_steps=steps, seed=4, readout="both", dt=0.01).read_raw()
    ref = orc.simulate(net, kin, dt=0.01, cell_num=N, n_steps=steps, seed=4, tauleap=True)
    assert np.array_equal(got["prom"], ref["prom"])
    for k in ("M", "P"):
        assert np.mean(got[k] != ref[k]) < 0.01, k
        mg, mr = got[k].mean(1), ref[k].mean(1)
        assert np.max(np.abs(mg - mr) / np.maximum(mr, 1.0)) < 0.01, k


@pytest.mark.parametrize("G", [23, 130])
def test_schedules_equal_on_regulated_network(pkg, monkeypatch, G):
    """Lock-step and one-after-another draws, gene quads and gene pairs per thread: same
    counts, promoters and volumes, with regulation, telegraph genes and a population (cells
    beyond several tiles; 130 genes: several units per thread)."""
    net = pkg.sample_network(G, seed=5, bursty=True)
    kin = pkg.WORKLOAD_KINETICS
    pop = pkg.PopulationConfig(cell_num=700, growth_rate=0.7, V_div=2.0, V_init=(1.0, 2.0), div_check_interval=10)
    outs = []
    for mode, unit in (("0", "4"), ("1", "4"), ("1", "2"), ("0", "2"), ("1", "1")):
        monkeypatch.setenv("SCRNA_TAU_LOCKSTEP", mode)
        monkeypatch.setenv("SCRNA_TAU_GENES_PER_THREAD", unit)
        outs.append(_tau_run(pkg, net, kin, cell_num=700, T=0.0, n_steps=250, seed=3, readout="both", dt=0.01,
                             population=pop, path="register").read_raw())
    for o in outs[1:]:
        for k in ("M", "P", "prom", "V"):
            assert np.array_equal(outs[0][k], o[k]), k


@pytest.mark.parametrize("kind,G", [("sampled", 129), ("sampled", 300), ("dense", 300)])
def test_tensor_form_equals_register_path(pkg, kind, G):
    """The tau-leap's tensor form (regulation in FP32 with the register path's operations in
    its order, state cell-major in HBM, gene pairs in lock step) against the register path on
    regulated networks: counts, promoters and volumes bit for bit, with and without a
    population.  The automatic path takes the tensor form beyond 128 genes, so its results
    are the register path's as well."""
    if kind == "sampled":
        net = pkg.sample_network(G, seed=G, bursty=True)
    else:
        net = pkg.dense_network(G, seed=G, density=0.1, n_coop=4, n_redun=4)
    kin = pkg.WORKLOAD_KINETICS
    pop = pkg.PopulationConfig(cell_num=500, growth_rate=0.7, V_div=2.0, V_init=(1.0, 2.0), div_check_interval=10)
    for population in (None, pop):
        outs = [_tau_run(pkg, net, kin, cell_num=500, T=0.0, n_steps=120, seed=3, readout="both", dt=0.01,
                         population=population, path=path) for path in ("register", "tensor", "auto")]
        raws = [r.read_raw() for r in outs]
        Xs = [r.read() for r in outs]
        for r in outs:
            r.close()
        for k in ("M", "P", "prom") + (("V",) if population else ()):
            assert np.array_equal(raws[0][k], raws[1][k]), (population is not None, k)
            assert np.array_equal(raws[0][k], raws[2][k]), (population is not None, k)
        assert np.array_equal(Xs[0], Xs[1]) and np.array_equal(Xs[0], Xs[2])


def test_means_outside_the_quotient_range_bit_exact(pkg, orc, schedule):
    """Basals so small that the transcription means fall below 2^-100 (a quad then takes IEEE
    division instead of the branch-free quotient), beside ordinary genes in the same quads."""
    G = 7
    basals = np.array([1e-33, 3.0, 2e-32, 5.0, 1e-34, 0.5, 4.0])
    net = pkg.GeneNetwork(G, basals, np.zeros((G, G)))
    kin = pkg.KineticParams(k_t=2.0, K_d=10.0, n=2.0, mu_m=0.6, mu_p=0.3)
    got = _tau_run(pkg, net, kin, cell_num=100, T=0.0, n_steps=150, seed=9, readout="both").read_raw()
    ref = orc.simulate(net, kin, dt=0.05, cell_num=100, n_steps=150, seed=9, tauleap=True)
    assert np.array_equal(got["M"], ref["M"]) and np.array_equal(got["P"], ref["P"])


def test_small_div_matches_ieee_division(pkg):
    """The tau-leap's branch-free quotient lam / k (Markstein's correction of lam * RN(1/k))
    equals IEEE division for every float lam in [2^-100, 2^100] and every k = 1..50."""
    lo = 27 << 23          # 2^-100
    hi = (227 << 23) + 1   # 2^100, included
    n, lam, k = pkg.debug_small_div_check(lo, hi)
    assert n == 0, (hex(lam), k)
    assert pkg.debug_small_div_check(0, 1)[0] == 0  # lam = 0


def test_two_stage_moments(pkg):
    """test/test_analytical_moments.jl:85-96 on the GPU tau-leap."""
    beta, mu_m, mu_p, k_t = 2.0, 0.1, 0.2, 1.0
    net = pkg.GeneNetwork(1, [beta], np.zeros((1, 1)))
    kin = pkg.KineticParams(k_t=k_t, K_d=50.0, n=2.0, mu_m=mu_m, mu_p=mu_p)
    Y = pkg.simulate(net, pkg.BinomialTauLeap(0.1), kin, cell_num=10000, T=500.0, readout="both", seed=42)
    m, p = Y[:, 0], Y[:, 1]
    assert abs(m.mean() / (beta / mu_m) - 1) < 0.03
    assert abs(m.var(ddof=1) / (beta / mu_m) - 1) < 0.15
    assert abs(p.mean() / (k_t * beta / (mu_m * mu_p)) - 1) < 0.03
    assert abs((p.var(ddof=1) / p.mean()) / (1 + k_t / (mu_m + mu_p)) - 1) < 0.15


def test_gpu_vs_cpu_mean(pkg, orc):
    """test/test_gpu_parity.jl:32-42: GPU tau-leap mean within 5 % of the CPU run's."""
    net = pkg.GeneNetwork(1, [5.0], np.zeros((1, 1)))
    kin = pkg.KineticParams(k_t=2.0, K_d=50.0, n=2.0, mu_m=0.1, mu_p=0.2)
    Yg = pkg.simulate(net, pkg.BinomialTauLeap(0.1), kin, cell_num=5000, T=200.0, readout="protein", seed=42)
    Yc = orc.simulate(net, kin, dt=0.1, T=200.0, cell_num=5000, seed=7, tauleap=True)["P"][0]
    assert abs(Yg.mean() - Yc.mean()) / Yc.mean() < 0.05


def test_batch_equals_single_runs_and_oracle(pkg, orc):
    """simulate_gpu_batch(networks, BinomialTauLeap(dt), kinetics; ...) with uneven G and cells,
    per-network kinetics and populations (ext:666-837): equal to single runs bit for bit, and
    for the unregulated networks to the oracle."""
    nets = [_unregulated(pkg, G, bool(i % 2), seed=50 + i) for i, G in enumerate((2, 5, 9, 3))]
    nets.append(pkg.sample_network(12, seed=3, bursty=True))
    kins = [pkg.KineticParams(k_t=2.0 + i, K_d=10.0, n=2.0, mu_m=0.5 + 0.1 * i, mu_p=0.2) for i in range(5)]
    cells = [100, 257, 64, 300, 150]
    pops = [None, pkg.PopulationConfig(cell_num=257, growth_rate=0.7, V_div=2.0, V_init=(1.0, 2.0),
                                       div_check_interval=10, exclude_mother=False), None, None,
            pkg.PopulationConfig(cell_num=150, growth_rate=0.5, V_div=2.0, V_init=(1.0, 2.0), div_check_interval=5)]
    T, dt = 2.0, 0.05
    outs = pkg.simulate_gpu_batch(nets, pkg.BinomialTauLeap(dt), kins, cell_num=cells, T=T, populations=pops,
                                  readout="both", seed=6, stream=20)
    for b, net in enumerate(nets):
        single = pkg.simulate(net, pkg.BinomialTauLeap(dt), kins[b], population=pops[b], cell_num=cells[b], T=T,
                              readout="both", seed=6, stream=20 + b)
        assert np.array_equal(outs[b], single), b
        if b < 4:
            r = orc.simulate(net, kins[b], dt=dt, T=T, cell_num=cells[b], seed=6, stream=20 + b, population=pops[b],
                             tauleap=True)
            M, P = (r["M"] / r["V"], r["P"] / r["V"]) if pops[b] is not None else (r["M"], r["P"])
            assert np.array_equal(outs[b], np.hstack([M.T, P.T])), b


def test_tauleap_capture_and_validation(pkg, orc):
    net = _unregulated(pkg, 6, True, seed=77)
    kin = pkg.KineticParams(k_t=4.0, K_d=10.0, n=2.0, mu_m=1.0, mu_p=0.2)
    cap = pkg.CaptureModel(efficiency=0.3, efficiency_std=0.4, readout="protein")
    X, counts, eff = pkg.simulate(net, pkg.BinomialTauLeap(0.02), kin, cell_num=400, T=3.0, readout="protein",
                                  seed=12, capture=cap)
    want = orc.capture_counts(np.ascontiguousarray(X.T), eff, seed=12)
    assert np.array_equal(counts.T, want)
    with pytest.raises(pkg.ScrnaError):  # the lane kernel has no tau-leap form
        pkg.simulate(net, pkg.BinomialTauLeap(0.02), kin, cell_num=10, T=1.0, path="warp")
    # the tensor path's tau-leap (the library-GEMM variant under either name): with no regulation
    # its counts, capture included, equal the register path's
    for path in ("tensor", "tensor_library"):
        Xt, ct, et = pkg.simulate(net, pkg.BinomialTauLeap(0.02), kin, cell_num=400, T=3.0, readout="protein",
                                  seed=12, capture=cap, path=path)
        assert np.array_equal(Xt, X) and np.array_equal(ct, counts) and np.array_equal(et, eff), path


def test_regulated_batch_across_both_forms_bit_exact(pkg):
    """A batch of regulated tau-leap networks on both sides of 128 genes (the register path's
    grouped launch and the tensor form, running side by side): every network's readout and
    capture equal its single run on the register path bit for bit, populations included."""
    nets = [pkg.sample_network(40, seed=41, bursty=True), pkg.sample_network(200, seed=42, bursty=True),
            pkg.sample_network(12, seed=43, bursty=True), pkg.sample_network(300, seed=44, bursty=True)]
    kin = pkg.WORKLOAD_KINETICS
    cells = [300, 250, 400, 200]
    pops = [None, pkg.PopulationConfig(cell_num=250, growth_rate=0.7, V_div=2.0, V_init=(1.0, 2.0),
                                       div_check_interval=10), None, None]
    cap = pkg.CaptureModel(efficiency=0.3, efficiency_std=0.4, readout="protein")
    alg = pkg.BinomialTauLeap(0.01)
    outs, counts = pkg.simulate_gpu_batch(nets, alg, kin, cell_num=cells, T=0.8, readout="both", seed=9, stream=30,
                                          populations=pops, capture=cap)
    for b, net in enumerate(nets):
        X, c, _ = pkg.simulate(net, alg, kin, population=pops[b], cell_num=cells[b], T=0.8, readout="both", seed=9,
                               stream=30 + b, capture=cap, path="register")
        assert np.array_equal(outs[b], X), b
        assert np.array_equal(counts[b], c), b
