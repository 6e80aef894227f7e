"""Populations on the tensor path (the library-GEMM variant), through the C ABI: growth,
division checks, partition and Moran replacement over the cell-major state, for the CLE
(cle.jl:143-284, ext:409-529) and the binomial tau-leap (ext:531-663).

The tensor path is where networks beyond the register path's 512 genes run.  Without
regulation its GEMM gives exactly 0, and every other operation is the register path's, so
counts, promoters, volumes and the readout (concentrations for the tau-leap) equal the
register path's bit for bit at sizes both paths take, and the oracle's beyond them (the
tau-leap restatement is FP32 like the kernels).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _unregulated(pkg, G, seed, bursty=True):
    rng = np.random.default_rng(seed)
    kon = np.exp(rng.uniform(np.log(0.1), np.log(1.0), G)) if bursty else None
    koff = np.exp(rng.uniform(np.log(1.0), np.log(10.0), G)) if bursty else None
    return pkg.GeneNetwork(G, np.exp(rng.uniform(0.0, np.log(10.0), G)), np.zeros((G, G)), k_on=kon, k_off=koff)


def _run(pkg, net, alg, kin, pop, path, steps, seed=5):
    run = pkg.DeviceRun(net, alg, kin, cell_num=pop.cell_num, T=0.0, n_steps=steps, readout="both", seed=seed,
                        population=pop, path=path)
    run.launch()
    out = run.read_raw(), run.read()
    run.close()
    return out


@pytest.mark.parametrize("tau", [False, True], ids=["cle", "tauleap"])
@pytest.mark.parametrize("partition,exclude_mother", [("binomial", False), ("halve", True)])
def test_tensor_population_equals_register_path(pkg, tau, partition, exclude_mother):
    net = _unregulated(pkg, 9, seed=4)
    kin = pkg.KineticParams(k_t=2.0, K_d=10.0, n=2.0, mu_m=0.8, mu_p=0.25, dilution=0.1)
    pop = pkg.PopulationConfig(cell_num=300, growth_rate=0.7, V_div=2.0, V_init=(1.0, 2.0), div_check_interval=10,
                               partition=partition, exclude_mother=exclude_mother)
    alg = pkg.BinomialTauLeap(0.05) if tau else pkg.CLE(0.01)
    steps = 230  # 23 division checks, the last step one of them
    (ra, xa) = _run(pkg, net, alg, kin, pop, "register", steps)
    (rb, xb) = _run(pkg, net, alg, kin, pop, "tensor_library", steps)
    for k in ("V", "prom", "M", "P"):
        assert np.array_equal(ra[k], rb[k]), k
    assert np.array_equal(xa, xb)
    assert np.any(ra["V"] < 2.0)  # divisions happened


def test_tauleap_population_beyond_the_register_path_bit_exact(pkg, orc):
    net = _unregulated(pkg, 640, seed=6)
    kin = pkg.KineticParams(k_t=3.0, K_d=10.0, n=2.0, mu_m=0.7, mu_p=0.3)
    pop = pkg.PopulationConfig(cell_num=64, growth_rate=0.7, V_div=2.0, V_init=(1.0, 2.0), div_check_interval=10)
    raw, X = _run(pkg, net, pkg.BinomialTauLeap(0.05), kin, pop, "auto", 120, seed=8)
    ref = orc.simulate(net, kin, dt=0.05, cell_num=64, n_steps=120, seed=8, population=pop, tauleap=True)
    assert np.array_equal(raw["V"], ref["V"])
    for k in ("M", "P", "prom"):
        assert np.array_equal(raw[k], ref[k]), k
    G = net.G
    assert np.array_equal(X[:, :G], (ref["M"] / ref["V"]).T) and np.array_equal(X[:, G:], (ref["P"] / ref["V"]).T)


def test_batch_with_a_population_network_beyond_the_register_path(pkg):
    nets = [_unregulated(pkg, 6, 1), _unregulated(pkg, 600, 2), _unregulated(pkg, 20, 3, bursty=False)]
    kin = pkg.KineticParams(k_t=2.0, K_d=10.0, n=2.0, mu_m=0.6, mu_p=0.2)
    pops = [pkg.PopulationConfig(cell_num=80, growth_rate=0.7, V_div=2.0, V_init=(1.0, 2.0), div_check_interval=5),
            pkg.PopulationConfig(cell_num=50, growth_rate=0.7, V_div=2.0, V_init=(1.0, 2.0), div_check_interval=10),
            None]
    cells = [80, 50, 120]
    for alg in (pkg.CLE(0.01), pkg.BinomialTauLeap(0.05)):
        outs = pkg.simulate_gpu_batch(nets, alg, kin, cell_num=cells, T=1.5, readout="both", seed=2, stream=4,
                                      populations=pops)
        for b, net in enumerate(nets):
            single = pkg.simulate(net, alg, kin, population=pops[b], cell_num=cells[b], T=1.5, readout="both",
                                  seed=2, stream=4 + b)
            assert np.array_equal(outs[b], single), (type(alg).__name__, b)


def test_regulated_population_beyond_the_register_path_vs_oracle(pkg, orc):
    """A regulated 600-gene network with a population (CLE) against the FP64 oracle on the same
    increments: the BF16 contraction and FP32 state move individual trajectories, and a binomial
    partition of a count that the two round differently sends cells down different paths, so the
    check is statistical: per-gene mean mRNA and protein within 3 % (and within 1 count) and the
    cell volumes' mean within 0.5 %, as the divisions follow the same deterministic volumes."""
    net = pkg.sample_network(600, seed=21, bursty=True)
    kin = pkg.WORKLOAD_KINETICS
    pop = pkg.PopulationConfig(cell_num=400, growth_rate=0.7, V_div=2.0, V_init=(1.0, 2.0), div_check_interval=10)
    raw, _ = _run(pkg, net, pkg.CLE(0.01), kin, pop, "auto", 150, seed=12)
    ref = orc.simulate(net, kin, dt=0.01, cell_num=400, n_steps=150, seed=12, population=pop)
    assert abs(raw["V"].mean() / ref["V"].mean() - 1.0) < 0.005
    for k in ("M", "P"):
        mg, mr = raw[k].mean(1), ref[k].mean(1)
        assert np.all(np.abs(mg - mr) <= np.maximum(0.03 * mr, 1.0)), k
