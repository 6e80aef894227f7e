"""GPU tests of the tensor-core path (dense regulation, 16-bit GEMM inputs, FP32 state):
the fused tcgen05 kernel (path "tensor") and the library-GEMM variant ("tensor_library").

Tolerances: the GEMM rounds W = A_eff and the Hill activations to BF16 (8-bit mantissa) or
FP16 (11-bit), so trajectories are compared against the FP32 register path with
|tensor - register| <= TOL * max(|register|, 1): TOL = 5e-2 (BF16), 1e-2 (FP16) after 150 steps;
per-gene ensemble means against the FP64 oracle on the same increments within 2 %.
Promoter states and capture counts (given the path's own X and efficiencies) are exact.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dense(pkg, G, seed, density=0.3, bursty=False):
    net = pkg.dense_network(G, seed=seed, density=density, n_coop=4, n_redun=4)
    if bursty:
        rng = np.random.default_rng(seed)
        net = pkg.GeneNetwork(G, net.basals, net.interactions, net.cooperative, net.redundant,
                              k_on=np.exp(rng.uniform(np.log(0.1), np.log(1.0), G)),
                              k_off=np.exp(rng.uniform(np.log(1.0), np.log(10.0), G)))
    return net


def _run(pkg, net, kin, path, precision="fp32", N=300, steps=150, seed=3, **kw):
    run = pkg.DeviceRun(net, pkg.CLE(0.01), kin, cell_num=N, T=0.0, n_steps=steps, readout="both",
                        seed=seed, path=path, precision=precision, **kw)
    run.launch()
    return run


def _rel(a, b):
    return float(np.max(np.abs(np.asarray(a, np.float64) - b) / np.maximum(np.abs(b), 1.0)))


@pytest.mark.parametrize("path", ["tensor", "tensor_library"])
@pytest.mark.parametrize("precision,tol", [("fp32", 5e-2), ("fp32_f16", 1e-2)])
@pytest.mark.parametrize("bursty", [False, True])
def test_tensor_matches_register_path(pkg, path, precision, tol, bursty):
    net = _dense(pkg, 64, seed=1, bursty=bursty)
    kin = pkg.WORKLOAD_KINETICS
    ref = _run(pkg, net, kin, "block").read_raw()
    got = _run(pkg, net, kin, path, precision=precision).read_raw()
    assert np.array_equal(got["prom"], ref["prom"])
    assert _rel(got["M"], ref["M"].astype(np.float64)) < tol
    assert _rel(got["P"], ref["P"].astype(np.float64)) < tol


@pytest.mark.parametrize("path", ["tensor", "tensor_library"])
def test_tensor_per_gene_means_vs_oracle(pkg, orc, path):
    net = _dense(pkg, 200, seed=5, density=0.1)
    kin = pkg.WORKLOAD_KINETICS
    N, steps = 2048, 300
    got = _run(pkg, net, kin, path, N=N, steps=steps, seed=11).read_raw()
    ref = orc.simulate(net, kin, dt=0.01, cell_num=N, n_steps=steps, seed=11)
    for key in ("M", "P"):
        mg = got[key].astype(np.float64).mean(1)
        mr = ref[key].mean(1)
        err = np.abs(mg - mr) / np.maximum(np.abs(mr), 1.0)
        assert err.max() < 0.02, (key, err.max())


def test_tensor_readout_and_capture(pkg, orc):
    net = _dense(pkg, 96, seed=7)
    kin = pkg.WORKLOAD_KINETICS
    cap = pkg.CaptureModel(efficiency=0.2, efficiency_std=0.5, readout="protein")
    X, counts, eff = pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=333, T=1.0, readout="protein", seed=4,
                                  capture=cap, path="tensor")
    raw = pkg.DeviceRun(net, pkg.CLE(0.01), kin, cell_num=333, T=1.0, readout="both", seed=4, path="tensor")
    raw.launch()
    both = raw.read()
    assert np.array_equal(both[:, 96:], X)
    want = orc.capture_counts(np.ascontiguousarray(X.T), eff, seed=4)
    assert np.array_equal(counts.T, want)


def test_auto_picks_tensor_for_large_dense(pkg):
    net = _dense(pkg, 600, seed=2, density=0.1)
    kin = pkg.WORKLOAD_KINETICS
    a = pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=128, T=0.2, seed=1)
    b = pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=128, T=0.2, seed=1, path="tensor")
    assert np.array_equal(a, b)


def test_auto_routing_of_dense_networks(pkg):
    """The automatic path on networks of >= 256 genes at >= 5 % density (here 10 %): the
    tau-leap and populations run on the tensor path (the library-GEMM variant, their tensor
    form); the CLE of 256 genes (64 gene quads) stays on the register path below 8,192 cells
    and moves to the tensor path from there on."""
    kin = pkg.WORKLOAD_KINETICS
    net = _dense(pkg, 400, seed=4, density=0.1)
    pop = pkg.PopulationConfig(cell_num=300, growth_rate=0.7, V_div=2.0, V_init=(1.0, 2.0), div_check_interval=10)
    for alg, population in ((pkg.BinomialTauLeap(0.01), None), (pkg.BinomialTauLeap(0.01), pop), (pkg.CLE(0.01), pop)):
        kw = dict(cell_num=300, T=0.2, readout="both", seed=3, population=population)
        a = pkg.simulate(net, alg, kin, **kw)
        b = pkg.simulate(net, alg, kin, path="tensor_library", **kw)
        assert np.array_equal(a, b), (type(alg).__name__, population is not None)
    net = _dense(pkg, 256, seed=5, density=0.1)
    for N, path in ((1000, "register"), (8192, "tensor")):
        a = pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=N, T=0.05, readout="both", seed=1)
        b = pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=N, T=0.05, readout="both", seed=1, path=path)
        assert np.array_equal(a, b), N


@pytest.mark.parametrize("G,N,bursty", [(300, 333, False), (520, 700, True)])
def test_fused_matches_library_gemm_path(pkg, G, N, bursty):
    """Ragged tiles (G not a multiple of 256, N not of 128): the fused tcgen05 kernel and the
    library-GEMM variant agree on the same increments up to the 16-bit contraction's rounding
    (different accumulation order); promoter states are exact."""
    net = _dense(pkg, G, seed=G, density=0.1, bursty=bursty)
    kin = pkg.WORKLOAD_KINETICS
    a = _run(pkg, net, kin, "tensor", N=N, steps=60, seed=5).read_raw()
    b = _run(pkg, net, kin, "tensor_library", N=N, steps=60, seed=5).read_raw()
    assert np.array_equal(a["prom"], b["prom"])
    assert _rel(a["M"], b["M"].astype(np.float64)) < 2e-2
    assert _rel(a["P"], b["P"].astype(np.float64)) < 2e-2


@pytest.mark.parametrize("path", ["tensor", "tensor_library"])
@pytest.mark.parametrize("G,n_terms,n_src", [(67, 13, (5, 7)), (72, 9, (2, 6)), (64, 8, (4, 4))])
def test_tensor_long_and_ragged_terms(pkg, path, G, n_terms, n_src):
    """Term columns with more sources than one load round (4) takes, term groups that do
    not fill 8 columns, and term columns that start off a 16-byte boundary (G odd, or G+8k
    not a multiple of 8): against the FP32 register path."""
    net = pkg.dense_network(G, seed=G + n_terms, density=0.2, n_coop=(n_terms + 1) // 2, n_redun=n_terms // 2,
                            n_sources_range=n_src)
    assert max(len(e.sources) for e in list(net.cooperative) + list(net.redundant)) >= n_src[0]
    kin = pkg.WORKLOAD_KINETICS
    ref = _run(pkg, net, kin, "block", N=257).read_raw()
    got = _run(pkg, net, kin, path, N=257).read_raw()
    assert np.array_equal(got["prom"], ref["prom"])
    assert _rel(got["M"], ref["M"].astype(np.float64)) < 5e-2
    assert _rel(got["P"], ref["P"].astype(np.float64)) < 5e-2
