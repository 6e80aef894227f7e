"""The paths at their size limits, through the C ABI: the register path's largest network
(512 genes = 128 gene quads; the lane kernel's limit too), the binomial tau-leap's, and the
fused tensor-core kernel's (4,096 genes, its epilogue gene table in shared memory), plus the
sizes just beyond them: rejected on the register path, routed to the library-GEMM variant
on the tensor path (the tau-leap included).  Tolerances as in the parity tests (2e-3 relative against the FP64
oracle on the same increments; bit-exact for the unregulated tau-leap; the 16-bit
contraction's rounding between the two tensor variants)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 2e-3


def _rel(a, b):
    return float(np.max(np.abs(np.asarray(a, np.float64) - b) / np.maximum(np.abs(b), 1.0)))


def _raw(pkg, net, alg, kin, *, N, steps, seed, path="auto", precision="fp32"):
    run = pkg.DeviceRun(net, alg, kin, cell_num=N, T=0.0, n_steps=steps, readout="both", seed=seed, path=path,
                        precision=precision)
    run.launch()
    out = run.read_raw()
    run.close()
    return out


def test_register_path_at_512_genes(pkg, orc):
    net = pkg.sample_network(512, seed=31, bursty=True)
    kin = pkg.WORKLOAD_KINETICS
    N, steps = 40, 60
    lane = _raw(pkg, net, pkg.CLE(0.01), kin, N=N, steps=steps, seed=2, path="warp")
    block = _raw(pkg, net, pkg.CLE(0.01), kin, N=N, steps=steps, seed=2, path="block")
    for k in ("M", "P", "prom"):
        assert np.array_equal(lane[k], block[k]), k
    ref = orc.simulate(net, kin, dt=0.01, cell_num=N, n_steps=steps, seed=2)
    assert np.array_equal(lane["prom"], ref["prom"])
    assert _rel(lane["M"], ref["M"]) < RTOL and _rel(lane["P"], ref["P"]) < RTOL


def test_register_path_rejects_513_genes(pkg):
    net = pkg.sample_network(513, seed=32, bursty=False)
    for path in ("register", "warp", "block"):
        with pytest.raises(pkg.ScrnaError):
            pkg.simulate(net, pkg.CLE(0.01), pkg.WORKLOAD_KINETICS, cell_num=8, T=0.1, path=path)
    for path in ("register", "block", "warp"):
        with pytest.raises(pkg.ScrnaError):
            pkg.simulate(net, pkg.BinomialTauLeap(0.01), pkg.WORKLOAD_KINETICS, cell_num=8, T=0.1, path=path)
    # the automatic path takes them to the tensor path, populations included
    pop = pkg.PopulationConfig(cell_num=8, growth_rate=0.7, V_div=2.0, V_init=(1.0, 2.0), div_check_interval=10)
    for alg in (pkg.CLE(0.01), pkg.BinomialTauLeap(0.01)):
        X = pkg.simulate(net, alg, pkg.WORKLOAD_KINETICS, population=pop, T=0.2, readout="both")
        assert X.shape == (8, 2 * 513) and np.all(np.isfinite(X))


def _unregulated(pkg, G, seed):
    rng = np.random.default_rng(seed)
    return pkg.GeneNetwork(G, np.exp(rng.uniform(0.0, np.log(10.0), G)), np.zeros((G, G)),
                           k_on=np.exp(rng.uniform(np.log(0.1), np.log(1.0), G)),
                           k_off=np.exp(rng.uniform(np.log(1.0), np.log(10.0), G)))


@pytest.mark.parametrize("G", [601, 1200])
def test_tauleap_beyond_the_register_path_bit_exact(pkg, orc, G):
    """G > 512: the tau-leap runs on the tensor path's library-GEMM variant (ext:215-399 takes any
    G).  Without regulation the GEMM gives exactly 0, so counts and promoters equal the oracle's."""
    net = _unregulated(pkg, G, seed=G)
    kin = pkg.KineticParams(k_t=3.0, K_d=10.0, n=2.0, mu_m=0.7, mu_p=0.3)
    N, steps = 48, 60
    got = _raw(pkg, net, pkg.BinomialTauLeap(0.05), kin, N=N, steps=steps, seed=8)
    ref = orc.simulate(net, kin, dt=0.05, cell_num=N, n_steps=steps, seed=8, tauleap=True)
    for k in ("M", "P", "prom"):
        assert np.array_equal(got[k], ref[k]), k


def test_tauleap_tensor_path_matches_register_path(pkg):
    """A regulated 300-gene network on both tau-leap forms with the same uniforms.  At FP32
    precision the tensor form's regulation is the register path's FP32 arithmetic: the same
    counts bit for bit.  With FP16 inputs it comes from an FP16 contraction, so a count can
    move where a uniform falls within rounding of a Poisson CDF step: promoters are exact,
    counts agree almost everywhere and per-gene means within 1 %."""
    net = pkg.sample_network(300, seed=9, bursty=True)
    kin = pkg.WORKLOAD_KINETICS
    a = _raw(pkg, net, pkg.BinomialTauLeap(0.01), kin, N=500, steps=200, seed=4, path="register")
    b = _raw(pkg, net, pkg.BinomialTauLeap(0.01), kin, N=500, steps=200, seed=4, path="tensor")
    for k in ("M", "P", "prom"):
        assert np.array_equal(a[k], b[k]), k
    c = _raw(pkg, net, pkg.BinomialTauLeap(0.01), kin, N=500, steps=200, seed=4, path="tensor", precision="fp32_f16")
    assert np.array_equal(a["prom"], c["prom"])
    for k in ("M", "P"):
        assert np.mean(a[k] != c[k]) < 0.05, k
        ma, mc = a[k].mean(1), c[k].mean(1)
        assert np.max(np.abs(ma - mc) / np.maximum(ma, 1.0)) < 0.01, k


def test_tauleap_batch_with_a_network_beyond_the_register_path(pkg, orc):
    nets = [_unregulated(pkg, 7, 1), _unregulated(pkg, 700, 2), _unregulated(pkg, 30, 3)]
    kin = pkg.KineticParams(k_t=2.0, K_d=10.0, n=2.0, mu_m=0.6, mu_p=0.2)
    cells = [100, 40, 70]
    outs = pkg.simulate_gpu_batch(nets, pkg.BinomialTauLeap(0.05), kin, cell_num=cells, T=2.0, readout="both",
                                  seed=3, stream=11)
    for b, net in enumerate(nets):
        single = pkg.simulate(net, pkg.BinomialTauLeap(0.05), kin, cell_num=cells[b], T=2.0, readout="both", seed=3,
                              stream=11 + b)
        assert np.array_equal(outs[b], single), b
        r = orc.simulate(net, kin, dt=0.05, T=2.0, cell_num=cells[b], seed=3, stream=11 + b, tauleap=True)
        assert np.array_equal(outs[b], np.hstack([r["M"].T, r["P"].T])), b


@pytest.mark.parametrize("path", ["register", "auto"])
def test_tauleap_at_512_genes_bit_exact(pkg, orc, path):
    rng = np.random.default_rng(512)
    G = 512
    net = pkg.GeneNetwork(G, np.exp(rng.uniform(0.0, np.log(10.0), G)), np.zeros((G, G)),
                          k_on=np.exp(rng.uniform(np.log(0.1), np.log(1.0), G)),
                          k_off=np.exp(rng.uniform(np.log(1.0), np.log(10.0), G)))
    kin = pkg.KineticParams(k_t=3.0, K_d=10.0, n=2.0, mu_m=0.7, mu_p=0.3)
    N, steps = 40, 80
    got = _raw(pkg, net, pkg.BinomialTauLeap(0.05), kin, N=N, steps=steps, seed=6, path=path)
    ref = orc.simulate(net, kin, dt=0.05, cell_num=N, n_steps=steps, seed=6, tauleap=True)
    for k in ("M", "P", "prom"):
        assert np.array_equal(got[k], ref[k]), k


def _dense(pkg, G, seed):
    return pkg.dense_network(G, seed=seed, density=0.02, n_coop=4, n_redun=4)


def test_fused_tensor_kernel_at_4096_genes(pkg):
    """G = 4096: the fused kernel's largest network, against the library-GEMM variant."""
    net = _dense(pkg, 4096, seed=41)
    kin = pkg.WORKLOAD_KINETICS
    a = _raw(pkg, net, pkg.CLE(0.01), kin, N=256, steps=20, seed=3, path="tensor")
    b = _raw(pkg, net, pkg.CLE(0.01), kin, N=256, steps=20, seed=3, path="tensor_library")
    assert np.array_equal(a["prom"], b["prom"])
    assert _rel(a["M"], b["M"]) < 2e-2 and _rel(a["P"], b["P"]) < 2e-2
    assert np.all(np.isfinite(a["M"])) and np.all(a["M"] >= 0)


def test_tensor_path_beyond_4096_genes_uses_library_variant(pkg):
    """G = 4100 on path "tensor": the library-GEMM variant runs (the same result as asking
    for it), since the fused kernel's gene table holds 4,096 genes."""
    net = _dense(pkg, 4100, seed=42)
    kin = pkg.WORKLOAD_KINETICS
    a = _raw(pkg, net, pkg.CLE(0.01), kin, N=200, steps=10, seed=4, path="tensor")
    b = _raw(pkg, net, pkg.CLE(0.01), kin, N=200, steps=10, seed=4, path="tensor_library")
    for k in ("M", "P", "prom"):
        assert np.array_equal(a[k], b[k]), k


def _dense_wide(pkg):
    """500 genes at 10 % density (about 25,000 additive edges) with 4 cooperative and 4
    redundant terms: within the register path's 512 genes, but its tables need about 340 KB
    of shared memory."""
    return pkg.dense_network(500, seed=500, density=0.1, n_coop=4, n_redun=4)


def test_tables_beyond_shared_memory_route_to_the_tensor_path(pkg, orc):
    """The automatic path runs a network whose tables the register path cannot hold on the
    tensor path, the tau-leap and populations included (the same result as asking for it);
    the register path refuses it.  Against the oracle on the same uniforms: promoters exact
    for the tau-leap (the switching draws do not see regulation), per-gene means within 3 %
    (or 1 count), the BF16 contraction moving single trajectories."""
    net = _dense_wide(pkg)
    kin = pkg.WORKLOAD_KINETICS
    N, steps = 300, 100
    with pytest.raises(pkg.ScrnaError):
        _raw(pkg, net, pkg.BinomialTauLeap(0.01), kin, N=8, steps=5, seed=1, path="register")
    auto = _raw(pkg, net, pkg.BinomialTauLeap(0.01), kin, N=N, steps=steps, seed=5)
    tens = _raw(pkg, net, pkg.BinomialTauLeap(0.01), kin, N=N, steps=steps, seed=5, path="tensor")
    for k in ("M", "P", "prom"):
        assert np.array_equal(auto[k], tens[k]), k
    ref = orc.simulate(net, kin, dt=0.01, cell_num=N, n_steps=steps, seed=5, tauleap=True)
    assert np.array_equal(auto["prom"], ref["prom"])
    for k in ("M", "P"):
        mg, mr = auto[k].mean(1), ref[k].mean(1)
        assert np.all(np.abs(mg - mr) <= np.maximum(0.03 * mr, 1.0)), k

    pop = pkg.PopulationConfig(cell_num=N, growth_rate=0.7, V_div=2.0, V_init=(1.0, 2.0), div_check_interval=10)
    for alg, tau in ((pkg.CLE(0.01), False), (pkg.BinomialTauLeap(0.01), True)):
        runs = []
        for path in ("auto", "tensor_library"):
            run = pkg.DeviceRun(net, alg, kin, cell_num=N, T=0.0, n_steps=steps, readout="both", seed=7,
                                population=pop, path=path)
            run.launch()
            runs.append(run.read_raw())
            run.close()
        for k in ("V", "M", "P", "prom"):
            assert np.array_equal(runs[0][k], runs[1][k]), (tau, k)
        ref = orc.simulate(net, kin, dt=0.01, cell_num=N, n_steps=steps, seed=7, population=pop, tauleap=tau)
        assert abs(runs[0]["V"].mean() / ref["V"].mean() - 1.0) < 0.005, tau
        for k in ("M", "P"):
            mg, mr = runs[0][k].mean(1), ref[k].mean(1)
            assert np.all(np.abs(mg - mr) <= np.maximum(0.03 * mr, 1.0)), (tau, k)


def test_batch_and_server_with_tables_beyond_shared_memory(pkg):
    """A batch takes such a network on the tensor path beside register-path networks (each
    network's result equals its single run); the server, which runs the register path only,
    refuses it at submission."""
    nets = [_unregulated(pkg, 12, 1), _dense_wide(pkg), _unregulated(pkg, 40, 3)]
    kin = pkg.WORKLOAD_KINETICS
    cells = [90, 64, 50]
    for alg in (pkg.CLE(0.01), pkg.BinomialTauLeap(0.01)):
        outs = pkg.simulate_gpu_batch(nets, alg, kin, cell_num=cells, T=0.5, readout="both", seed=6, stream=2)
        for b, net in enumerate(nets):
            single = pkg.simulate(net, alg, kin, cell_num=cells[b], T=0.5, readout="both", seed=6, stream=2 + b)
            assert np.array_equal(outs[b], single), (type(alg).__name__, b)
    server = pkg.Server()
    try:
        with pytest.raises(pkg.ScrnaError):
            server.submit(pkg.NetHandle(_dense_wide(pkg)), pkg.CLE(0.01), kin, cell_num=16, T=0.1)
    finally:
        server.close()
