"""The autotuner on the GPU: every kernel variant it chooses between computes the same sums in
the same order, so tuned runs (measured, then read from the cache) equal untuned runs bit for
bit, for single runs with and without population and for a batch; the measurement happens
once per network shape, for runs of at least 5e8 cell-gene-steps, and later contexts read the
choice from the cache file."""
import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _nets(pkg):
    return [(pkg.sample_network(10, seed=1, bursty=True), 3000), (pkg.sample_network(40, seed=2), 777),
            (pkg.sample_network(150, seed=3, bursty=True), 500), (pkg.sample_network(300, seed=4), 257)]


MIN_UNITS = 5e8  # a run shorter than this (cell-gene-steps) is not worth measuring for


def _steps(net, N):
    return int(MIN_UNITS // (net.G * N)) + 1


def test_tuned_equals_untuned(pkg, tmp_path):
    kin = pkg.WORKLOAD_KINETICS
    cache = tmp_path / "autotune.json"
    plain = pkg.Context(0)
    plain.set_autotune(0)
    tuned = pkg.Context(0)
    tuned.set_autotune(1, str(cache))
    for net, N in _nets(pkg):
        kw = dict(cell_num=N, T=0.0, n_steps=_steps(net, N), readout="both", seed=3)
        want = pkg.simulate(net, pkg.CLE(0.01), kin, ctx=plain, **kw)
        l0 = tuned.launches
        got = pkg.simulate(net, pkg.CLE(0.01), kin, ctx=tuned, **kw)
        assert tuned.launches - l0 > 1  # measured: the candidates ran before the run itself
        assert tuned.last_kernel_choice()["found"] == 1
        assert np.array_equal(got, want)
        l0 = tuned.launches
        again = pkg.simulate(net, pkg.CLE(0.01), kin, ctx=tuned, **kw)
        assert tuned.launches - l0 == 1  # the shape is known: one launch, no measurement
        assert np.array_equal(again, want)
    entries = json.load(open(cache))["entries"]
    assert len(entries) == 4
    # a new context reads the file: no measurement, same results
    fresh = pkg.Context(0)
    fresh.set_autotune(2, str(cache))
    net, N = _nets(pkg)[0]
    kw = dict(cell_num=N, T=0.0, n_steps=_steps(net, N), readout="both", seed=3)
    l0 = fresh.launches
    got = pkg.simulate(net, pkg.CLE(0.01), kin, ctx=fresh, **kw)
    # the run plus, on a new context, the one-time fill of its switch-time table; no measurement
    assert fresh.launches - l0 <= 2 and fresh.last_kernel_choice()["found"] == 1
    assert np.array_equal(got, pkg.simulate(net, pkg.CLE(0.01), kin, ctx=plain, **kw))
    for c in (plain, tuned, fresh):
        c.close()


def test_short_runs_take_the_static_choice(pkg, tmp_path):
    """A run of fewer than 5e8 cell-gene-steps measures nothing and stores nothing: the
    candidates' measurement (and their kernels' first loads) would cost more than the run."""
    cache = tmp_path / "autotune.json"
    ctx = pkg.Context(0)
    ctx.set_autotune(1, str(cache))
    net = pkg.sample_network(10, seed=1, bursty=True)
    pkg.simulate(net, pkg.CLE(0.01), pkg.WORKLOAD_KINETICS, cell_num=50, T=0.1, seed=1, ctx=ctx)  # table fill
    l0 = ctx.launches
    pkg.simulate(net, pkg.CLE(0.01), pkg.WORKLOAD_KINETICS, cell_num=5000, T=10.0, seed=1, ctx=ctx)
    assert ctx.launches - l0 == 1 and ctx.last_kernel_choice()["found"] == 0
    assert not cache.exists() or json.load(open(cache))["entries"] == {}
    ctx.close()


def test_tuned_population_and_batch_equal_untuned(pkg, tmp_path):
    kin = pkg.WORKLOAD_KINETICS
    plain = pkg.Context(0)
    plain.set_autotune(0)
    tuned = pkg.Context(0)
    tuned.set_autotune(1, str(tmp_path / "autotune.json"))
    nets = [n for n, _ in _nets(pkg)]
    pops = [pkg.PopulationConfig(cell_num=400 + 100 * i, growth_rate=0.7, V_div=2.0, V_init=(1.0, 2.0),
                                 div_check_interval=10) if i % 2 else None for i in range(len(nets))]
    cells = [600, 500, 300, 700]
    for net, pop, N in zip(nets, pops, cells):
        a = pkg.simulate(net, pkg.CLE(0.01), kin, population=pop, cell_num=N, T=0.5, readout="both", seed=8, ctx=plain)
        b = pkg.simulate(net, pkg.CLE(0.01), kin, population=pop, cell_num=N, T=0.5, readout="both", seed=8, ctx=tuned)
        assert np.array_equal(a, b)
    a = pkg.simulate_gpu_batch(nets, pkg.CLE(0.01), kin, cell_num=cells, T=0.5, populations=pops, readout="both",
                               seed=5, ctx=plain)
    b = pkg.simulate_gpu_batch(nets, pkg.CLE(0.01), kin, cell_num=cells, T=0.5, populations=pops, readout="both",
                               seed=5, ctx=tuned)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    plain.close()
    tuned.close()


def test_tuned_tensor_tile_equals_default(pkg, tmp_path):
    """The fused tensor-core step's tile width (160, 192 or 224 genes) changes which genes share a
    tile, not the order of the contraction over K, so a tuned run equals the default width's."""
    kin = pkg.WORKLOAD_KINETICS
    plain = pkg.Context(0)
    plain.set_autotune(0)
    tuned = pkg.Context(0)
    tuned.set_autotune(1, str(tmp_path / "autotune.json"))
    for G, N in ((300, 700), (520, 333)):
        net = pkg.dense_network(G, seed=G, density=0.1, n_coop=4, n_redun=4)
        a = pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=N, T=0.3, readout="both", seed=2, path="tensor", ctx=plain)
        b = pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=N, T=0.3, readout="both", seed=2, path="tensor", ctx=tuned)
        choice = tuned.last_kernel_choice()
        assert choice["kernel"] == 2 and choice["found"] == 1 and choice["genes_per_lane"] in (160, 192, 224)
        assert np.array_equal(a, b), (G, choice)
    plain.close()
    tuned.close()
