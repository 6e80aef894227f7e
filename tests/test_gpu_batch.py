"""GPU batch path (scrna_cle_simulate_batch) against the FP64 oracle directly, through the
C ABI: networks of uneven G and cell counts, some with Moran populations, and per-network
kinetics (ext/SyntheticscRNAseqCUDAExt.jl:689-720 passes one KineticParams per network).

Tolerances as in the parity tests: trajectories |gpu - oracle| <= RTOL * max(|oracle|, 1)
with RTOL = 2e-3; with a binomial partition at division, FP32 and FP64 values that straddle
k + 1/2 can round to different counts, so there fewer than 1 % of entries may differ by more.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 2e-3


def _rel(got, ref):
    return np.abs(np.asarray(got, np.float64) - ref) / np.maximum(np.abs(ref), 1.0)


def _oracle_both(orc, net, kin, *, dt, N, steps, seed, stream, pop=None):
    r = orc.simulate(net, kin, dt=dt, cell_num=N, n_steps=steps, seed=seed, stream=stream, population=pop)
    return np.hstack([r["M"].T, r["P"].T])


def test_uneven_batch_with_populations_vs_oracle(pkg, orc):
    rng = np.random.default_rng(7)
    kin = pkg.WORKLOAD_KINETICS
    nets, cells, pops = [], [], []
    for b in range(10):
        G = int(rng.choice([1, 3, 6, 11, 24, 45, 90]))
        nets.append(pkg.sample_network(G, seed=300 + b, bursty=bool(b % 3 != 1)))
        N = int(rng.integers(30, 400))
        cells.append(N)
        pops.append(pkg.PopulationConfig(cell_num=N, growth_rate=0.7, V_div=2.0, V_init=(1.0, 2.0),
                                         div_check_interval=10, partition="halve" if b % 4 == 1 else "binomial",
                                         exclude_mother=bool(b % 2)) if b % 2 else None)
    T, dt, seed, stream = 1.5, 0.01, 13, 40
    steps = pkg.n_steps(T, dt)
    outs = pkg.simulate_gpu_batch(nets, pkg.CLE(dt), kin, cell_num=cells, T=T, readout="both", seed=seed,
                                  stream=stream, populations=pops)
    for b, net in enumerate(nets):
        want = _oracle_both(orc, net, kin, dt=dt, N=cells[b], steps=steps, seed=seed, stream=stream + b, pop=pops[b])
        err = _rel(outs[b], want)
        if pops[b] is not None and pops[b].partition == "binomial":
            assert np.mean(err > RTOL) < 0.01, b
        else:
            assert err.max() < RTOL, (b, err.max())


def test_batch_per_network_kinetics(pkg, orc):
    """n_kins = B: each network runs with its own KineticParams; equal to single runs bit for
    bit and to the oracle within RTOL."""
    nets = [pkg.sample_network(G, seed=400 + G, bursty=bool(G % 2)) for G in (4, 9, 16, 33)]
    kins = [pkg.KineticParams(k_t=5.0, K_d=10.0, n=2.0, mu_m=1.0, mu_p=0.2),
            pkg.KineticParams(k_t=2.0, K_d=20.0, n=3.0, mu_m=0.5, mu_p=0.3),
            pkg.KineticParams(k_t=8.0, K_d=15.0, n=2.0, mu_m=1.5, mu_p=0.1, dilution=0.05),
            pkg.KineticParams(k_t=4.0, K_d=12.0, n=2.5, mu_m=0.8, mu_p=0.25)]
    cells = [123, 257, 64, 300]
    T, dt, seed, stream = 2.0, 0.01, 21, 7
    outs = pkg.simulate_gpu_batch(nets, pkg.CLE(dt), kins, cell_num=cells, T=T, readout="both", seed=seed,
                                  stream=stream)
    for b, net in enumerate(nets):
        single = pkg.simulate(net, pkg.CLE(dt), kins[b], cell_num=cells[b], T=T, readout="both", seed=seed,
                              stream=stream + b)
        assert np.array_equal(outs[b], single), b
        want = _oracle_both(orc, net, kins[b], dt=dt, N=cells[b], steps=pkg.n_steps(T, dt), seed=seed,
                            stream=stream + b)
        assert _rel(outs[b], want).max() < RTOL, b
    # the kinetics really differ per network: the shared-kinetics batch gives other results
    shared = pkg.simulate_gpu_batch(nets, pkg.CLE(dt), kins[0], cell_num=cells, T=T, readout="both", seed=seed,
                                    stream=stream)
    assert np.array_equal(shared[0], outs[0]) and not np.array_equal(shared[1], outs[1])


def test_sharded_batch_equals_one_batch(pkg):
    """simulate_gpu_batch_sharded over two contexts (here both on one GPU; normally one per
    GPU): whole networks in contiguous ranges, each keeping its Philox stream, so readouts
    and captured counts equal one simulate_gpu_batch call's bit for bit (populations,
    per-network kinetics and capture included)."""
    rng = np.random.default_rng(11)
    nets, cells, pops, kins = [], [], [], []
    for b in range(7):
        G = int(rng.choice([3, 8, 20, 45, 90]))
        nets.append(pkg.sample_network(G, seed=500 + b, bursty=bool(b % 2)))
        N = int(rng.integers(40, 300))
        cells.append(N)
        pops.append(pkg.PopulationConfig(cell_num=N, growth_rate=0.7, V_div=2.0, V_init=(1.0, 2.0),
                                         div_check_interval=10) if b % 3 == 0 else None)
        kins.append(pkg.KineticParams(k_t=3.0 + b, K_d=10.0, n=2.0, mu_m=0.8, mu_p=0.2))
    cap = pkg.CaptureModel(efficiency=0.3, efficiency_std=0.4, readout="protein")
    kw = dict(cell_num=cells, T=1.2, readout="both", seed=17, stream=30, populations=pops, capture=cap)
    want_x, want_c = pkg.simulate_gpu_batch(nets, pkg.CLE(0.01), kins, **kw)
    ctxs = [pkg.Context(0), pkg.Context(0)]
    got_x, got_c = pkg.simulate_gpu_batch_sharded(nets, pkg.CLE(0.01), kins, contexts=ctxs, **kw)
    for c in ctxs:
        c.close()
    assert len(got_x) == len(nets)
    for b in range(len(nets)):
        assert np.array_equal(got_x[b], want_x[b]), b
        assert np.array_equal(got_c[b], want_c[b]), b


def test_concurrent_calls_on_two_contexts_of_one_gpu(pkg):
    """Two threads, each with its own context on the same GPU, run networks whose kernels need
    different amounts of dynamic shared memory, many times over.  The kernels' shared-memory
    limit is one attribute of the device's context, which both contexts share; the library only
    ever raises it, so no launch finds it set below its own size by the other thread.  Every
    result equals the same call made alone."""
    import threading
    kin = pkg.WORKLOAD_KINETICS
    jobs = [(pkg.sample_network(G, seed=900 + G, bursty=bool(G % 2)), G) for G in (12, 45, 90, 150)]
    want = {G: pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=200, T=0.3, readout="both", seed=G)
            for net, G in jobs}
    errors = []

    def worker(k):
        ctx = pkg.Context(0)
        try:
            for rep in range(12):
                net, G = jobs[(k + rep) % len(jobs)]
                got = pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=200, T=0.3, readout="both", seed=G, ctx=ctx)
                if not np.array_equal(got, want[G]):
                    errors.append((k, G, "differs"))
        except Exception as e:  # noqa: BLE001 (reported below)
            errors.append((k, repr(e)))
        finally:
            ctx.close()

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
