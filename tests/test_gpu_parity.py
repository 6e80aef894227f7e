"""GPU parity: the CUDA library against the FP64 CPU oracle on the same Philox
increments, through the C ABI.

Tolerances (FP32 state and fast special functions against FP64):
  trajectories after <= 400 steps: |gpu - oracle| <= RTOL * max(|oracle|, 1) with RTOL = 2e-3;
  promoter states, division schedule (volumes) and capture counts: bit-exact;
  FP64 baseline kernel: RTOL64 = 1e-9.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 2e-3
RTOL64 = 1e-9


def _rel(got, ref):
    return float(np.max(np.abs(np.asarray(got, np.float64) - ref) / np.maximum(np.abs(ref), 1.0)))


def _device_run(pkg, net, kin, *, N, steps, seed=0, dt=0.01, readout="both", **kw):
    run = pkg.DeviceRun(net, pkg.CLE(dt), kin, cell_num=N, T=0.0, n_steps=steps, readout=readout,
                        seed=seed, **kw)
    run.launch()
    return run


def test_device_philox_known_answers(pkg, ctx):
    ctr = np.array([[0, 0, 0, 0], [0xFFFFFFFF] * 4, [0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344]],
                   dtype=np.uint32)
    # the published vectors use different keys per row; run each row with its key
    keys = [[0, 0], [0xFFFFFFFF] * 2, [0xA4093822, 0x299F31D0]]
    want = [[0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8],
            [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD],
            [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]]
    for c, k, w in zip(ctr, keys, want):
        assert pkg.debug_philox(c[None, :], k, ctx)[0].tolist() == w


def test_device_philox_matches_oracle_random(pkg, ctx, orc):
    rng = np.random.default_rng(0)
    ctr = rng.integers(0, 2**32, size=(257, 4), dtype=np.uint64).astype(np.uint32)
    key = [0x12345678, 0x9ABCDEF0]
    got = pkg.debug_philox(ctr, key, ctx)
    want = np.array([orc.philox(c, key) for c in ctr])
    assert np.array_equal(got, want)


@pytest.mark.parametrize("G,N,steps", [(1, 64, 300), (2, 33, 200), (5, 100, 400)])
def test_constitutive_trajectories(pkg, orc, G, N, steps):
    net = pkg.GeneNetwork(G, np.linspace(2.0, 9.0, G), np.zeros((G, G)))
    kin = pkg.KineticParams(k_t=2.0, K_d=50.0, n=2.0, mu_m=0.1, mu_p=0.2)
    run = _device_run(pkg, net, kin, N=N, steps=steps, seed=42, dt=0.1)
    got = run.read_raw()
    ref = orc.simulate(net, kin, dt=0.1, cell_num=N, n_steps=steps, seed=42)
    assert _rel(got["M"], ref["M"]) < RTOL
    assert _rel(got["P"], ref["P"]) < RTOL


@pytest.mark.parametrize("G,seed", [(5, 0), (10, 3), (17, 5), (40, 8)])
def test_regulated_bursty_trajectories(pkg, orc, G, seed):
    """Additive + cooperative + redundant regulation and telegraph switching."""
    net = pkg.sample_network(G, seed=seed, bursty=True)
    assert net.cooperative or net.redundant
    kin = pkg.WORKLOAD_KINETICS
    N, steps = 70, 300
    run = _device_run(pkg, net, kin, N=N, steps=steps, seed=seed + 1)
    got = run.read_raw()
    ref = orc.simulate(net, kin, dt=0.01, cell_num=N, n_steps=steps, seed=seed + 1)
    assert np.array_equal(got["prom"], ref["prom"])
    assert _rel(got["M"], ref["M"]) < RTOL
    assert _rel(got["P"], ref["P"]) < RTOL


def test_generic_hill_exponent(pkg, orc):
    net = pkg.sample_network(8, seed=12)
    for n in (3.0, 2.5):
        kin = pkg.KineticParams(k_t=5.0, K_d=10.0, n=n, mu_m=1.0, mu_p=0.2)
        run = _device_run(pkg, net, kin, N=40, steps=200, seed=2)
        got = run.read_raw()
        ref = orc.simulate(net, kin, dt=0.01, cell_num=40, n_steps=200, seed=2)
        assert _rel(got["P"], ref["P"]) < RTOL


def test_readout_layouts(pkg):
    net = pkg.sample_network(6, seed=4)
    kin = pkg.WORKLOAD_KINETICS
    both = pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=50, T=1.0, readout="both", seed=3)
    m = pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=50, T=1.0, readout="mrna", seed=3)
    p = pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=50, T=1.0, readout="protein", seed=3)
    assert both.shape == (50, 12) and m.shape == (50, 6) and p.shape == (50, 6)
    assert np.array_equal(both[:, :6], m) and np.array_equal(both[:, 6:], p)


def test_fp64_baseline_matches_oracle(pkg, orc):
    net = pkg.sample_network(10, seed=3, bursty=True)
    kin = pkg.WORKLOAD_KINETICS
    N, steps = 90, 250
    run = _device_run(pkg, net, kin, N=N, steps=steps, seed=9, precision="fp64_plain")
    got = run.read_raw()
    ref = orc.simulate(net, kin, dt=0.01, cell_num=N, n_steps=steps, seed=9)
    assert np.array_equal(got["prom"], ref["prom"])
    assert _rel(got["M"], ref["M"]) < RTOL64
    assert _rel(got["P"], ref["P"]) < RTOL64


def test_capture_bit_exact(pkg, orc):
    net = pkg.sample_network(10, seed=1, bursty=True)
    kin = pkg.WORKLOAD_KINETICS
    cap = pkg.CaptureModel(efficiency=0.1, efficiency_std=0.5, readout="mrna", mean_correction=False)
    N = 500
    X, counts, eff = pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=N, T=3.0, readout="mrna", seed=17,
                                  capture=cap)
    want = orc.capture_counts(X.T, eff, seed=17)
    assert np.array_equal(counts.T, want)
    eff_ref = orc.capture_efficiency(N, 0.1, 0.5, 0, seed=17)
    assert np.max(np.abs(eff - eff_ref) / eff_ref) < 1e-12


def test_capture_protein_large_counts_bit_exact(pkg, orc):
    """Counts above one 512-trial chunk and efficiencies above 1/2 (flip branch)."""
    rng = np.random.default_rng(5)
    X = np.round(rng.random((300, 7)) * 3000.0)
    cap = pkg.CaptureModel(efficiency=0.6, efficiency_std=0.4, readout="protein")
    Y, eff = pkg.apply_capture(X, cap, seed=23, return_efficiencies=True)
    want = orc.capture_counts(np.ascontiguousarray(X.T), eff, seed=23)
    assert np.array_equal(Y.T, want)
    assert np.all(Y <= X) and np.all(Y >= 0)
    assert np.any(eff > 0.5)


@pytest.mark.parametrize("partition", ["halve", "binomial"])
@pytest.mark.parametrize("exclude_mother", [True, False])
def test_population_division(pkg, orc, partition, exclude_mother):
    net = pkg.sample_network(6, seed=21, bursty=True)
    kin = pkg.WORKLOAD_KINETICS
    N, steps = 150, 320
    pop = pkg.PopulationConfig(cell_num=N, growth_rate=0.7, V_div=2.0, V_init=(1.0, 2.0),
                               div_check_interval=10, partition=partition,
                               exclude_mother=exclude_mother)
    run = _device_run(pkg, net, kin, N=N, steps=steps, seed=31, population=pop)
    got = run.read_raw()
    ref = orc.simulate(net, kin, dt=0.01, cell_num=N, n_steps=steps, seed=31, population=pop)
    assert np.array_equal(got["V"], ref["V"])  # identical division schedule and Moran placements
    if partition == "halve":
        assert np.array_equal(got["prom"], ref["prom"])
        assert _rel(got["M"], ref["M"]) < RTOL
        assert _rel(got["P"], ref["P"]) < RTOL
    else:
        # rounding of FP32 vs FP64 values straddling k + 1/2 can move a count by one
        err = np.abs(got["P"] - ref["P"]) / np.maximum(np.abs(ref["P"]), 1.0)
        assert np.mean(err > RTOL) < 0.01


def test_population_final_check_step(pkg, orc):
    """n_steps a multiple of the check interval: the last division is applied before readout."""
    net = pkg.sample_network(4, seed=2)
    kin = pkg.WORKLOAD_KINETICS
    pop = pkg.PopulationConfig(cell_num=64, growth_rate=0.7, V_div=2.0, V_init=(1.0, 2.0),
                               div_check_interval=10, partition="halve")
    run = _device_run(pkg, net, kin, N=64, steps=100, seed=4, population=pop)
    got = run.read_raw()
    ref = orc.simulate(net, kin, dt=0.01, cell_num=64, n_steps=100, seed=4, population=pop)
    assert np.array_equal(got["V"], ref["V"])
    assert _rel(got["P"], ref["P"]) < RTOL


def test_batch_equals_single_runs(pkg):
    nets = [pkg.sample_network(G, seed=G) for G in (3, 11, 29)]
    kin = pkg.WORKLOAD_KINETICS
    cells = [40, 77, 129]
    outs = pkg.simulate_gpu_batch(nets, pkg.CLE(0.01), kin, cell_num=cells, T=1.0, readout="both", seed=5,
                                  stream=10)
    for b, (n, N) in enumerate(zip(nets, cells)):
        single = pkg.simulate(n, pkg.CLE(0.01), kin, cell_num=N, T=1.0, readout="both", seed=5, stream=10 + b)
        assert np.array_equal(outs[b], single)


def test_cell_sharding_is_exact(pkg):
    """Cells keyed by global index: two half runs with cell offsets equal one full run."""
    net = pkg.sample_network(10, seed=3, bursty=True)
    kin = pkg.WORKLOAD_KINETICS
    full = pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=100, T=1.0, seed=8)
    a = pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=37, T=1.0, seed=8)
    b = pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=63, T=1.0, seed=8, cell_offset=37)
    assert np.array_equal(full, np.vstack([a, b]))


def test_edge_cases(pkg, orc):
    kin = pkg.WORKLOAD_KINETICS
    net = pkg.GeneNetwork(1, [3.0], np.zeros((1, 1)))
    one = pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=1, T=0.5, seed=1, readout="both")
    ref = orc.simulate(net, kin, dt=0.01, T=0.5, cell_num=1, seed=1)
    assert one.shape == (1, 2) and _rel(one[:, 1], ref["P"][0]) < RTOL
    zero = pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=10, T=0.0, readout="both")
    m_ss, p_ss = pkg.steady_state(net, kin)
    assert np.all(zero[:, 0] == math.ceil(m_ss[0])) and np.all(zero[:, 1] == math.ceil(p_ss[0]))
    with pytest.raises(pkg.ScrnaError):
        pkg.simulate(net, pkg.CLE(-0.1), kin, cell_num=10, T=1.0)
    with pytest.raises(pkg.ScrnaError):
        pkg.simulate(net, pkg.CLE(0.1), kin, cell_num=0, T=1.0)
    with pytest.raises(pkg.ScrnaError):
        pkg.simulate(net, pkg.CLE(0.1), kin, population=pkg.PopulationConfig(cell_num=1), T=1.0)


def test_gpu_two_stage_moments(pkg):
    """test/test_analytical_moments.jl:110-121 on the GPU path."""
    beta, mu_m, mu_p, k_t = 2.0, 0.1, 0.2, 1.0
    net = pkg.GeneNetwork(1, [beta], np.zeros((1, 1)))
    kin = pkg.KineticParams(k_t=k_t, K_d=50.0, n=2.0, mu_m=mu_m, mu_p=mu_p)
    Y = pkg.simulate(net, pkg.CLE(0.1), kin, cell_num=10000, T=500.0, readout="both", seed=42)
    m, p = Y[:, 0], Y[:, 1]
    assert abs(m.mean() / (beta / mu_m) - 1) < 0.05
    assert abs(m.var(ddof=1) / (beta / mu_m) - 1) < 0.20
    assert abs(p.mean() / (k_t * beta / (mu_m * mu_p)) - 1) < 0.05
    assert abs((p.var(ddof=1) / p.mean()) / (1 + k_t / (mu_m + mu_p)) - 1) < 0.20


def test_gpu_vs_cpu_ensemble(pkg, orc):
    """test/test_gpu_parity.jl:12-30: GPU CLE vs CPU CLE, mean < 5%, variance < 15%."""
    net = pkg.GeneNetwork(1, [5.0], np.zeros((1, 1)))
    kin = pkg.KineticParams(k_t=2.0, K_d=50.0, n=2.0, mu_m=0.1, mu_p=0.2)
    Yg = pkg.simulate(net, pkg.CLE(0.1), kin, cell_num=5000, T=200.0, readout="protein", seed=42)
    Yc = orc.simulate(net, kin, dt=0.1, T=200.0, cell_num=5000, seed=7)["P"][0]
    assert abs(Yg.mean() - Yc.mean()) / Yc.mean() < 0.05
    assert abs(Yg.var() - Yc.var()) / Yc.var() < 0.15


@pytest.mark.parametrize("G,bursty,seed", [(1, False, 1), (2, True, 2), (3, True, 3), (5, False, 4),
                                           (10, True, 5), (13, True, 6), (17, False, 7), (32, True, 8),
                                           (40, True, 9), (77, False, 10), (150, True, 11), (300, False, 12),
                                           (500, True, 13)])
def test_warp_and_block_kernels_identical(pkg, G, bursty, seed):
    """The lane-per-gene-unit kernel (cells within a warp, or spanning up to 8 warps with a
    named barrier) and the block-tile kernel compute the same sums in the same order on the
    same increments: their results are bit-identical."""
    net = pkg.sample_network(G, seed=seed, bursty=bursty)
    kin = pkg.WORKLOAD_KINETICS
    N = 257
    outs = []
    for path in ("warp", "block"):
        run = _device_run(pkg, net, kin, N=N, steps=150, seed=seed, path=path)
        outs.append(run.read_raw())
    for k in ("M", "P", "prom"):
        assert np.array_equal(outs[0][k], outs[1][k]), k


def _terms_per_target(net):
    cnt = {}
    for e in list(net.cooperative) + list(net.redundant):
        cnt[e.target] = cnt.get(e.target, 0) + 1
    return max(cnt.values()) if cnt else 0


@pytest.mark.parametrize("G,seed,n_coop,n_redun,n_src", [(12, 21, (3, 4), (3, 4), (2, 3)),   # 1 term, 3 sources
                                                         (8, 0, (2, 3), (2, 3), (2, 3)),      # 2 terms
                                                         (10, 1, (3, 3), (3, 3), (2, 3)),     # 2 terms
                                                         (14, 1, (5, 6), (5, 6), (2, 3))])    # 3 terms
def test_warp_kernel_padded_terms_identical(pkg, G, seed, n_coop, n_redun, n_src):
    """Networks with several cooperative / redundant terms per gene over 2-3 sources: the
    warp kernel evaluates each term once per cell into its own activation slot (padded
    sources read constant 0/1 slots) and adds it as an in-edge of its target; the sums
    equal the block kernel's bit for bit."""
    net = pkg.sample_network(G, seed=seed, bursty=True, n_coop_range=n_coop, n_redun_range=n_redun,
                             n_sources_range=n_src)
    assert 1 <= _terms_per_target(net) <= 4
    kin = pkg.WORKLOAD_KINETICS
    outs = [_device_run(pkg, net, kin, N=301, steps=120, seed=seed, path=p).read_raw() for p in ("warp", "block")]
    for k in ("M", "P", "prom"):
        assert np.array_equal(outs[0][k], outs[1][k]), k


def test_warp_kernel_rejects_long_terms(pkg):
    """A cooperative term over 4 sources is beyond the warp kernel's term evaluation:
    asking for that kernel fails with a clear error, the automatic choice runs the block
    kernel."""
    net = pkg.sample_network(8, seed=3, n_coop_range=(1, 1), n_redun_range=(0, 0), n_sources_range=(4, 4))
    assert any(len(e.sources) == 4 for e in net.cooperative)
    kin = pkg.WORKLOAD_KINETICS
    with pytest.raises(pkg.ScrnaError):
        _device_run(pkg, net, kin, N=64, steps=10, seed=1, path="warp")
    a = _device_run(pkg, net, kin, N=64, steps=10, seed=1, path="auto").read_raw()
    b = _device_run(pkg, net, kin, N=64, steps=10, seed=1, path="block").read_raw()
    assert np.array_equal(a["P"], b["P"])


@pytest.mark.parametrize("partition,G", [("halve", 7), ("binomial", 7), ("binomial", 120)])
def test_warp_and_block_kernels_identical_population(pkg, partition, G):
    net = pkg.sample_network(G, seed=9, bursty=True)
    kin = pkg.WORKLOAD_KINETICS
    pop = pkg.PopulationConfig(cell_num=300, growth_rate=0.7, V_div=2.0, V_init=(1.0, 2.0),
                               div_check_interval=10, partition=partition)
    outs = []
    for path in ("warp", "block"):
        run = _device_run(pkg, net, kin, N=300, steps=250, seed=3, population=pop, path=path)
        outs.append(run.read_raw())
    for k in ("M", "P", "prom", "V"):
        assert np.array_equal(outs[0][k], outs[1][k]), k


def test_batch_mixed_population_equals_single_runs(pkg):
    """Uneven networks, some with Moran populations, in one batch call (persistent launches
    per kernel group, captured population chunks) give the same results as single runs."""
    rng = np.random.default_rng(0)
    kin = pkg.WORKLOAD_KINETICS
    nets, cells, pops = [], [], []
    for b in range(14):
        G = int(rng.choice([2, 5, 9, 16, 31, 40, 77]))
        nets.append(pkg.sample_network(G, seed=100 + b, bursty=bool(b % 3 == 0)))
        N = int(rng.integers(40, 900))
        cells.append(N)
        pops.append(pkg.PopulationConfig(cell_num=N, growth_rate=0.7, V_div=2.0, V_init=(1.0, 2.0),
                                         div_check_interval=10) if b % 2 else None)
    outs = pkg.simulate_gpu_batch(nets, pkg.CLE(0.01), kin, cell_num=cells, T=1.25, readout="both", seed=9,
                                  stream=3, populations=pops)
    for b in range(len(nets)):
        single = pkg.simulate(nets[b], pkg.CLE(0.01), kin, population=pops[b], cell_num=cells[b], T=1.25,
                              readout="both", seed=9, stream=3 + b)
        assert np.array_equal(outs[b], single), b


def test_pinned_result_arrays(pkg):
    """Results land in pooled page-locked blocks: live arrays are never reused, released ones
    are, and the values equal a copy into pageable memory (DeviceRun.read of the same run)."""
    from scrna_b200 import _pinned
    net = pkg.sample_network(9, seed=12, bursty=True)
    kin = pkg.WORKLOAD_KINETICS
    cap = pkg.CaptureModel(efficiency=0.3, efficiency_std=0.1, readout="protein")
    first = pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=300, T=2.0, seed=4, capture=cap)
    keep = [a.copy() for a in first]
    second = pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=300, T=2.0, seed=5, capture=cap)
    for a, b in zip(first, keep):  # the live first results were not overwritten
        assert np.array_equal(a, b)
    assert not np.array_equal(first[0], second[0])
    assert not _pinned._pool._disabled  # pinning works on a GPU box
    ptrs = {a.__array_interface__["data"][0] for a in first + second}
    assert len(ptrs) == 6
    del first, keep, second
    third = pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=300, T=2.0, seed=4, capture=cap)
    assert {a.__array_interface__["data"][0] for a in third} <= ptrs  # released blocks reused
    run = pkg.DeviceRun(net, pkg.CLE(0.01), kin, cell_num=300, T=2.0, seed=4, capture=cap)
    run.launch()
    X, counts, eff = run.read()
    assert np.array_equal(third[0], X) and np.array_equal(third[1], counts) and np.array_equal(third[2], eff)
    pageable = np.empty_like(X, order="F")
    pkg._lib.check(run.ctx.lib.scrna_state_read(run.ctx.h, run.st, pageable.ctypes.data, None, None))
    assert np.array_equal(pageable, X)
    assert third[0].flags["F_CONTIGUOUS"] and third[1].flags["F_CONTIGUOUS"]
    run.close()


def test_network_upload_cache(pkg):
    """simulate() reuses an uploaded network for the same content on the same context and
    uploads again after an in-place change: results equal those of an explicit handle."""
    ctx = pkg.Context(0)
    net = pkg.sample_network(8, seed=21, bursty=True)
    kin = pkg.WORKLOAD_KINETICS
    a = pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=64, T=1.0, seed=2, ctx=ctx)
    b = pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=64, T=1.0, seed=2, ctx=ctx)
    assert len(ctx._net_cache) == 1 and np.array_equal(a, b)
    net.basals[0] *= 3.0  # same object, new content
    c = pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=64, T=1.0, seed=2, ctx=ctx)
    ref = pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=64, T=1.0, seed=2, ctx=ctx,
                       handle=pkg.NetHandle(net, ctx))
    assert len(ctx._net_cache) == 2 and np.array_equal(c, ref) and not np.array_equal(a, c)
    ctx.close()
