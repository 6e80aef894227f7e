"""GPU test of scrna_cle_simulate_noalloc, the entry point for callers that cannot
allocate device memory while they run a simulation (their allocator is owned by
another component, or cudaMalloc would stall a serving loop).  It must give the
same results as the regular entry point scrna_cle_simulate on the same inputs,
on consecutive calls that reuse its one device-resident working array.

Kept in its own file, collected last, so a failure here comes after every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 2e-3  # the trajectory tolerance of the GPU parity tests; counts are compared exactly


def _run_noalloc(pkg, ctx, handle, kin, pop, cap, opts, N, G):
    import torch
    from scrna_b200 import api
    dev = torch.device("cuda", ctx.device)
    d_out = torch.empty(N * G, dtype=torch.float64, device=dev)
    d_counts = torch.empty(N * G, dtype=torch.int32, device=dev)
    d_eff = torch.empty(N, dtype=torch.float64, device=dev)
    k, p, c = api._kin(kin), api._pop(pop), api._cap(cap)
    rc = ctx.lib.scrna_cle_simulate_noalloc(ctx.h, handle.h, C.byref(k), C.byref(p) if p else None,
                                            C.byref(c) if c else None, C.byref(opts),
                                            C.c_void_p(d_out.data_ptr()), C.c_void_p(d_counts.data_ptr()),
                                            C.c_void_p(d_eff.data_ptr()))
    pkg._lib.check(rc)
    ctx.synchronize()
    torch.cuda.synchronize()
    out = d_out.cpu().numpy().reshape(G, N).T
    counts = d_counts.cpu().numpy().reshape(G, N).T
    return out, counts, d_eff.cpu().numpy()


def test_noalloc_matches_regular_entry_point_twice(pkg):
    from scrna_b200 import api
    ctx = pkg.default_context()
    net = pkg.sample_network(6, seed=21, bursty=True)
    kin = pkg.WORKLOAD_KINETICS
    N, G = 500, net.G
    handle = pkg.NetHandle(net, ctx)
    cap = pkg.CaptureModel(efficiency=0.2, efficiency_std=0.5, readout="mrna")
    for seed, partition in ((11, "binomial"), (12, "halve")):
        pop = pkg.PopulationConfig(cell_num=N, growth_rate=0.7, V_div=2.0, V_init=(1.0, 2.0),
                                   div_check_interval=10, partition=partition)
        opts = api._opts(pkg.CLE(0.01), T=3.0, cell_num=N, readout="mrna", seed=seed, stream=0,
                         precision="fp32", path="auto", n_steps=0, cell_offset=0)
        got, got_counts, got_eff = _run_noalloc(pkg, ctx, handle, kin, pop, cap, opts, N, G)
        want, want_counts, want_eff = pkg.simulate(net, pkg.CLE(0.01), kin, population=pop, T=3.0,
                                                   readout="mrna", seed=seed, capture=cap, ctx=ctx)
        err = np.max(np.abs(got - want) / np.maximum(np.abs(want), 1.0))
        assert err <= RTOL, (seed, err)
        assert np.array_equal(got_counts, want_counts)
        assert np.array_equal(got_eff, want_eff)


def test_noalloc_plain_run_after_population_runs(pkg):
    """Without population or capture (one launch, readout of both species), twice in a row
    after the population runs above: leftovers of earlier calls in the shared array do not
    leak into the result.  The second call maps no device memory (the first may still load
    the kernel's code module, which CUDA loads lazily at a kernel's first launch)."""
    import torch
    from scrna_b200 import api
    ctx = pkg.default_context()
    net = pkg.sample_network(9, seed=5, bursty=True)
    kin = pkg.WORKLOAD_KINETICS
    N, G = 777, net.G
    handle = pkg.NetHandle(net, ctx)
    opts = api._opts(pkg.CLE(0.01), T=2.0, cell_num=N, readout="both", seed=3, stream=2,
                     precision="fp32", path="auto", n_steps=0, cell_offset=0)
    want = pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=N, T=2.0, readout="both", seed=3, stream=2, ctx=ctx)
    dev = torch.device("cuda", ctx.device)
    d_out = torch.empty(N * 2 * G, dtype=torch.float64, device=dev)
    k = api._kin(kin)
    torch.cuda.synchronize()
    for i in range(2):
        free0 = torch.cuda.mem_get_info(dev)[0]
        rc = ctx.lib.scrna_cle_simulate_noalloc(ctx.h, handle.h, C.byref(k), None, None, C.byref(opts),
                                                C.c_void_p(d_out.data_ptr()), None, None)
        pkg._lib.check(rc)
        ctx.synchronize()
        if i == 1:
            assert torch.cuda.mem_get_info(dev)[0] == free0
        got = d_out.cpu().numpy().reshape(2 * G, N).T
        err = np.max(np.abs(got - want) / np.maximum(np.abs(want), 1.0))
        assert err <= RTOL, err


def test_noalloc_rejects_oversized_runs(pkg):
    from scrna_b200 import api
    ctx = pkg.default_context()
    net = pkg.sample_network(10, seed=1)
    handle = pkg.NetHandle(net, ctx)
    opts = api._opts(pkg.CLE(0.01), T=1.0, cell_num=100000, readout="protein", seed=0, stream=0,
                     precision="fp32", path="auto", n_steps=0, cell_offset=0)
    import torch
    k = api._kin(pkg.WORKLOAD_KINETICS)
    d_out = torch.zeros(100000 * net.G, dtype=torch.float64, device=torch.device("cuda", ctx.device))
    rc = ctx.lib.scrna_cle_simulate_noalloc(ctx.h, handle.h, C.byref(k), None, None, C.byref(opts),
                                            C.c_void_p(d_out.data_ptr()), None, None)
    assert rc == -1
    assert b"too large" in ctx.lib.scrna_last_error()
    opts = api._opts(pkg.CLE(0.01), T=1.0, cell_num=100, readout="protein", seed=0, stream=0,
                     precision="fp32", path="tensor", n_steps=0, cell_offset=0)
    rc = ctx.lib.scrna_cle_simulate_noalloc(ctx.h, handle.h, C.byref(k), None, None, C.byref(opts),
                                            C.c_void_p(d_out.data_ptr()), None, None)
    assert rc == -6
