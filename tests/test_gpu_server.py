"""GPU tests of the serving loop (continuous batching): results equal simulate() alone and
in any mix (bit-exact: same kernels, same increments, exact state round trips between
chunks), admission by device-memory budget, capture, cancellation."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WAIT_MS = 120000


def _nets(pkg):
    return [pkg.sample_network(G, seed=200 + G, bursty=bool(G % 2)) for G in (3, 8, 13, 24, 40, 97)]


def test_server_alone_equals_mixed_equals_simulate(pkg):
    kin = pkg.WORKLOAD_KINETICS
    nets = _nets(pkg)
    handles = [pkg.NetHandle(n) for n in nets]
    target = dict(cell_num=777, T=1.37, readout="both", seed=21, stream=5)
    want = pkg.simulate(nets[4], pkg.CLE(0.01), kin, **target)

    srv = pkg.Server(chunk_steps=37)
    t = srv.submit(handles[4], pkg.CLE(0.01), kin, **target)
    alone = srv.wait(t, WAIT_MS)[0]
    assert np.array_equal(alone, want)

    tickets = []
    for i, h in enumerate(handles):
        tickets.append(srv.submit(h, pkg.CLE(0.01), kin, cell_num=300 + 97 * i, T=0.5 + 0.3 * i, seed=i,
                                  stream=i, readout="protein"))
    t_mixed = srv.submit(handles[4], pkg.CLE(0.01), kin, **target)
    for i, h in enumerate(handles):
        tickets.append(srv.submit(h, pkg.CLE(0.01), kin, cell_num=200 + 31 * i, T=1.0, seed=50 + i, stream=9))
    mixed = srv.wait(t_mixed, WAIT_MS)[0]
    assert np.array_equal(mixed, want)
    for i, t in enumerate(tickets):
        out, _, _, lat = srv.wait(t, WAIT_MS)
        assert np.all(np.isfinite(out)) and lat >= 0.0
    st = srv.stats()
    assert st["completed"] == 2 + len(tickets) and st["failed"] == 0 and st["bytes_in_use"] == 0
    # the chunk trace accounts for every cell·gene·step and every group launch
    tr = srv.trace()
    assert sum(r["units"] for r in tr) == st["units_done"] and sum(r["groups"] for r in tr) == st["chunks"]
    assert all(r["t_end"] >= r["t_start"] >= 0.0 and r["requests"] >= 1 for r in tr)
    assert all(a["t_end"] <= b["t_start"] for a, b in zip(tr, tr[1:]))
    srv.close()


def test_server_capture_matches_simulate(pkg):
    kin = pkg.WORKLOAD_KINETICS
    net = pkg.sample_network(10, seed=1, bursty=True)
    cap = pkg.CaptureModel(efficiency=0.1, efficiency_std=0.5, readout="mrna", mean_correction=False)
    X, counts, eff = pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=500, T=2.0, readout="mrna", seed=3,
                                  capture=cap)
    srv = pkg.Server(chunk_steps=64)
    t = srv.submit(pkg.NetHandle(net), pkg.CLE(0.01), kin, cell_num=500, T=2.0, readout="mrna", seed=3,
                   capture=cap)
    X2, c2, e2, _ = srv.wait(t, WAIT_MS)
    assert np.array_equal(X, X2) and np.array_equal(counts, c2) and np.array_equal(eff, e2)
    srv.close()


def test_server_admission_budget_and_rejection(pkg):
    kin = pkg.WORKLOAD_KINETICS
    net = pkg.sample_network(20, seed=4)
    h = pkg.NetHandle(net)
    # footprint of a 2000-cell protein run is ~0.5 MB; a 1.2 MB budget admits two at a time
    srv = pkg.Server(hbm_budget_bytes=1_200_000, chunk_steps=50)
    ts = [srv.submit(h, pkg.CLE(0.01), kin, cell_num=2000, T=0.6, seed=s) for s in range(6)]
    outs = [srv.wait(t, WAIT_MS)[0] for t in ts]
    for s, o in enumerate(outs):
        assert np.array_equal(o, pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=2000, T=0.6, seed=s))
    big = srv.submit(h, pkg.CLE(0.01), kin, cell_num=200000, T=0.1)
    with pytest.raises(pkg.ScrnaError):
        srv.wait(big, WAIT_MS)
    srv.close()


def test_server_cancel(pkg):
    kin = pkg.WORKLOAD_KINETICS
    net = pkg.sample_network(30, seed=5)
    srv = pkg.Server(chunk_steps=20)
    t = srv.submit(pkg.NetHandle(net), pkg.CLE(0.01), kin, cell_num=20000, T=200.0)
    srv.cancel(t)
    with pytest.raises(pkg.ScrnaError):
        srv.wait(t, WAIT_MS)
    # the server keeps serving after a cancellation
    t2 = srv.submit(pkg.NetHandle(net), pkg.CLE(0.01), kin, cell_num=100, T=0.2)
    assert np.all(np.isfinite(srv.wait(t2, WAIT_MS)[0]))
    srv.close()


def test_server_pool_spreads_requests_and_matches_simulate(pkg):
    """Two servers (here on one GPU, normally one per device): requests go to the less
    loaded one, and every result equals simulate's."""
    kin = pkg.WORKLOAD_KINETICS
    nets = _nets(pkg)
    ctxs = [pkg.Context(0), pkg.Context(0)]
    pool = pkg.ServerPool(ctxs, chunk_steps=45)
    jobs = [(nets[i % len(nets)], dict(cell_num=150 + 60 * i, T=0.6 + 0.1 * i, readout="mrna", seed=70 + i, stream=i))
            for i in range(8)]
    tickets = [pool.submit(n, pkg.CLE(0.01), kin, **kw) for n, kw in jobs]
    assert {pool.server_of(t) for t in tickets} == {0, 1}
    for (n, kw), t in zip(jobs, tickets):
        got = pool.wait(t, WAIT_MS)[0]
        assert np.array_equal(got, pkg.simulate(n, pkg.CLE(0.01), kin, **kw))
    st = pool.stats()
    assert st["completed"] == len(jobs) and st["failed"] == 0 and pool.loads() == [0, 0]
    pool.close()
    for c in ctxs:
        c.close()


def test_cancel_queued_requests_then_keep_serving(pkg):
    """Requests cancelled while still queued leave the queue at once, so waiting on them (which
    frees them) cannot race the worker's admission; requests cancelled during admission are
    dropped at the next chunk boundary.  Repeated, with new requests submitted in between,
    every surviving request still completes with the result of a lone run."""
    kin = pkg.WORKLOAD_KINETICS
    net = pkg.sample_network(30, seed=5)
    h = pkg.NetHandle(net)
    want = pkg.simulate(net, pkg.CLE(0.01), kin, cell_num=150, T=0.3, readout="protein", seed=9)
    srv = pkg.Server(chunk_steps=10)
    for rep in range(6):
        doomed = [srv.submit(h, pkg.CLE(0.01), kin, cell_num=5000, T=20.0, seed=rep * 10 + k) for k in range(4)]
        keep = srv.submit(h, pkg.CLE(0.01), kin, cell_num=150, T=0.3, readout="protein", seed=9)
        for t in doomed:
            srv.cancel(t)
            with pytest.raises(pkg.ScrnaError):
                srv.wait(t, WAIT_MS)
        assert np.array_equal(srv.wait(keep, WAIT_MS)[0], want)
    st = srv.stats()
    assert st["failed"] == 0 and st["bytes_in_use"] == 0
    srv.close()
