"""Multi-process (gloo, world size 2, CPU) check of the cell-sharded layout: each rank
runs the oracle on its slice with the global cell offset; the gathered slices equal
the single-process run and the all-reduced FP64 moment sums equal the full moments."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, n_cells, q):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    import datetime
    import __graft_entry__
    import oracle
    pkg = __graft_entry__.load_package()
    from scrna_b200 import sharding
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        net = pkg.sample_network(10, seed=3, bursty=True)
        off, cnt = sharding.shard_cells(n_cells, world, rank)
        r = oracle.simulate(net, pkg.WORKLOAD_KINETICS, dt=0.01, n_steps=150, cell_num=cnt, seed=5,
                            cell_offset=off, nthreads=1)
        X = r["P"].T  # cells x genes
        sums = sharding.allreduce_moments(sharding.moment_sums(X))
        import torch
        parts = [None] * world
        dist.all_gather_object(parts, (off, X))
        if rank == 0:
            q.put((sums, parts))
    finally:
        dist.destroy_process_group()


def test_cell_sharding_gloo(pkg, orc):
    import torch.multiprocessing as mp
    from scrna_b200 import sharding
    world, n_cells = 2, 101
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n_cells, q)) for r in range(world)]
    for p in procs:
        p.start()
    sums, parts = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    net = pkg.sample_network(10, seed=3, bursty=True)
    full = orc.simulate(net, pkg.WORKLOAD_KINETICS, dt=0.01, n_steps=150, cell_num=n_cells, seed=5)["P"].T
    gathered = np.vstack([x for _, x in sorted(parts, key=lambda t: t[0])])
    assert np.array_equal(gathered, full)
    mean, var = sharding.moments_from_sums(sums)
    assert np.allclose(mean, full.mean(0), rtol=1e-12)
    assert np.allclose(var, full.var(0, ddof=1), rtol=1e-9)


def test_shard_helpers(pkg):
    from scrna_b200 import sharding
    spans = [sharding.shard_cells(103, 4, r) for r in range(4)]
    assert sum(c for _, c in spans) == 103
    assert [o for o, _ in spans] == [0, 26, 52, 78]
    placement = sharding.shard_networks([5, 1, 1, 1, 4], 2)
    assert sorted(sum(placement, [])) == [0, 1, 2, 3, 4]
    loads = [sum([5, 1, 1, 1, 4][i] for i in pl) for pl in placement]
    assert max(loads) - min(loads) <= 1


def _best_contiguous(costs, world):
    """Smallest largest-range cost over all contiguous splits (exhaustive, small inputs)."""
    import itertools
    n = len(costs)
    if n == 0:
        return 0.0
    best = float("inf")
    for cuts in itertools.combinations(range(1, n), min(world - 1, n - 1)):
        b = (0,) + cuts + (n,)
        best = min(best, max(sum(costs[b[i]:b[i + 1]]) for i in range(len(b) - 1)))
    return best


def test_shard_network_ranges(pkg):
    from scrna_b200 import sharding
    rng = np.random.default_rng(3)
    for trial in range(40):
        n = int(rng.integers(0, 9))
        world = int(rng.integers(1, 5))
        costs = [float(x) for x in rng.integers(1, 50, n)]
        r = sharding.shard_network_ranges(costs, world)
        assert len(r) == world
        # contiguous, in order, covering every network once
        assert r[0][0] == 0 and r[-1][1] == n and all(a[1] == b[0] for a, b in zip(r, r[1:]))
        assert all(lo <= hi for lo, hi in r)
        worst = max((sum(costs[lo:hi]) for lo, hi in r), default=0.0)
        assert worst <= _best_contiguous(costs, world) * (1 + 1e-9) + 1e-9, (costs, world, r)
    with pytest.raises(ValueError):
        sharding.shard_network_ranges([1.0], 0)
