"""CPU tests of the host-side helpers of the Python API: the pool of page-locked result
blocks (with a stand-in allocator, so no GPU is needed) and the content digest that keys
the per-context cache of uploaded networks."""
import ctypes as C

import numpy as np
import pytest


class _FakeLib:
    """Stands in for scrna_host_alloc / scrna_host_free with ordinary host memory."""

    def __init__(self):
        self.allocs = 0
        self.frees = 0
        self._keep = {}

    def scrna_host_alloc(self, size, pp):
        buf = C.create_string_buffer(size)
        addr = C.addressof(buf)
        self._keep[addr] = buf
        pp._obj.value = addr
        self.allocs += 1
        return 0

    def scrna_host_free(self, p):
        self._keep.pop(p.value, None)
        self.frees += 1
        return 0


@pytest.fixture
def pool(pkg, monkeypatch):
    from scrna_b200 import _pinned
    fake = _FakeLib()
    monkeypatch.setattr(_pinned, "_lib", type("L", (), {"load": staticmethod(lambda: fake)}))
    return _pinned.PinnedPool(cap_bytes=64 << 20), fake


def test_pool_reuses_released_blocks(pool):
    p, fake = pool
    x = None
    for i in range(6):  # the previous result stays alive while the next one is allocated
        x = p.empty((20000, 10), np.float64, order="F")
        x[:] = i
    assert fake.allocs == 2  # first block + the spare pinned with it
    assert x.flags["F_CONTIGUOUS"] and x.shape == (20000, 10) and float(x[3, 4]) == 5.0


def test_pool_never_hands_out_a_live_block(pool):
    p, _ = pool
    a = p.empty(1000, np.int32)
    b = p.empty(1000, np.int32)
    a[:] = 1
    b[:] = 2
    assert a.__array_interface__["data"][0] != b.__array_interface__["data"][0]
    assert np.all(a == 1) and np.all(b == 2)


def test_pool_size_classes_and_limits(pool):
    from scrna_b200 import _pinned
    p, fake = pool
    assert _pinned._round(1) == 4096 and _pinned._round(4097) == 8192 and _pinned._round(1 << 20) == 1 << 20
    big = p.empty(((_pinned.MAX_BLOCK // 8) + 1,), np.float64)  # above the largest block: pageable
    assert fake.allocs == 0 and big.size == _pinned.MAX_BLOCK // 8 + 1
    assert p.empty((0, 5), np.float64).shape == (0, 5) and fake.allocs == 0


def test_pool_caps_idle_blocks(pkg, monkeypatch):
    from scrna_b200 import _pinned
    fake = _FakeLib()
    monkeypatch.setattr(_pinned, "_lib", type("L", (), {"load": staticmethod(lambda: fake)}))
    p = _pinned.PinnedPool(cap_bytes=1 << 20)
    arrays = [p.empty(1 << 17, np.float64) for _ in range(3)]  # 1 MiB blocks
    del arrays
    assert p._idle <= 1 << 20 and fake.frees >= 2


def test_pool_falls_back_when_pinning_is_refused(pkg, monkeypatch):
    from scrna_b200 import _pinned

    class Refuse(_FakeLib):
        def scrna_host_alloc(self, size, pp):
            return -3

    monkeypatch.setattr(_pinned, "_lib", type("L", (), {"load": staticmethod(lambda: Refuse())}))
    p = _pinned.PinnedPool()
    a = p.empty((7, 3), np.float32, order="F")
    a[:] = 1.5
    assert p._disabled and a.flags["F_CONTIGUOUS"] and float(a.sum()) == 31.5


def test_network_digest_follows_content(pkg):
    from scrna_b200 import api
    net = pkg.sample_network(8, seed=21, bursty=True)
    d0 = api._net_digest(net)
    same = pkg.sample_network(8, seed=21, bursty=True)  # another object, same content
    assert api._net_digest(same) == d0
    net.basals[0] *= 3.0  # same object, changed in place
    assert api._net_digest(net) != d0
    other = pkg.sample_network(8, seed=22, bursty=True)
    assert api._net_digest(other) != d0


def test_network_digest_skips_large_networks(pkg):
    from scrna_b200 import api
    big = pkg.dense_network(400, seed=1, density=0.1, n_coop=2, n_redun=2)  # 400 x 400 doubles = 1.28 MB
    assert api._net_digest(big) is None


class _FakeServer:
    """A server stand-in that records submissions and never finishes them."""

    def __init__(self):
        self.ctx = object()
        self.jobs = []

    def submit(self, handle, alg, kin, **kw):
        self.jobs.append(kw)
        return len(self.jobs)

    def stats(self):
        return {"units_done": 0, "completed": 0, "failed": 0, "busy_s": 0.0}


def test_least_loaded_and_pool_placement(pkg, monkeypatch):
    assert pkg.least_loaded([3, 1, 1, 5]) == 1 and pkg.least_loaded([0]) == 0
    from importlib import import_module
    api = import_module(pkg.__name__ + ".api")
    monkeypatch.setattr(api, "_handle_for", lambda net, ctx: None)
    pool = object.__new__(pkg.ServerPool)
    pool.servers = [_FakeServer(), _FakeServer()]
    pool._submitted = [0, 0]
    pool._where = {}
    pool._next = 1
    kin = pkg.WORKLOAD_KINETICS
    big = pkg.GeneNetwork(100, np.ones(100), np.zeros((100, 100)))
    small = pkg.GeneNetwork(2, np.ones(2), np.zeros((2, 2)))
    t1 = pool.submit(big, pkg.CLE(0.01), kin, cell_num=1000, T=1.0)      # 1e7 units -> server 0
    t2 = pool.submit(small, pkg.CLE(0.01), kin, cell_num=1000, T=1.0)    # server 1 (empty)
    t3 = pool.submit(small, pkg.CLE(0.01), kin, cell_num=1000, T=1.0)    # server 1 (2e5 < 1e7)
    assert [pool.server_of(t) for t in (t1, t2, t3)] == [0, 1, 1]
    assert pool.loads() == [100 * 1000 * 100, 2 * 2 * 1000 * 100]
