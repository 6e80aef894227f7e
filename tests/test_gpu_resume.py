"""Continuation and checkpoints of register-path runs, through the C ABI: a run of T1 steps
continued to T2 equals one run of T2 steps bit for bit (state, volumes and readout), for the
lane and block kernels, populations whose first leg ends on and off a division check, the
tau-leap, and a checkpoint restored into a fresh state (another layout than the one that
wrote it)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pair(pkg, net, alg, kin, T1, T2, **kw):
    full = pkg.DeviceRun(net, alg, kin, T=T2, **kw)
    full.launch()
    part = pkg.DeviceRun(net, alg, kin, T=T1, **kw)
    part.launch()
    assert part.steps_done == pkg.n_steps(T1, alg.dt)
    part.resume(T=T2)
    assert part.steps_done == pkg.n_steps(T2, alg.dt)
    return full, part


def _same(a, b, pop):
    ra, rb = a.read_raw(), b.read_raw()
    for k in ("M", "P", "prom") + (("V",) if pop else ()):
        assert np.array_equal(ra[k], rb[k]), k
    xa, xb = a.read(), b.read()
    for u, v in zip(xa if isinstance(xa, tuple) else (xa,), xb if isinstance(xb, tuple) else (xb,)):
        assert np.array_equal(u, v)


@pytest.mark.parametrize("path", ["auto", "block"])
def test_resume_equals_one_run(pkg, path):
    net = pkg.sample_network(10, seed=1, bursty=True)
    full, part = _pair(pkg, net, pkg.CLE(0.01), pkg.WORKLOAD_KINETICS, 0.73, 2.0, cell_num=999, readout="both",
                       seed=4, path=path)
    _same(full, part, False)


@pytest.mark.parametrize("T1", [0.7, 0.75])  # 70 steps: a division check; 75: inside a chunk
def test_resume_population(pkg, T1):
    net = pkg.sample_network(8, seed=3, bursty=True)
    pop = pkg.PopulationConfig(cell_num=500, growth_rate=0.7, V_div=2.0, V_init=(1.0, 2.0), div_check_interval=10)
    full, part = _pair(pkg, net, pkg.CLE(0.01), pkg.WORKLOAD_KINETICS, T1, 1.6, cell_num=500, readout="both",
                       seed=7, population=pop)
    _same(full, part, True)


def test_resume_tauleap_population_with_capture(pkg):
    net = pkg.sample_network(6, seed=5, bursty=True)
    pop = pkg.PopulationConfig(cell_num=300, growth_rate=0.6, V_div=2.0, V_init=(1.0, 2.0), div_check_interval=5,
                               exclude_mother=False)
    cap = pkg.CaptureModel(efficiency=0.3, efficiency_std=0.3, readout="mrna")
    full, part = _pair(pkg, net, pkg.BinomialTauLeap(0.02), pkg.WORKLOAD_KINETICS, 0.5, 1.3, cell_num=300,
                       readout="mrna", seed=2, population=pop, capture=cap)
    _same(full, part, True)


def test_checkpoint_restore_resume(pkg):
    net = pkg.sample_network(12, seed=8, bursty=True)
    pop = pkg.PopulationConfig(cell_num=400, growth_rate=0.7, V_div=2.0, V_init=(1.0, 2.0), div_check_interval=10)
    kin = pkg.WORKLOAD_KINETICS
    full = pkg.DeviceRun(net, pkg.CLE(0.01), kin, T=1.5, cell_num=400, readout="both", seed=9, population=pop)
    full.launch()
    first = pkg.DeviceRun(net, pkg.CLE(0.01), kin, T=0.55, cell_num=400, readout="both", seed=9, population=pop)
    first.launch()
    data = first.checkpoint()
    assert data[:8] == b"SCRNACK1"
    second = pkg.DeviceRun(net, pkg.CLE(0.01), kin, T=0.55, cell_num=400, readout="both", seed=9, population=pop)
    with pytest.raises(pkg.ScrnaError):
        second.resume(T=1.5)  # holds no run yet
    second.restore(data)
    assert second.steps_done == 55
    second.resume(T=1.5)
    _same(full, second, True)
    with pytest.raises(pkg.ScrnaError):
        second.restore(data[:-1])
    other = pkg.DeviceRun(pkg.sample_network(11, seed=1), pkg.CLE(0.01), kin, T=0.5, cell_num=400)
    with pytest.raises(pkg.ScrnaError):
        other.restore(data)


def test_tensor_path_state_is_not_resumable(pkg):
    """A tensor-path run keeps no register-path state between calls: continuing it or taking a
    checkpoint is refused with an error, and the run's own results stay readable."""
    net = pkg.sample_network(30, seed=3, bursty=True)
    run = pkg.DeviceRun(net, pkg.CLE(0.01), pkg.WORKLOAD_KINETICS, cell_num=64, T=0.0, n_steps=20,
                        readout="both", path="tensor_library")
    run.launch()
    X = run.read()
    with pytest.raises(pkg.ScrnaError):
        run.resume(n_steps=40)
    with pytest.raises(pkg.ScrnaError):
        run.checkpoint()
    assert np.array_equal(run.read(), X)
    run.close()


@pytest.mark.parametrize("population", [False, True])
def test_tauleap_tensor_form_resumes_and_checkpoints(pkg, population):
    """A tau-leap run of 300 genes, which the automatic path runs on the tensor form, leaves
    the register path's state: it continues there, directly and through a checkpoint, bit for
    bit one run of the total length."""
    net = pkg.sample_network(300, seed=7, bursty=True)
    kin = pkg.WORKLOAD_KINETICS
    pop = pkg.PopulationConfig(cell_num=300, growth_rate=0.7, V_div=2.0, V_init=(1.0, 2.0), div_check_interval=10)
    kw = dict(cell_num=300, readout="both", seed=5, population=pop if population else None)
    alg = pkg.BinomialTauLeap(0.01)
    full, part = _pair(pkg, net, alg, kin, 0.55, 1.2, **kw)
    _same(full, part, population)
    first = pkg.DeviceRun(net, alg, kin, T=0.55, path="tensor", **kw)
    first.launch()
    data = first.checkpoint()
    second = pkg.DeviceRun(net, alg, kin, T=0.55, **kw)
    second.restore(data)
    second.resume(T=1.2)
    _same(full, second, population)
    first.resume(T=1.2)  # asked of the tensor path: continues on the register path
    _same(full, first, population)
    for r in (full, part, first, second):
        r.close()
