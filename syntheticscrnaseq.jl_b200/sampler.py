"""Seeded synthetic inputs for the CLE workloads.

The reference's sample_network (src/kinetics.jl:105-182, _sample_pair_edge
:185-205) draws TF-level sparse networks.  The workloads here keep its
structure (active TFs, targets per TF, used (target, source) pairs, cooperative
/ redundant edges over 2 sources, one guaranteed non-additive edge for :mixed)
but use the distributions the benchmark workloads name: basals
LogUniform(1, 10), edge strengths +/-U(1, 5), telegraph rates
k_on ~ LogUniform(0.1, 1), k_off ~ LogUniform(1, 10).  Julia's RNG streams are
not reproducible here, so numpy's PCG64 seeded by `seed` is used.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

from .model import (CaptureModel, CoopEdge, GeneNetwork, KineticParams, PopulationConfig,
                    RedunEdge)


def _loguniform(rng, lo, hi, size=None):
    return np.exp(rng.uniform(math.log(lo), math.log(hi), size))


def _strength(rng, lo, hi):
    s = rng.uniform(lo, hi)
    return -s if rng.random() < 0.5 else s


def _pair_edge(rng, G, used, n_src, lo, hi):
    """Pick n_src sources and a target whose (target, source) pairs are unused
    (kinetics.jl:185-205: at most 20 attempts)."""
    if G < n_src + 1:
        return None
    for _ in range(20):
        sources = sorted(rng.choice(G, size=n_src, replace=False).tolist())
        possible = [g for g in range(G) if g not in sources]
        if not possible:
            continue
        target = int(rng.choice(possible))
        if all((target, s) not in used for s in sources):
            for s in sources:
                used.add((target, s))
            return target, tuple(int(s) for s in sources), _strength(rng, lo, hi)
    return None


def sample_network(G: int, *, seed: int = 0, regulation: str = "mixed",
                   n_tf_range: Optional[Tuple[int, int]] = None,
                   targets_per_tf_range: Optional[Tuple[int, int]] = None,
                   n_coop_range: Optional[Tuple[int, int]] = None,
                   n_redun_range: Optional[Tuple[int, int]] = None,
                   n_sources_range: Tuple[int, int] = (2, 2),
                   basal_range: Tuple[float, float] = (1.0, 10.0),
                   strength_range: Tuple[float, float] = (1.0, 5.0),
                   bursty: bool = False,
                   k_on_range: Tuple[float, float] = (0.1, 1.0),
                   k_off_range: Tuple[float, float] = (1.0, 10.0)) -> GeneNetwork:
    """TF-sparse random network (structure of kinetics.jl:105-182). Ranges are inclusive."""
    rng = np.random.Generator(np.random.PCG64(seed))
    if n_tf_range is None:
        n_tf_range = (1, 2) if G <= 5 else (2, 3) if G <= 10 else (4, 5)
    if targets_per_tf_range is None:
        targets_per_tf_range = (1, 3) if G <= 5 else (2, 4) if G <= 10 else (3, 6)
    if n_coop_range is None:
        n_coop_range = (1, 2) if G > 10 else (0, 1)
    if n_redun_range is None:
        n_redun_range = (1, 2) if G > 10 else (0, 1)
    lo, hi = strength_range
    basals = _loguniform(rng, *basal_range, size=G)
    A = np.zeros((G, G))
    used = set()
    n_tf = int(rng.integers(n_tf_range[0], n_tf_range[1] + 1))
    n_tf = min(n_tf, G)
    tfs = sorted(rng.choice(G, size=n_tf, replace=False).tolist()) if G > 1 else []
    for tf in tfs:
        nt = int(rng.integers(targets_per_tf_range[0], targets_per_tf_range[1] + 1))
        possible = [g for g in range(G) if g != tf]
        nt = min(nt, len(possible))
        for t in rng.choice(possible, size=nt, replace=False).tolist():
            A[t, tf] = _strength(rng, lo, hi)
            used.add((t, tf))
    coop: List[CoopEdge] = []
    redun: List[RedunEdge] = []

    def n_src():
        return int(rng.integers(n_sources_range[0], n_sources_range[1] + 1))

    if regulation in ("mixed", "cooperative"):
        for _ in range(int(rng.integers(n_coop_range[0], n_coop_range[1] + 1))):
            r = _pair_edge(rng, G, used, n_src(), lo, hi)
            if r is not None:
                coop.append(CoopEdge(*r))
    if regulation in ("mixed", "redundant"):
        for _ in range(int(rng.integers(n_redun_range[0], n_redun_range[1] + 1))):
            r = _pair_edge(rng, G, used, n_src(), lo, hi)
            if r is not None:
                redun.append(RedunEdge(*r))
    if regulation == "mixed" and not coop and not redun:
        r = _pair_edge(rng, G, used, n_src(), lo, hi)
        if r is not None:
            redun.append(RedunEdge(*r))
    k_on = k_off = None
    if bursty:
        k_on = _loguniform(rng, *k_on_range, size=G)
        k_off = _loguniform(rng, *k_off_range, size=G)
    return GeneNetwork(G, basals, A, coop, redun, k_on, k_off)


def dense_network(G: int, *, seed: int = 0, density: float = 0.10, n_coop: int = 40,
                  n_redun: int = 40, n_sources_range: Tuple[int, int] = (2, 3),
                  basal_range: Tuple[float, float] = (1.0, 10.0),
                  strength_range: Tuple[float, float] = (1.0, 5.0)) -> GeneNetwork:
    """Large dense-regulation network: each off-diagonal A entry nonzero with
    probability `density`, +/-U(lo, hi); cooperative and redundant edges over
    2-3 sources on unused (target, source) pairs."""
    rng = np.random.Generator(np.random.PCG64(seed))
    lo, hi = strength_range
    basals = _loguniform(rng, *basal_range, size=G)
    mask = rng.random((G, G)) < density
    np.fill_diagonal(mask, False)
    sign = np.where(rng.random((G, G)) < 0.5, -1.0, 1.0)
    A = np.where(mask, sign * rng.uniform(lo, hi, (G, G)), 0.0)
    used = set(zip(*np.nonzero(mask)))
    used = {(int(a), int(b)) for a, b in used}
    coop, redun = [], []
    for _ in range(n_coop):
        r = _pair_edge(rng, G, used, int(rng.integers(n_sources_range[0], n_sources_range[1] + 1)), lo, hi)
        if r is not None:
            coop.append(CoopEdge(*r))
    for _ in range(n_redun):
        r = _pair_edge(rng, G, used, int(rng.integers(n_sources_range[0], n_sources_range[1] + 1)), lo, hi)
        if r is not None:
            redun.append(RedunEdge(*r))
    return GeneNetwork(G, basals, A, coop, redun)


# ---- the benchmark workloads ------------------------------------------------------------------
WORKLOAD_KINETICS = KineticParams(k_t=5.0, K_d=10.0, n=2.0, mu_m=1.0, mu_p=0.2, dilution=0.0)


@dataclass
class Workload:
    name: str
    net: GeneNetwork
    kin: KineticParams
    dt: float
    T: float
    cell_num: int
    capture: Optional[CaptureModel] = None
    population: Optional[PopulationConfig] = None
    readout: str = "protein"


def config0(seed: int = 0) -> Workload:
    """Plain CLE, G=5 mixed regulation, 5000 cells, dt=0.01 h, T=50 h."""
    return Workload("plain-G5-N5000", sample_network(5, seed=seed), WORKLOAD_KINETICS, 0.01, 50.0, 5000)


def config1(seed: int = 1) -> Workload:
    """Telegraph bursty CLE + capture, G=10, 20,000 cells; capture efficiency per cell
    LogNormal(log 0.1, 0.5) clipped to (0, 1), without the -sigma^2/2 correction."""
    net = sample_network(10, seed=seed, bursty=True)
    cap = CaptureModel(efficiency=0.1, efficiency_std=0.5, readout="mrna", mean_correction=False)
    return Workload("telegraph-capture-G10-N20000", net, WORKLOAD_KINETICS, 0.01, 50.0, 20000, capture=cap,
                    readout="mrna")


def config2(seed: int = 2) -> Workload:
    """Large dense regulation: G=2000, 65,536 cells, 10% A, 40+40 non-additive edges, dt=0.005, T=40."""
    return Workload("dense-G2000-N65536", dense_network(2000, seed=seed), WORKLOAD_KINETICS, 0.005, 40.0,
                    65536)


def config3(seed: int = 3, n_networks: int = 256) -> List[Workload]:
    """256 networks, G ~ round(LogUniform(5, 500)), cells ~ LogUniform(1k, 50k), half with a
    Moran population (growth 0.7/h, division at V_div = 2, birth volume ~1)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for b in range(n_networks):
        G = int(round(float(_loguniform(rng, 5, 500))))
        N = int(round(float(_loguniform(rng, 1000, 50000))))
        net = sample_network(G, seed=seed * 100003 + b)
        pop = None
        if b % 2 == 1:
            pop = PopulationConfig(cell_num=N, growth_rate=0.7, V_div=2.0, V_init=(1.0, 2.0),
                                   div_check_interval=10)
        out.append(Workload(f"batch-{b}", net, WORKLOAD_KINETICS, 0.01, 50.0, N, population=pop))
    return out


def config4_requests(seed: int = 4, n_requests: int = 200, rate_per_s: float = 50.0):
    """Serving stream: Poisson arrivals, G ~ LogUniform(5, 500), cells ~ LogUniform(1k, 100k),
    T ~ U(20, 60) h, random bursty / constitutive mix, capture on."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t = 0.0
    reqs = []
    for i in range(n_requests):
        t += float(rng.exponential(1.0 / rate_per_s))
        G = int(round(float(_loguniform(rng, 5, 500))))
        N = int(round(float(_loguniform(rng, 1000, 100000))))
        T = float(rng.uniform(20.0, 60.0))
        bursty = bool(rng.random() < 0.5)
        net = sample_network(G, seed=seed * 1000003 + i, bursty=bursty)
        cap = CaptureModel(efficiency=0.1, efficiency_std=0.5, readout="mrna", mean_correction=False)
        reqs.append((t, Workload(f"req-{i}", net, WORKLOAD_KINETICS, 0.01, T, N, capture=cap, readout="mrna")))
    return reqs
