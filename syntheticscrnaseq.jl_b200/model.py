"""Model types of the CLE path, mirroring the reference's Julia structs.

GeneNetwork / CoopEdge / RedunEdge     src/network.jl:16-96
KineticParams                          src/kinetics.jl:25-50
PopulationConfig / CaptureModel        src/population.jl:27-74
CLE                                    src/algorithms/cle.jl:21-23
BinomialTauLeap                        src/algorithms/tauleap_binomial.jl:19-22

Indices are 0-based in Python (the Julia shim converts from 1-based).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

INF = math.inf


@dataclass(frozen=True)
class CoopEdge:
    """AND gate: reg[target] += strength * beta[target] * prod(act[src]) (network.jl:16-20)."""
    target: int
    sources: Tuple[int, ...]
    strength: float


@dataclass(frozen=True)
class RedunEdge:
    """OR gate: reg[target] += strength * beta[target] * (1 - prod(1 - act[src])) (network.jl:30-34)."""
    target: int
    sources: Tuple[int, ...]
    strength: float


@dataclass
class GeneNetwork:
    """G genes with basals, interaction matrix A (A[i, j] = effect of protein j on
    gene i, zero diagonal), cooperative and redundant edges and telegraph rates
    (inf = constitutive).  Same fields and checks as network.jl:55-96."""
    G: int
    basals: np.ndarray
    interactions: np.ndarray
    cooperative: List[CoopEdge] = field(default_factory=list)
    redundant: List[RedunEdge] = field(default_factory=list)
    k_on: Optional[np.ndarray] = None
    k_off: Optional[np.ndarray] = None

    def __post_init__(self):
        self.basals = np.asarray(self.basals, dtype=np.float64).reshape(-1)
        self.interactions = np.asarray(self.interactions, dtype=np.float64)
        G = int(self.G)
        if self.basals.shape != (G,):
            raise ValueError(f"basals must have length G={G}")
        if self.interactions.shape != (G, G):
            raise ValueError(f"interactions must be {G}x{G}")
        if np.any(np.diag(self.interactions) != 0.0):
            raise ValueError("interaction diagonal must be zero")
        self.k_on = np.full(G, INF) if self.k_on is None else np.asarray(self.k_on, dtype=np.float64)
        self.k_off = np.full(G, INF) if self.k_off is None else np.asarray(self.k_off, dtype=np.float64)
        if self.k_on.shape != (G,) or self.k_off.shape != (G,):
            raise ValueError("k_on / k_off must have length G")
        for e in list(self.cooperative) + list(self.redundant):
            if not (0 <= e.target < G) or any(not (0 <= s < G) for s in e.sources) or not e.sources:
                raise ValueError(f"edge {e} references genes outside 0..{G - 1}")

    @classmethod
    def from_basals(cls, basals, interactions, *, cooperative=(), redundant=(), k_on=None,
                    k_off=None):
        """Convenience constructor inferring G (network.jl:85-96)."""
        b = np.asarray(basals, dtype=np.float64)
        return cls(len(b), b, interactions, list(cooperative), list(redundant), k_on, k_off)


def is_bursty(net: GeneNetwork) -> bool:
    """Any finite telegraph rate (network.jl:103)."""
    return bool(np.any(np.isfinite(net.k_on)) or np.any(np.isfinite(net.k_off)))


def hill_activation(p, K, n):
    """p^n / (p^n + K^n) (network.jl:112-115)."""
    pn = np.power(p, n)
    return pn / (pn + K ** n)


def hill_repression(p, K, n):
    """K^n / (p^n + K^n) (network.jl:122-125)."""
    pn = np.power(p, n)
    return K ** n / (pn + K ** n)


def precompute_hill_matrices(net: GeneNetwork):
    """(A_pos, A_neg) with A_eff[i, j] = A[i, j] * beta_i off the diagonal (network.jl:206-219)."""
    A_eff = net.interactions * net.basals[:, None]
    np.fill_diagonal(A_eff, 0.0)
    return np.maximum(A_eff, 0.0), np.maximum(-A_eff, 0.0)


@dataclass(frozen=True)
class KineticParams:
    """Translation k_t, Hill K_d and n, decays mu_m / mu_p, dilution (kinetics.jl:25-50);
    defaults are the reference's."""
    k_t: float = 4.3376521035785345
    K_d: float = 61.47011276535837
    n: float = 10.0
    mu_m: float = 0.04987442692380366
    mu_p: float = 0.36777724535966944
    dilution: float = 0.0


def steady_state(net: GeneNetwork, kin: KineticParams):
    """Unregulated deterministic steady state (kinetics.jl:65-70)."""
    mu = kin.dilution
    m = net.basals / (kin.mu_m + mu)
    p = kin.k_t * m / (kin.mu_p + mu)
    return m, p


@dataclass(frozen=True)
class PopulationConfig:
    """Moran population (population.jl:27-45).  `partition` is "binomial" (split of
    rounded counts, ext/SyntheticscRNAseqCUDAExt.jl:641-651) or "halve"
    (cle.jl:249-261); `exclude_mother` picks the replaced slot among the other
    cells as cle.jl:265-268 does (False: any cell, ext:509)."""
    cell_num: int = 1000
    growth_rate: float = 0.03
    V_div: float = 2.0
    V_init: Tuple[float, float] = (0.8, 1.2)
    div_check_interval: int = 10
    growth_noise: float = 0.0
    partition: str = "binomial"
    exclude_mother: bool = True

    @property
    def partition_code(self) -> int:
        return {"binomial": 0, "halve": 1}[self.partition]


@dataclass(frozen=True)
class CaptureModel:
    """LogNormal-Binomial capture (population.jl:57-74, capture.jl:25-47).
    mean_correction=True uses mu_log = log(efficiency) - sigma^2/2 as the reference."""
    efficiency: float = 0.1
    efficiency_std: float = 0.2
    readout: str = "mrna"
    mean_correction: bool = True

    def __post_init__(self):
        if self.readout not in ("mrna", "protein"):
            raise ValueError("readout must be :mrna or :protein")


@dataclass(frozen=True)
class CLE:
    """Chemical Langevin Equation with Euler-Maruyama and collapsed noise (cle.jl:21-23)."""
    dt: float


@dataclass(frozen=True)
class BinomialTauLeap:
    """Binomial tau-leap with step dt (tauleap_binomial.jl:19-22); on the GPU the reference's
    FP32 inverse-CDF form (ext/SyntheticscRNAseqCUDAExt.jl:215-399)."""
    dt: float


def n_steps(T: float, dt: float) -> int:
    """ceil(T / dt) in FP64 (cle.jl:56)."""
    return int(math.ceil(T / dt))


def default_algorithm(G: int, *, gpu: bool = False, dt: float = 0.1):
    """Routing (default_algorithm.jl:31-39): the GPU route is CLE(dt).  The CPU-only
    tau-leap algorithms are outside this library, so gpu=False with G <= 10 raises."""
    if gpu or G > 10:
        return CLE(dt)
    raise NotImplementedError("BinomialTauLeapFast (CPU, G <= 10) is not part of the GPU CLE library")
