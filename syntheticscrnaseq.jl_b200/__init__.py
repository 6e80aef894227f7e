"""B200-native batched CLE for synthetic scRNA-seq (drop-in for the GPU CLE of
Msturroc/SyntheticscRNAseq.jl).

Compute runs in libscrna_cle.so (hand-written sm_100a CUDA behind the C ABI in
include/scrna_cle.h); this package is the host-side mirror of the reference's
Julia interface.  The directory name is not a Python identifier, so the package
is imported under the name ``scrna_b200`` (see __graft_entry__.load_package).
"""
from .model import (CLE, INF, BinomialTauLeap, CaptureModel, CoopEdge, GeneNetwork, KineticParams, PopulationConfig,
                    RedunEdge, default_algorithm, hill_activation, hill_repression, is_bursty, n_steps,
                    precompute_hill_matrices, steady_state)
from .sampler import (WORKLOAD_KINETICS, Workload, config0, config1, config2, config3, config4_requests,
                      dense_network, sample_network)
from .api import (Context, DeviceRun, NetHandle, Server, ServerPool, apply_capture, debug_philox,
                  debug_small_div_check, default_context, ks_statistic_device, least_loaded, measure_philox_rate,
                  measure_pipe_peaks, simulate, simulate_gpu_batch, simulate_gpu_batch_sharded)
from ._lib import ScrnaError
from .validate import (column_moments, compare_moments, empirical_pmf, ks_critical_value, ks_statistic, ks_vs_exact,
                       l1_distance, max_moment_error, moment_errors, pmf_comparison_from_histogram,
                       telegraph_distribution, telegraph_fano, telegraph_mean, telegraph_pmf, telegraph_variance)
from .mtx import read_10x_mtx

__all__ = [
    "CLE", "BinomialTauLeap", "CaptureModel", "CoopEdge", "GeneNetwork", "KineticParams", "PopulationConfig", "RedunEdge",
    "default_algorithm", "hill_activation", "hill_repression", "is_bursty", "n_steps",
    "precompute_hill_matrices", "steady_state", "sample_network", "dense_network", "config0", "config1",
    "config2", "config3", "config4_requests", "Workload", "WORKLOAD_KINETICS", "Context", "DeviceRun",
    "NetHandle", "Server", "ServerPool", "least_loaded", "apply_capture", "debug_philox", "debug_small_div_check", "default_context",
    "measure_philox_rate", "measure_pipe_peaks", "simulate",
    "simulate_gpu_batch", "simulate_gpu_batch_sharded", "ScrnaError", "INF", "column_moments", "compare_moments", "max_moment_error",
    "moment_errors", "ks_statistic", "ks_critical_value", "ks_statistic_device", "telegraph_pmf", "telegraph_mean",
    "telegraph_variance", "telegraph_fano", "read_10x_mtx", "telegraph_distribution", "empirical_pmf",
    "l1_distance", "ks_vs_exact", "pmf_comparison_from_histogram",
]
