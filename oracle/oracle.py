"""ctypes front end of the CPU oracle — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference leg
use this module, as the checker.  It wraps oracle/_build/libcle_oracle.so, an
FP64 restatement of the reference Julia CLE (src/algorithms/cle.jl:34-284 and
the files listed in cle_oracle.h), built by oracle/Makefile.

Parity status: pinned statistically against the reference's closed-form moment
tests (test/test_analytical_moments.jl) and, for the Philox generator, against
the published Philox4x32-10 known-answer vectors.  The Julia reference itself
cannot run in this environment.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libcle_oracle.so")
_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class _Net(C.Structure):
    _fields_ = [
        ("G", C.c_int32), ("basals", C.c_void_p), ("A", C.c_void_p),
        ("n_coop", C.c_int32), ("coop_target", C.c_void_p), ("coop_ptr", C.c_void_p),
        ("coop_src", C.c_void_p), ("coop_strength", C.c_void_p),
        ("n_redun", C.c_int32), ("redun_target", C.c_void_p), ("redun_ptr", C.c_void_p),
        ("redun_src", C.c_void_p), ("redun_strength", C.c_void_p),
        ("k_on", C.c_void_p), ("k_off", C.c_void_p),
    ]


class _Kin(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("k_t", "K_d", "n", "mu_m", "mu_p", "dilution")]


class _Pop(C.Structure):
    _fields_ = [("growth_rate", C.c_double), ("V_div", C.c_double), ("V_lo", C.c_double),
                ("V_hi", C.c_double), ("div_check_interval", C.c_int32),
                ("partition", C.c_int32), ("exclude_mother", C.c_int32)]


class _Opts(C.Structure):
    _fields_ = [("dt", C.c_double), ("T", C.c_double), ("cell_num", C.c_int64),
                ("seed", C.c_uint64), ("stream", C.c_uint32), ("n_steps", C.c_int64),
                ("cell_offset", C.c_int64)]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_philox4x32_10.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_step_normals.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32,
                                       C.c_uint32, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_cle_simulate.argtypes = [C.POINTER(_Net), C.POINTER(_Kin), C.POINTER(_Pop),
                                       C.POINTER(_Opts), C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_int]
        L.orc_cle_simulate.restype = C.c_int
        L.orc_tauleap_simulate.argtypes = L.orc_cle_simulate.argtypes
        L.orc_tauleap_simulate.restype = C.c_int
        L.orc_expf.argtypes = [C.c_float]
        L.orc_expf.restype = C.c_float
        L.orc_poisson_icdf.argtypes = [C.c_float, C.c_float]
        L.orc_poisson_icdf.restype = C.c_float
        L.orc_capture_efficiency.argtypes = [C.c_int64, C.c_double, C.c_double, C.c_int32,
                                             C.c_uint64, C.c_uint32, C.c_void_p]
        L.orc_capture_counts.argtypes = [C.c_int64, C.c_int32, C.c_void_p, C.c_void_p,
                                         C.c_uint64, C.c_uint32, C.c_void_p, C.c_int]
        L.orc_binomial_invcdf.argtypes = [C.c_int64, C.c_double, C.c_uint64, C.c_uint32,
                                          C.c_uint32, C.c_uint32]
        L.orc_binomial_invcdf.restype = C.c_int64
        L.orc_binomial_half.argtypes = [C.c_int64, C.c_uint64, C.c_uint32, C.c_uint32,
                                        C.c_uint32, C.c_uint32, C.c_uint32]
        L.orc_binomial_half.restype = C.c_int64
        _lib = L
    return _lib


def philox(ctr, key):
    c = np.asarray(ctr, dtype=np.uint32)
    k = np.asarray(key, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    lib().orc_philox4x32_10(c.ctypes.data, k.ctypes.data, out.ctypes.data)
    return out


def step_normals(seed, stream, cell, step, gene):
    zm, zp = C.c_double(), C.c_double()
    lib().orc_step_normals(seed, stream, cell, step, gene, C.byref(zm), C.byref(zp))
    return zm.value, zp.value


class _Keep:
    """Holds numpy buffers alive for the duration of a ctypes call."""

    def __init__(self):
        self.items = []

    def arr(self, x, dtype):
        a = np.ascontiguousarray(np.asarray(x, dtype=dtype))
        self.items.append(a)
        return a.ctypes.data if a.size else None


def _edges(keep, edges, G):
    n = len(edges)
    tgt = [e.target for e in edges]
    ptr = [0]
    src = []
    for e in edges:
        src.extend(e.sources)
        ptr.append(len(src))
    st = [e.strength for e in edges]
    return (n, keep.arr(tgt, np.int32), keep.arr(ptr, np.int32), keep.arr(src, np.int32),
            keep.arr(st, np.float64))


def simulate(net, kin, *, dt, T=50.0, cell_num=1000, seed=0, stream=0, population=None,
             n_steps=0, nthreads=0, cell_offset=0, tauleap=False):
    """FP64 oracle run. `net` is a host GeneNetwork (0-based edge indices).

    Returns dict with M, P ([G, N] float64), prom ([G, N] uint8) and V ([N]) when
    population is given. `population` is a PopulationConfig-like object with
    growth_rate, V_div, V_init, div_check_interval, partition, exclude_mother.
    tauleap=True runs the GPU binomial tau-leap restatement (M, P are counts)."""
    keep = _Keep()
    G = int(net.G)
    cn = _edges(keep, net.cooperative, G)
    rn = _edges(keep, net.redundant, G)
    A = np.asarray(net.interactions, dtype=np.float64).reshape(G, G)
    n = _Net(G, keep.arr(net.basals, np.float64), keep.arr(A, np.float64),
             cn[0], cn[1], cn[2], cn[3], cn[4], rn[0], rn[1], rn[2], rn[3], rn[4],
             keep.arr(net.k_on, np.float64), keep.arr(net.k_off, np.float64))
    k = _Kin(kin.k_t, kin.K_d, kin.n, kin.mu_m, kin.mu_p, kin.dilution)
    N = int(cell_num)
    o = _Opts(float(dt), float(T), N, int(seed), int(stream), int(n_steps), int(cell_offset))
    M = np.zeros((G, N)); P = np.zeros((G, N)); prom = np.zeros((G, N), dtype=np.uint8)
    V = np.zeros(N)
    pp = None
    if population is not None:
        lo, hi = population.V_init
        pp = _Pop(population.growth_rate, population.V_div, lo, hi,
                  population.div_check_interval, population.partition_code,
                  int(population.exclude_mother))
    fn = lib().orc_tauleap_simulate if tauleap else lib().orc_cle_simulate
    rc = fn(C.byref(n), C.byref(k), C.byref(pp) if pp is not None else None, C.byref(o), M.ctypes.data,
            P.ctypes.data, V.ctypes.data, prom.ctypes.data, int(nthreads))
    if rc != 0:
        raise ValueError("oracle rejected the arguments")
    out = {"M": M, "P": P, "prom": prom}
    if population is not None:
        out["V"] = V
    return out


def capture_efficiency(N, efficiency, efficiency_std, mean_correction, seed, stream=0):
    eff = np.zeros(int(N))
    lib().orc_capture_efficiency(int(N), float(efficiency), float(efficiency_std),
                                 int(mean_correction), int(seed), int(stream), eff.ctypes.data)
    return eff


def capture_counts(X_gn, eff, seed, stream=0, nthreads=0):
    """X_gn: [G, N] float64 molecule values, eff: [N]. Returns [G, N] int32."""
    X = np.ascontiguousarray(X_gn, dtype=np.float64)
    e = np.ascontiguousarray(eff, dtype=np.float64)
    G, N = X.shape
    Y = np.zeros((G, N), dtype=np.int32)
    lib().orc_capture_counts(N, G, X.ctypes.data, e.ctypes.data, int(seed), int(stream),
                             Y.ctypes.data, int(nthreads))
    return Y


def binomial_invcdf(n, p, seed, stream, cell, gene):
    return lib().orc_binomial_invcdf(int(n), float(p), int(seed), int(stream), int(cell), int(gene))


def binomial_half(n, seed, stream, cell, step, gene, species):
    return lib().orc_binomial_half(int(n), int(seed), int(stream), int(cell), int(step),
                                   int(gene), int(species))


def log2f(u):
    L = lib()
    L.orc_log2f.argtypes = [C.c_float]
    L.orc_log2f.restype = C.c_float
    return L.orc_log2f(float(u))


def geom_steps(w, inv):
    L = lib()
    L.orc_geom_steps.argtypes = [C.c_uint32, C.c_float]
    L.orc_geom_steps.restype = C.c_int32
    return L.orc_geom_steps(int(w), float(inv))


def geom_steps_u(u, inv):
    L = lib()
    L.orc_geom_steps_u.argtypes = [C.c_float, C.c_float]
    L.orc_geom_steps_u.restype = C.c_int32
    return L.orc_geom_steps_u(float(u), float(inv))


def switch_uniform(w0, w1):
    L = lib()
    L.orc_switch_uniform.argtypes = [C.c_uint32, C.c_uint32]
    L.orc_switch_uniform.restype = C.c_float
    return L.orc_switch_uniform(int(w0), int(w1))


def expf(x):
    return lib().orc_expf(float(x))


def poisson_icdf(u, lam):
    return lib().orc_poisson_icdf(float(u), float(lam))
