"""Reference-facing entry points of the GPU CLE and binomial tau-leap, over the C ABI.

simulate(net, CLE(dt), kin, gpu=True; cell_num, T, readout)      ext/SyntheticscRNAseqCUDAExt.jl:48-117
simulate(net, CLE(dt), kin, gpu=True, population=pop; T, readout) ext:409-529
simulate_gpu_batch(networks, CLE(dt), kin; cell_num, T, readout)  ext:132-213
simulate(net, BinomialTauLeap(dt), kin, ...)                       ext:215-284, population ext:531-663
simulate_gpu_batch(networks, BinomialTauLeap(dt), kin[s], ...)     ext:290-399, ext:666-837
apply_capture(X, capture)                                          src/capture.jl:25-47

Outputs are cells x G (cells x 2G for readout "both") float64 arrays in
column-major (Fortran) order, the layout of the reference's Matrix{Float64}.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import math
import threading
from collections import OrderedDict
from typing import List, Optional, Sequence, Union

import numpy as np

from . import _lib, _pinned
from ._lib import Capture, Kinetics, Opts, Population, check
from .model import BinomialTauLeap, CLE, CaptureModel, GeneNetwork, KineticParams, PopulationConfig, n_steps as n_steps_of

READOUT = {"mrna": 0, "protein": 1, "both": 2}
PRECISION = {"fp32": 0, "fp64_plain": 1, "fp32_f16": 2}
PATH = {"auto": 0, "register": 1, "tensor": 2, "block": 3, "warp": 4, "tensor_library": 5}


class Context:
    """One device + one CUDA stream (scrna_ctx)."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        h = C.c_void_p()
        check(self.lib.scrna_ctx_create(int(device), C.byref(h)))
        self.h = h
        self.device = device

    def set_stream(self, cuda_stream_handle: int):
        check(self.lib.scrna_ctx_set_stream(self.h, C.c_void_p(int(cuda_stream_handle))))

    def synchronize(self):
        check(self.lib.scrna_ctx_synchronize(self.h))

    @property
    def launches(self) -> int:
        return int(self.lib.scrna_ctx_launch_count(self.h))

    def set_autotune(self, mode: int, cache_path: Optional[str] = None):
        """Kernel-variant autotuning: 0 off (static choice), 1 cached or measured, 2 cache only.
        cache_path None keeps the current cache file, "" keeps choices in memory only."""
        check(self.lib.scrna_ctx_set_autotune(self.h, int(mode), None if cache_path is None else cache_path.encode()))

    def last_kernel_choice(self) -> dict:
        """The register-path kernel variant of this context's last run (found: 1 if tuned)."""
        c = _lib.TuneChoice()
        check(self.lib.scrna_autotune_last_choice(self.h, C.byref(c)))
        return {n: getattr(c, n) for n, _ in c._fields_}

    def transfer_bytes(self):
        """(host->device, device->host) bytes this context's calls have copied so far."""
        h2d, d2h = C.c_int64(), C.c_int64()
        check(self.lib.scrna_ctx_transfer_bytes(self.h, C.byref(h2d), C.byref(d2h)))
        return int(h2d.value), int(d2h.value)

    def close(self):
        if getattr(self, "h", None):
            for nh in self.__dict__.pop("_net_cache", {}).values():  # networks before the context
                nh.close()
            self.lib.scrna_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx: Optional[Context] = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


class _Keep(list):
    def arr(self, x, dtype):
        a = np.ascontiguousarray(np.asarray(x, dtype=dtype))
        self.append(a)
        return a.ctypes.data if a.size else None


def _edge_arrays(keep: _Keep, edges):
    tgt = [e.target for e in edges]
    ptr = [0]
    src: List[int] = []
    for e in edges:
        src.extend(e.sources)
        ptr.append(len(src))
    st = [e.strength for e in edges]
    if not edges:
        return 0, None, None, None, None
    return (len(edges), keep.arr(tgt, np.int32), keep.arr(ptr, np.int32), keep.arr(src, np.int32),
            keep.arr(st, np.float64))


class NetHandle:
    """A network uploaded to the device (scrna_net)."""

    def __init__(self, net: GeneNetwork, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self.net = net
        keep = _Keep()
        A_col = np.asfortranarray(net.interactions, dtype=np.float64)
        keep.append(A_col)
        c = _edge_arrays(keep, net.cooperative)
        r = _edge_arrays(keep, net.redundant)
        h = C.c_void_p()
        check(self.ctx.lib.scrna_net_create(
            self.ctx.h, int(net.G), keep.arr(net.basals, np.float64), A_col.ctypes.data,
            c[0], c[1], c[2], c[3], c[4], r[0], r[1], r[2], r[3], r[4],
            keep.arr(net.k_on, np.float64), keep.arr(net.k_off, np.float64), 0, C.byref(h)))
        self.h = h
        self.G = int(net.G)

    def close(self):
        # after the context is closed (e.g. finalized first at interpreter exit) the handle
        # must not be used; the context's teardown already released the device
        if getattr(self, "h", None):
            if getattr(self.ctx, "h", None):
                self.ctx.lib.scrna_net_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# Uploaded networks reused across simulate / simulate_gpu_batch calls on one context, keyed
# by the network's content (not its identity, so an array changed in place is a new
# network).  Only networks whose arrays total at most _HANDLE_CACHE_BYTES are hashed and
# kept; the cache lives on the context and goes with it.
_HANDLE_CACHE_BYTES = 1 << 20
_HANDLE_CACHE_SIZE = 64
_handle_lock = threading.Lock()


def _net_digest(net: GeneNetwork) -> Optional[bytes]:
    arrays = (net.basals, net.interactions, net.k_on, net.k_off)
    if sum(a.nbytes for a in arrays) > _HANDLE_CACHE_BYTES:
        return None
    h = hashlib.blake2b(digest_size=20)
    h.update(int(net.G).to_bytes(8, "little"))
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    for tag, edges in ((b"c", net.cooperative), (b"r", net.redundant)):
        h.update(tag)
        for e in edges:
            h.update(repr((int(e.target), tuple(int(x) for x in e.sources), float(e.strength))).encode())
    return h.digest()


def _handle_for(net: GeneNetwork, ctx: Context) -> "NetHandle":
    d = _net_digest(net)
    if d is None:
        return NetHandle(net, ctx)
    with _handle_lock:
        cache = ctx.__dict__.setdefault("_net_cache", OrderedDict())
        hit = cache.get(d)
        if hit is not None and hit.h and getattr(ctx, "h", None):
            cache.move_to_end(d)
            return hit
    h = NetHandle(net, ctx)
    with _handle_lock:  # an evicted handle is released when its last user drops it
        cache[d] = h
        while len(cache) > _HANDLE_CACHE_SIZE:
            cache.popitem(last=False)
    return h


def _kin(kin: KineticParams) -> Kinetics:
    return Kinetics(kin.k_t, kin.K_d, kin.n, kin.mu_m, kin.mu_p, kin.dilution)


def _pop(pop: Optional[PopulationConfig]):
    if pop is None:
        return None
    lo, hi = pop.V_init
    return Population(int(pop.cell_num), float(pop.growth_rate), float(pop.V_div), float(lo), float(hi),
                      int(pop.div_check_interval), int(pop.partition_code), int(bool(pop.exclude_mother)),
                      0, float(pop.growth_noise))


def _cap(cap: Optional[CaptureModel]):
    if cap is None:
        return None
    return Capture(float(cap.efficiency), float(cap.efficiency_std), READOUT[cap.readout],
                   int(bool(cap.mean_correction)))


def _is_tau(alg) -> bool:
    if isinstance(alg, BinomialTauLeap):
        return True
    if isinstance(alg, CLE):
        return False
    raise TypeError(f"algorithm must be CLE(dt) or BinomialTauLeap(dt), got {alg!r}")


def _opts(alg, *, T, cell_num, readout, seed, stream, precision, path, n_steps, cell_offset):
    if readout not in READOUT:
        raise ValueError("readout must be 'mrna', 'protein' or 'both'")
    return Opts(float(alg.dt), float(T), int(cell_num), READOUT[readout], PRECISION[precision], int(seed),
                int(stream), PATH[path], int(n_steps), int(cell_offset))


def _ptr(x):
    return None if x is None else C.byref(x)


def simulate(net: GeneNetwork, alg, kin: KineticParams, gpu: bool = True, population=None, *,
             cell_num: int = 1000, T: float = 50.0, readout: str = "protein", seed: int = 0,
             stream: int = 0, capture: Optional[CaptureModel] = None, precision: str = "fp32",
             path: str = "auto", n_steps: int = 0, cell_offset: int = 0,
             ctx: Optional[Context] = None, handle: Optional[NetHandle] = None):
    """GPU run of CLE(dt) or BinomialTauLeap(dt).  Returns the readout matrix, or (matrix,
    counts, efficiencies) when `capture` is given.  With `population`, pop.cell_num cells are
    simulated (the tau-leap then reads out concentrations M / V, P / V)."""
    if not gpu:
        raise NotImplementedError("only the GPU path is provided by this library")
    ctx = ctx or default_context()
    h = handle or _handle_for(net, ctx)
    N = population.cell_num if population is not None else cell_num
    cols = net.G * (2 if readout == "both" else 1)
    out = _pinned.empty((N, cols), np.float64, order="F")
    counts = _pinned.empty((N, net.G), np.int32, order="F") if capture is not None else None
    eff = _pinned.empty(N, np.float64) if capture is not None else None
    k, p, c = _kin(kin), _pop(population), _cap(capture)
    o = _opts(alg, T=T, cell_num=N, readout=readout, seed=seed, stream=stream, precision=precision,
              path=path, n_steps=n_steps, cell_offset=cell_offset)
    fn = ctx.lib.scrna_tauleap_simulate if _is_tau(alg) else ctx.lib.scrna_cle_simulate
    check(fn(ctx.h, h.h, C.byref(k), _ptr(p), _ptr(c), C.byref(o), out.ctypes.data,
             None if counts is None else counts.ctypes.data, None if eff is None else eff.ctypes.data))
    if capture is not None:
        return out, counts, eff
    return out


def simulate_gpu_batch(networks: Sequence[GeneNetwork], alg, kin, *,
                       cell_num: Union[int, Sequence[int]] = 1000, T: float = 50.0,
                       readout: str = "protein", seed: int = 0, stream: int = 0,
                       populations: Optional[Sequence[Optional[PopulationConfig]]] = None,
                       capture: Optional[CaptureModel] = None, ctx: Optional[Context] = None):
    """Batched GPU CLE over networks of any sizes.  `kin` is one KineticParams or one
    per network; `cell_num` one count or one per network.  Network b uses Philox
    stream `stream + b`.  Returns a list of readout matrices (and count matrices
    when `capture` is given)."""
    ctx = ctx or default_context()
    B = len(networks)
    kins = list(kin) if isinstance(kin, (list, tuple)) else [kin]
    cns = list(cell_num) if isinstance(cell_num, (list, tuple, np.ndarray)) else [int(cell_num)] * B
    handles = [_handle_for(n, ctx) for n in networks]
    pops = list(populations) if populations is not None else [None] * B
    outs, cnts = [], []
    for b, n in enumerate(networks):
        N = pops[b].cell_num if pops[b] is not None else cns[b]
        cols = n.G * (2 if readout == "both" else 1)
        outs.append(_pinned.empty((N, cols), np.float64, order="F"))
        if capture is not None:
            cnts.append(_pinned.empty((N, n.G), np.int32, order="F"))
    karr = (Kinetics * len(kins))(*[_kin(k) for k in kins])
    harr = (C.c_void_p * B)(*[h.h.value for h in handles])
    cn_arr = (C.c_int64 * B)(*[int(x) for x in cns])
    pop_structs = [_pop(p) for p in pops]
    parr = (C.c_void_p * B)(*[None if p is None else C.addressof(p) for p in pop_structs])
    oarr = (C.c_void_p * B)(*[o.ctypes.data for o in outs])
    carr = (C.c_void_p * B)(*[c.ctypes.data for c in cnts]) if capture is not None else None
    c = _cap(capture)
    o = _opts(alg, T=T, cell_num=0, readout=readout, seed=seed, stream=stream, precision="fp32",
              path="auto", n_steps=0, cell_offset=0)
    fn = ctx.lib.scrna_tauleap_simulate_batch if _is_tau(alg) else ctx.lib.scrna_cle_simulate_batch
    check(fn(ctx.h, B, harr, karr, len(kins), cn_arr, parr, _ptr(c), C.byref(o), oarr, carr))
    if capture is not None:
        return outs, cnts
    return outs


def simulate_gpu_batch_sharded(networks: Sequence[GeneNetwork], alg, kin, *, contexts: Sequence[Context],
                               cell_num: Union[int, Sequence[int]] = 1000, T: float = 50.0,
                               readout: str = "protein", seed: int = 0, stream: int = 0,
                               populations: Optional[Sequence[Optional[PopulationConfig]]] = None,
                               capture: Optional[CaptureModel] = None):
    """simulate_gpu_batch over several contexts, normally one per GPU: whole networks (a
    Moran population couples a network's cells) in contiguous ranges of balanced cost
    (genes x cells), one batch call per context in its own thread.  A range starting at
    network lo runs with base stream `stream + lo`, so network b keeps stream `stream + b`
    and the results equal one simulate_gpu_batch call's."""
    from concurrent.futures import ThreadPoolExecutor
    from .sharding import shard_network_ranges
    B = len(networks)
    kins = list(kin) if isinstance(kin, (list, tuple)) else None
    cns = list(cell_num) if isinstance(cell_num, (list, tuple, np.ndarray)) else [int(cell_num)] * B
    pops = list(populations) if populations is not None else [None] * B
    sizes = [pops[b].cell_num if pops[b] is not None else cns[b] for b in range(B)]
    ranges = shard_network_ranges([networks[b].G * sizes[b] for b in range(B)], len(contexts))

    def run(k):
        lo, hi = ranges[k]
        if hi <= lo:
            return ([], []) if capture is not None else []
        return simulate_gpu_batch(networks[lo:hi], alg, kins[lo:hi] if kins is not None else kin,
                                  cell_num=cns[lo:hi], T=T, readout=readout, seed=seed, stream=stream + lo,
                                  populations=pops[lo:hi], capture=capture, ctx=contexts[k])

    with ThreadPoolExecutor(max_workers=len(contexts)) as ex:
        parts = list(ex.map(run, range(len(contexts))))
    if capture is not None:
        return [x for p in parts for x in p[0]], [x for p in parts for x in p[1]]
    return [x for p in parts for x in p]


def apply_capture(X: np.ndarray, capture: CaptureModel, *, seed: int = 0, stream: int = 0,
                  ctx: Optional[Context] = None, return_efficiencies: bool = False):
    """GPU LogNormal-Binomial capture of a cells x G molecule matrix (capture.jl:25-47)."""
    ctx = ctx or default_context()
    Xf = np.asfortranarray(X, dtype=np.float64)
    N, G = Xf.shape
    Y = np.empty((N, G), dtype=np.int32, order="F")
    eff = np.empty(N, dtype=np.float64)
    c = _cap(capture)
    check(ctx.lib.scrna_apply_capture(ctx.h, N, G, Xf.ctypes.data, C.byref(c), int(seed), int(stream),
                                      Y.ctypes.data, eff.ctypes.data))
    return (Y, eff) if return_efficiencies else Y


class DeviceRun:
    """Device-resident run of one network (scrna_state): `launch()` enqueues a whole
    simulation on the context stream without host traffic; `read()` fetches results."""

    def __init__(self, net: GeneNetwork, alg, kin: KineticParams, *, cell_num: int, T: float,
                 readout: str = "protein", seed: int = 0, stream: int = 0,
                 capture: Optional[CaptureModel] = None, population: Optional[PopulationConfig] = None,
                 precision: str = "fp32", n_steps: int = 0, cell_offset: int = 0,
                 path: str = "auto", ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self.handle = NetHandle(net, self.ctx)
        self.N = population.cell_num if population is not None else cell_num
        self.G = net.G
        self.readout = readout
        self.capture = capture
        self.k, self.p, self.c = _kin(kin), _pop(population), _cap(capture)
        self.tau = _is_tau(alg)
        self.o = _opts(alg, T=T, cell_num=self.N, readout=readout, seed=seed, stream=stream,
                       precision=precision, path=path, n_steps=n_steps, cell_offset=cell_offset)
        h = C.c_void_p()
        check(self.ctx.lib.scrna_state_create(self.ctx.h, self.handle.h, self.N, READOUT[readout],
                                              int(capture is not None), C.byref(h)))
        self.st = h

    def launch(self):
        fn = self.ctx.lib.scrna_tauleap_run_device if self.tau else self.ctx.lib.scrna_cle_run_device
        check(fn(self.ctx.h, self.handle.h, C.byref(self.k), _ptr(self.p), _ptr(self.c), C.byref(self.o), self.st))

    def resume(self, *, T: Optional[float] = None, n_steps: int = 0):
        """Continue the held run to T (or n_steps) steps in total from its current step; the
        results equal one run of that length."""
        o = _opts(BinomialTauLeap(self.o.dt) if self.tau else CLE(self.o.dt), T=self.o.T if T is None else T,
                  cell_num=self.N, readout=self.readout, seed=self.o.seed, stream=self.o.stream,
                  precision="fp32", path=[k for k, v in PATH.items() if v == self.o.path][0], n_steps=n_steps,
                  cell_offset=self.o.cell_offset)
        fn = self.ctx.lib.scrna_tauleap_resume if self.tau else self.ctx.lib.scrna_cle_resume
        check(fn(self.ctx.h, self.handle.h, C.byref(self.k), _ptr(self.p), _ptr(self.c), C.byref(o), self.st))

    @property
    def steps_done(self) -> int:
        v = C.c_int64()
        check(self.ctx.lib.scrna_state_steps_done(self.st, C.byref(v)))
        return int(v.value)

    def checkpoint(self) -> bytes:
        """The held run's state as bytes (scrna_state_checkpoint)."""
        n = C.c_size_t()
        check(self.ctx.lib.scrna_state_checkpoint(self.ctx.h, self.st, None, 0, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        check(self.ctx.lib.scrna_state_checkpoint(self.ctx.h, self.st, buf, n.value, C.byref(n)))
        return buf.raw

    def restore(self, data: bytes):
        """Load a checkpoint (of the same G and cell count) to continue with resume()."""
        buf = C.create_string_buffer(bytes(data), len(data))
        check(self.ctx.lib.scrna_state_restore(self.ctx.h, self.st, buf, len(data)))

    def read(self):
        cols = self.G * (2 if self.readout == "both" else 1)
        out = _pinned.empty((self.N, cols), np.float64, order="F")
        counts = eff = None
        if self.capture is not None:
            counts = _pinned.empty((self.N, self.G), np.int32, order="F")
            eff = _pinned.empty(self.N, np.float64)
        check(self.ctx.lib.scrna_state_read(self.ctx.h, self.st, out.ctypes.data,
                                            None if counts is None else counts.ctypes.data,
                                            None if eff is None else eff.ctypes.data))
        return (out, counts, eff) if self.capture is not None else out

    def read_raw(self):
        """Raw state of the last run: dict with M, P ([G, N]; float32, or float64 for the
        FP64 baseline), prom ([G, N] uint8) and V ([N], population runs)."""
        dt = np.float64 if self.o.precision == PRECISION["fp64_plain"] else np.float32
        M = np.empty((self.G, self.N), dtype=dt)
        Pm = np.empty((self.G, self.N), dtype=dt)
        prom = np.empty((self.G, self.N), dtype=np.uint8)
        V = np.empty(self.N, dtype=np.float64) if self.p is not None else None
        check(self.ctx.lib.scrna_state_read_raw(self.ctx.h, self.st, M.ctypes.data, Pm.ctypes.data,
                                                prom.ctypes.data, None if V is None else V.ctypes.data))
        out = {"M": M, "P": Pm, "prom": prom}
        if V is not None:
            out["V"] = V
        return out

    def moments(self, source: str = "readout"):
        """Per-column (mean, unbiased variance) of the last run's readout or captured counts,
        reduced on the device (FP64)."""
        src = _SOURCE[source]
        cols = self.G * (2 if (src == 0 and self.readout == "both") else 1)
        mean = np.empty(cols)
        var = np.empty(cols)
        check(self.ctx.lib.scrna_state_moments(self.ctx.h, self.st, src, mean.ctypes.data, var.ctypes.data))
        return mean, var

    def histogram(self, column: int, nbins: int, source: str = "readout") -> np.ndarray:
        """Counts of one column's values rounded to integers, clamped to [0, nbins - 1]."""
        h = np.empty(int(nbins), dtype=np.int64)
        check(self.ctx.lib.scrna_state_histogram(self.ctx.h, self.st, _SOURCE[source], int(column), int(nbins),
                                                 h.ctypes.data))
        return h

    def compare_pmf(self, column: int, p_exact, source: str = "readout") -> dict:
        """L1 distance and KS statistic of one column's rounded values against an exact
        distribution P(0..L-1) (experiments/validate_telegraph.jl:80-125), from a histogram
        computed on the device: {"l1", "ks", "n"}."""
        from .validate import pmf_comparison_from_histogram
        return pmf_comparison_from_histogram(self.histogram(column, len(p_exact) + 1, source), p_exact)

    def write_mtx(self, directory: str, gene_names: Optional[Sequence[str]] = None, barcode_prefix: str = "cell"):
        """10x Matrix Market files (matrix.mtx, genes.tsv, barcodes.tsv) of the captured counts."""
        names = None
        if gene_names is not None:
            if len(gene_names) != self.G:
                raise ValueError(f"need {self.G} gene names")
            enc = [n.encode() for n in gene_names]
            names = (C.c_char_p * self.G)(*enc)
        check(self.ctx.lib.scrna_state_write_mtx(self.ctx.h, self.st, str(directory).encode(),
                                                 None if names is None else C.cast(names, C.c_void_p),
                                                 barcode_prefix.encode()))

    def device_state(self):
        """Device pointers of the FP32 mRNA / protein state: [G][N] after a block-kernel run,
        [N][G] after a lane-kernel run."""
        m, p = C.c_void_p(), C.c_void_p()
        check(self.ctx.lib.scrna_state_device_ptrs(self.st, C.byref(m), C.byref(p)))
        return m.value, p.value

    def close(self):
        if getattr(self, "st", None):
            if getattr(self.ctx, "h", None):
                self.ctx.lib.scrna_state_destroy(self.st)
            self.st = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_SOURCE = {"readout": 0, "counts": 1}


def ks_statistic_device(a: "DeviceRun", b: "DeviceRun", source: str = "readout") -> np.ndarray:
    """Per-column two-sample Kolmogorov-Smirnov statistic of two runs' last results, computed on
    the device (the walk of src/validate.jl:14-41)."""
    if a.ctx is not b.ctx:
        raise ValueError("both runs must belong to one context")
    src = _SOURCE[source]
    cols = a.G * (2 if (src == 0 and a.readout == "both") else 1)
    D = np.empty(cols)
    check(a.ctx.lib.scrna_state_ks(a.ctx.h, a.st, b.st, src, D.ctypes.data))
    return D


def debug_philox(ctr: np.ndarray, key, ctx: Optional[Context] = None) -> np.ndarray:
    ctx = ctx or default_context()
    c = np.ascontiguousarray(ctr, dtype=np.uint32).reshape(-1, 4)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.zeros_like(c)
    check(ctx.lib.scrna_debug_philox(ctx.h, c.shape[0], c.ctypes.data, k.ctypes.data, out.ctypes.data))
    return out


def debug_small_div_check(lo_bits: int, hi_bits: int, ctx: Optional[Context] = None):
    """(mismatches, first differing lam bits, its k) of the tau-leap's branch-free quotient
    lam / k against IEEE division over the floats with bit patterns in [lo_bits, hi_bits)."""
    ctx = ctx or default_context()
    n, lam, k = C.c_int64(), C.c_uint32(), C.c_int32()
    check(ctx.lib.scrna_debug_small_div_check(ctx.h, lo_bits, hi_bits, C.byref(n), C.byref(lam), C.byref(k)))
    return n.value, lam.value, k.value


def measure_philox_rate(ctx: Optional[Context] = None) -> float:
    """Philox4x32-10 generator calls per second, measured by the library's microkernel."""
    ctx = ctx or default_context()
    r = C.c_double()
    check(ctx.lib.scrna_measure_philox_rate(ctx.h, C.byref(r)))
    return r.value


def measure_pipe_peaks(ctx: Optional[Context] = None):
    """(fma_ops/s, sfu_ops/s, int_ops/s) measured by the library's microkernels."""
    ctx = ctx or default_context()
    a, b, c = C.c_double(), C.c_double(), C.c_double()
    check(ctx.lib.scrna_measure_pipe_peaks(ctx.h, C.byref(a), C.byref(b), C.byref(c)))
    return a.value, b.value, c.value


class Server:
    """Request server with continuous batching (scrna_server_*): requests are admitted by
    device footprint, keep their state on the GPU and advance in shared chunks of
    `chunk_steps` Euler steps; `wait` returns the same results `simulate` gives."""

    STATES = {0: "queued", 1: "running", 2: "done", 3: "failed", 4: "cancelled"}

    def __init__(self, ctx: Optional[Context] = None, *, hbm_budget_bytes: int = 0, chunk_steps: int = 250):
        self.ctx = ctx or default_context()
        h = C.c_void_p()
        check(self.ctx.lib.scrna_server_create(self.ctx.h, int(hbm_budget_bytes), int(chunk_steps), C.byref(h)))
        self.h = h
        self._meta = {}

    def submit(self, handle: NetHandle, alg: CLE, kin: KineticParams, *, cell_num: int, T: float = 50.0,
               readout: str = "protein", seed: int = 0, stream: int = 0, capture: Optional[CaptureModel] = None,
               n_steps: int = 0, cell_offset: int = 0) -> int:
        req = _lib.Request()
        req.net = handle.h
        req.kin = _kin(kin)
        req.opts = _opts(alg, T=T, cell_num=cell_num, readout=readout, seed=seed, stream=stream, precision="fp32",
                         path="auto", n_steps=n_steps, cell_offset=cell_offset)
        if capture is not None:
            req.with_capture = 1
            req.capture = _cap(capture)
        t = C.c_uint64()
        check(self.ctx.lib.scrna_submit(self.h, C.byref(req), C.byref(t)))
        self._meta[t.value] = (handle, int(cell_num), handle.G * (2 if readout == "both" else 1), capture is not None)
        return t.value

    def poll(self, ticket: int) -> str:
        st = C.c_int32()
        check(self.ctx.lib.scrna_poll(self.h, int(ticket), C.byref(st)))
        return self.STATES[st.value]

    def wait(self, ticket: int, timeout_ms: int = -1):
        """(readout, counts, efficiencies, latency_s); counts/efficiencies are None without capture."""
        handle, N, cols, cap = self._meta[ticket]
        # one-off sizes: pageable (pinning a fresh block costs more than the copy it saves)
        out = np.empty((N, cols), dtype=np.float64, order="F")
        counts = np.empty((N, handle.G), dtype=np.int32, order="F") if cap else None
        eff = np.empty(N, dtype=np.float64) if cap else None
        lat = C.c_double()
        check(self.ctx.lib.scrna_wait(self.h, int(ticket), int(timeout_ms), out.ctypes.data,
                                      None if counts is None else counts.ctypes.data,
                                      None if eff is None else eff.ctypes.data, C.byref(lat)))
        del self._meta[ticket]
        return out, counts, eff, lat.value

    def cancel(self, ticket: int):
        check(self.ctx.lib.scrna_cancel(self.h, int(ticket)))

    def stats(self) -> dict:
        s = _lib.ServerStats()
        check(self.ctx.lib.scrna_server_get_stats(self.h, C.byref(s)))
        return {n: getattr(s, n) for n, _ in s._fields_}

    def trace(self) -> List[dict]:
        """The most recent chunks (oldest first): t_start / t_end on the server's clock
        (seconds since creation), requests, kernel groups and cell·gene·steps of each."""
        n = C.c_int32()
        check(self.ctx.lib.scrna_server_trace(self.h, None, 0, C.byref(n)))
        recs = (_lib.ChunkRecord * max(n.value, 1))()
        check(self.ctx.lib.scrna_server_trace(self.h, recs, n.value, C.byref(n)))
        return [{f: getattr(recs[i], f) for f, _ in _lib.ChunkRecord._fields_} for i in range(n.value)]

    def close(self):
        if getattr(self, "h", None):
            if getattr(self.ctx, "h", None):
                self.ctx.lib.scrna_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def least_loaded(loads: Sequence[float]) -> int:
    """Index of the smallest outstanding load (the first of equal ones)."""
    best = 0
    for i, x in enumerate(loads):
        if x < loads[best]:
            best = i
    return best


class ServerPool:
    """One Server per context (normally one context per GPU): each request goes to the server
    with the fewest outstanding cell·gene·steps (submitted, not yet done), so a request stream
    larger than one GPU's compute spreads over the devices.  Requests are independent and each
    runs wholly on one device, so results equal `simulate`'s whichever server takes them."""

    def __init__(self, contexts: Sequence[Context], *, hbm_budget_bytes: int = 0, chunk_steps: int = 250):
        if not contexts:
            raise ValueError("ServerPool needs at least one context")
        self.servers = [Server(c, hbm_budget_bytes=hbm_budget_bytes, chunk_steps=chunk_steps) for c in contexts]
        self._submitted = [0] * len(self.servers)
        self._where = {}
        self._next = 1

    def loads(self) -> list:
        """Outstanding cell·gene·steps of each server."""
        return [self._submitted[i] - s.stats()["units_done"] for i, s in enumerate(self.servers)]

    def submit(self, net: GeneNetwork, alg: CLE, kin: KineticParams, *, cell_num: int, T: float = 50.0,
               n_steps: int = 0, **kw) -> int:
        i = least_loaded(self.loads())
        srv = self.servers[i]
        t = srv.submit(_handle_for(net, srv.ctx), alg, kin, cell_num=cell_num, T=T, n_steps=n_steps, **kw)
        steps = n_steps if n_steps > 0 else n_steps_of(T, alg.dt)
        self._submitted[i] += net.G * int(cell_num) * steps
        ticket = self._next
        self._next += 1
        self._where[ticket] = (i, t)
        return ticket

    def server_of(self, ticket: int) -> int:
        return self._where[ticket][0]

    def poll(self, ticket: int) -> str:
        i, t = self._where[ticket]
        return self.servers[i].poll(t)

    def wait(self, ticket: int, timeout_ms: int = -1):
        i, t = self._where[ticket]
        out = self.servers[i].wait(t, timeout_ms)
        del self._where[ticket]
        return out

    def cancel(self, ticket: int):
        i, t = self._where[ticket]
        self.servers[i].cancel(t)

    def stats(self) -> dict:
        per = [s.stats() for s in self.servers]
        tot = {k: sum(p[k] for p in per) for k in per[0]}
        tot["busy_s_max"] = max(p["busy_s"] for p in per)
        tot["per_server"] = per
        return tot

    def close(self):
        for s in self.servers:
            s.close()
