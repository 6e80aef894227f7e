"""ctypes binding of libscrna_cle.so (declarations in include/scrna_cle.h).

The library is the only compute path: if it cannot be loaded, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

from . import build as _build

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libscrna_cle.so")

_lock = threading.Lock()
_lib = None


class ScrnaError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"scrna error {code}: {msg}")
        self.code = code


class Kinetics(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("k_t", "K_d", "n", "mu_m", "mu_p", "dilution")]


class Population(C.Structure):
    _fields_ = [("cell_num", C.c_int64), ("growth_rate", C.c_double), ("V_div", C.c_double),
                ("V_init_lo", C.c_double), ("V_init_hi", C.c_double),
                ("div_check_interval", C.c_int32), ("partition", C.c_int32),
                ("exclude_mother", C.c_int32), ("reserved", C.c_int32),
                ("growth_noise", C.c_double)]


class Capture(C.Structure):
    _fields_ = [("efficiency", C.c_double), ("efficiency_std", C.c_double),
                ("readout", C.c_int32), ("mean_correction", C.c_int32)]


class Opts(C.Structure):
    _fields_ = [("dt", C.c_double), ("T", C.c_double), ("cell_num", C.c_int64),
                ("readout", C.c_int32), ("precision", C.c_int32), ("seed", C.c_uint64),
                ("stream", C.c_uint32), ("path", C.c_int32), ("n_steps", C.c_int64),
                ("cell_offset", C.c_int64)]


class Request(C.Structure):
    _fields_ = [("net", C.c_void_p), ("kin", Kinetics), ("opts", Opts), ("with_capture", C.c_int32),
                ("reserved", C.c_int32), ("capture", Capture)]


class TuneChoice(C.Structure):
    _fields_ = [("kernel", C.c_int32), ("genes_per_lane", C.c_int32), ("block_warps", C.c_int32),
                ("found", C.c_int32), ("us_per_step", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [(n, C.c_int64) for n in ("submitted", "completed", "failed", "queued", "running",
                                          "units_done", "bytes_in_use")] + \
               [("busy_s", C.c_double), ("chunks", C.c_int64)]


class ChunkRecord(C.Structure):
    _fields_ = [("t_start", C.c_double), ("t_end", C.c_double), ("requests", C.c_int32), ("groups", C.c_int32),
                ("units", C.c_int64)]


P = C.c_void_p
I32, I64, U32, U64, DBL = C.c_int32, C.c_int64, C.c_uint32, C.c_uint64, C.c_double

# name -> (restype, argtypes); every function the header declares.
SIGNATURES = {
    "scrna_last_error": (C.c_char_p, []),
    "scrna_version": (C.c_int, []),
    "scrna_ctx_create": (C.c_int, [C.c_int, C.POINTER(P)]),
    "scrna_ctx_destroy": (C.c_int, [P]),
    "scrna_ctx_set_stream": (C.c_int, [P, P]),
    "scrna_ctx_synchronize": (C.c_int, [P]),
    "scrna_ctx_launch_count": (C.c_int64, [P]),
    "scrna_ctx_transfer_bytes": (C.c_int, [P, C.POINTER(I64), C.POINTER(I64)]),
    "scrna_net_create": (C.c_int, [P, I32, P, P, I32, P, P, P, P, I32, P, P, P, P, P, P, I32,
                                   C.POINTER(P)]),
    "scrna_net_destroy": (C.c_int, [P]),
    "scrna_net_genes": (C.c_int32, [P]),
    "scrna_cle_simulate": (C.c_int, [P, P, P, P, P, P, P, P, P]),
    "scrna_cle_simulate_batch": (C.c_int, [P, I32, P, P, I32, P, P, P, P, P, P]),
    "scrna_apply_capture": (C.c_int, [P, I64, I32, P, P, U64, U32, P, P]),
    "scrna_tauleap_simulate": (C.c_int, [P, P, P, P, P, P, P, P, P]),
    "scrna_tauleap_simulate_batch": (C.c_int, [P, I32, P, P, I32, P, P, P, P, P, P]),
    "scrna_tauleap_run_device": (C.c_int, [P, P, P, P, P, P, P]),
    "scrna_state_create": (C.c_int, [P, P, I64, I32, I32, C.POINTER(P)]),
    "scrna_state_destroy": (C.c_int, [P]),
    "scrna_cle_run_device": (C.c_int, [P, P, P, P, P, P, P]),
    "scrna_state_read": (C.c_int, [P, P, P, P, P]),
    "scrna_state_device_ptrs": (C.c_int, [P, C.POINTER(P), C.POINTER(P)]),
    "scrna_state_read_raw": (C.c_int, [P, P, P, P, P, P]),
    "scrna_cle_simulate_noalloc": (C.c_int, [P, P, P, P, P, P, P, P, P]),
    "scrna_ctx_set_autotune": (C.c_int, [P, I32, C.c_char_p]),
    "scrna_autotune_last_choice": (C.c_int, [P, C.POINTER(TuneChoice)]),
    "scrna_autotune_key": (C.c_int, [C.c_char_p, I32, I32, I32, I32, I32, I64, C.c_char_p, I32]),
    "scrna_autotune_cache_lookup": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(TuneChoice)]),
    "scrna_autotune_cache_store": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(TuneChoice)]),
    "scrna_state_moments": (C.c_int, [P, P, I32, P, P]),
    "scrna_state_ks": (C.c_int, [P, P, P, I32, P]),
    "scrna_state_histogram": (C.c_int, [P, P, I32, I32, I32, P]),
    "scrna_state_write_mtx": (C.c_int, [P, P, C.c_char_p, P, C.c_char_p]),
    "scrna_cle_resume": (C.c_int, [P, P, P, P, P, P, P]),
    "scrna_tauleap_resume": (C.c_int, [P, P, P, P, P, P, P]),
    "scrna_state_steps_done": (C.c_int, [P, C.POINTER(I64)]),
    "scrna_state_checkpoint": (C.c_int, [P, P, P, C.c_size_t, C.POINTER(C.c_size_t)]),
    "scrna_state_restore": (C.c_int, [P, P, P, C.c_size_t]),
    "scrna_server_create": (C.c_int, [P, I64, I32, C.POINTER(P)]),
    "scrna_server_destroy": (C.c_int, [P]),
    "scrna_submit": (C.c_int, [P, P, C.POINTER(U64)]),
    "scrna_poll": (C.c_int, [P, U64, C.POINTER(I32)]),
    "scrna_wait": (C.c_int, [P, U64, I32, P, P, P, C.POINTER(DBL)]),
    "scrna_cancel": (C.c_int, [P, U64]),
    "scrna_server_get_stats": (C.c_int, [P, P]),
    "scrna_server_trace": (C.c_int, [P, P, I32, P]),
    "scrna_debug_philox": (C.c_int, [P, I32, P, P, P]),
    "scrna_debug_small_div_check": (C.c_int, [P, U32, U32, P, P, P]),
    "scrna_debug_tc_gemm": (C.c_int, [P, P, P, P, I64, I32, I32, I32]),
    "scrna_debug_tc_gemm_withhold": (C.c_int, [P, P, P, P, I64, I32, I32, I32, I32]),
    "scrna_measure_pipe_peaks": (C.c_int, [P, C.POINTER(DBL), C.POINTER(DBL), C.POINTER(DBL)]),
    "scrna_measure_philox_rate": (C.c_int, [P, C.POINTER(DBL)]),
    "scrna_host_alloc": (C.c_int, [C.c_size_t, C.POINTER(C.c_void_p)]),
    "scrna_host_free": (C.c_int, [P]),
}


def load(build_if_missing: bool = True):
    """Load (building first if needed) and return the library handle."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if build_if_missing and not os.path.exists(LIB_PATH):
            _build.build()
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing; build it with python -m build or __graft_entry__.build()")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
        return lib


def check(rc: int):
    if rc != 0:
        msg = load().scrna_last_error()
        raise ScrnaError(rc, msg.decode() if msg else "")
    return rc
