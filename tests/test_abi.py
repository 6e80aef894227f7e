"""The C ABI: every function include/scrna_cle.h declares is exported by the
library, and the Python binding declares exactly those functions.  No GPU needed:
loading the library does not touch the device."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "scrna_cle.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*(scrna_[a-z0-9_]+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("scrna_ctx_create", "scrna_net_create", "scrna_cle_simulate", "scrna_cle_simulate_batch",
                 "scrna_apply_capture", "scrna_cle_run_device", "scrna_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol(pkg):
    from importlib import import_module
    lib = pkg._lib.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_matches_header(pkg):
    assert sorted(pkg._lib.SIGNATURES) == declared_functions()


def test_version_and_error_without_gpu(pkg):
    lib = pkg._lib.load()
    assert lib.scrna_version() == 1
    h = ctypes.c_void_p()
    # On a machine without a GPU the context cannot be created; the call must fail cleanly.
    rc = lib.scrna_ctx_create(0, ctypes.byref(h))
    if rc != 0:
        assert lib.scrna_last_error()
