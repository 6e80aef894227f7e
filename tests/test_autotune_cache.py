"""The autotuner's persisted cache on CPU (no device needed): the key of a network shape,
a miss, a store and a hit, entries kept when another writer (another process) adds its own,
and a damaged file read as empty instead of failing a run."""
import ctypes as C
import json
import subprocess
import sys

import pytest


def _choice(pkg, kernel=1, gpl=2, warps=4, us=0.5):
    c = pkg._lib.TuneChoice()
    c.kernel, c.genes_per_lane, c.block_warps, c.us_per_step = kernel, gpl, warps, us
    return c


def _lookup(lib, pkg, path, key):
    c = pkg._lib.TuneChoice()
    pkg._lib.check(lib.scrna_autotune_cache_lookup(str(path).encode(), key, C.byref(c)))
    return c


def _key(lib, pkg, G, emax, terms, bursty, hill2, N, device=b"sm100x148"):
    buf = C.create_string_buffer(160)
    pkg._lib.check(lib.scrna_autotune_key(device, G, emax, terms, bursty, hill2, N, buf, 160))
    return buf.value


def test_key_buckets_cell_counts(pkg):
    lib = pkg._lib.load()
    k = _key(lib, pkg, 10, 4, 2, 1, 1, 20000)
    assert k == b"sm100x148|G10|e4|t2|b1|h1|N14"
    assert _key(lib, pkg, 10, 4, 2, 1, 1, 16384) == k      # same power-of-two bucket
    assert _key(lib, pkg, 10, 4, 2, 1, 1, 40000) != k
    assert _key(lib, pkg, 11, 4, 2, 1, 1, 20000) != k
    assert lib.scrna_autotune_key(b"sm100", 0, 4, 0, 0, 1, 10, C.create_string_buffer(8), 8) == -1


def test_miss_store_hit_and_file_format(pkg, tmp_path):
    lib = pkg._lib.load()
    path = tmp_path / "sub" / "autotune.json"
    key = _key(lib, pkg, 10, 4, 2, 1, 1, 20000)
    assert _lookup(lib, pkg, path, key).found == 0
    pkg._lib.check(lib.scrna_autotune_cache_store(str(path).encode(), key, C.byref(_choice(pkg, 1, 2, 8, 0.71))))
    got = _lookup(lib, pkg, path, key)
    assert (got.found, got.kernel, got.genes_per_lane, got.block_warps) == (1, 1, 2, 8)
    assert abs(got.us_per_step - 0.71) < 1e-9
    data = json.load(open(path))
    assert data["version"] == 1 and data["entries"][key.decode()]["block_warps"] == 8
    assert _lookup(lib, pkg, path, b"sm100x148|G11|e4|t2|b1|h1|N14").found == 0
    bad = _choice(pkg, kernel=7)
    assert lib.scrna_autotune_cache_store(str(path).encode(), key, C.byref(bad)) == -1


def test_entries_of_another_process_are_kept(pkg, tmp_path):
    lib = pkg._lib.load()
    path = tmp_path / "autotune.json"
    k1 = _key(lib, pkg, 10, 4, 2, 1, 1, 20000)
    pkg._lib.check(lib.scrna_autotune_cache_store(str(path).encode(), k1, C.byref(_choice(pkg, 0, 0, 0, 1.5))))
    # another process adds an entry to the same file
    code = (
        "import ctypes as C, sys; sys.path.insert(0, %r); import __graft_entry__ as g; pkg = g.load_package(); "
        "lib = pkg._lib.load(); c = pkg._lib.TuneChoice(); c.kernel, c.genes_per_lane, c.block_warps = 1, 4, 2; "
        "pkg._lib.check(lib.scrna_autotune_cache_store(%r, b'sm100x148|G500|e4|t0|b0|h1|N10', C.byref(c)))"
        % (str(pkg.__path__[0]).rsplit("/", 1)[0], str(path).encode()))
    subprocess.run([sys.executable, "-c", code], check=True)
    k2 = b"sm100x148|G500|e4|t0|b0|h1|N10"
    got = _lookup(lib, pkg, path, k2)  # a miss in memory re-reads the file
    assert (got.found, got.kernel, got.genes_per_lane, got.block_warps) == (1, 1, 4, 2)
    k3 = _key(lib, pkg, 33, 8, 1, 0, 1, 500)
    pkg._lib.check(lib.scrna_autotune_cache_store(str(path).encode(), k3, C.byref(_choice(pkg, 1, 2, 4, 0.2))))
    entries = json.load(open(path))["entries"]
    assert set(entries) == {k1.decode(), k2.decode(), k3.decode()}


@pytest.mark.parametrize("content", ["", "not json", '{"version": 2, "entries": {}}', '{"entries": {"k": {'])
def test_damaged_file_reads_as_empty(pkg, tmp_path, content):
    lib = pkg._lib.load()
    path = tmp_path / "autotune.json"
    path.write_text(content)
    key = _key(lib, pkg, 10, 4, 2, 1, 1, 20000)
    assert _lookup(lib, pkg, path, key).found == 0
    pkg._lib.check(lib.scrna_autotune_cache_store(str(path).encode(), key, C.byref(_choice(pkg))))
    assert _lookup(lib, pkg, path, key).found == 1
    assert json.load(open(path))["version"] == 1
