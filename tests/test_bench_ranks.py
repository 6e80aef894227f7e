"""bench.py's multi-rank plumbing on CPU (gloo, world size 2): `--gpus N` without a torchrun
environment starts N ranks itself, every rank sees WORLD_SIZE = N, the timing reduction is
the max over ranks, and a rank count that differs from --gpus stops the run."""
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_spawn_ranks_starts_n_ranks(tmp_path, monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        monkeypatch.delenv(k, raising=False)
    probe = os.path.join(ROOT, "tests", "helpers", "rank_probe.py")
    rc = bench.spawn_ranks(2, script=probe, argv=[str(tmp_path), "2"])
    assert rc == 0
    got = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    assert [g["world"] for g in got] == [2, 2]
    assert [g["max"] for g in got] == [2.0, 2.0]


def test_rank_count_must_match_gpus():
    bench.check_world(1, 1)
    with pytest.raises(SystemExit):
        bench.check_world(2, 1)
    assert bench.max_over_ranks(3.5, 1) == 3.5
