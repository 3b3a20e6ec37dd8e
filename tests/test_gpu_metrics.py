"""Per-commit / per-request JSON-lines metrics (PICO_METRICS_LOG) and the
autotuner's cache file (PICO_TUNE_CACHE), on the GPU."""
import json

import numpy as np
import pytest

from pico_b200 import CommitServer, GpuContext, TwoAdicDomain, TwoAdicFriPcs
from pico_b200 import fields as F

pytestmark = pytest.mark.gpu


def test_metrics_log_records_commits_and_requests(gpu, tmp_path, monkeypatch):
    log = tmp_path / "metrics.jsonl"
    monkeypatch.setenv("PICO_METRICS_LOG", str(log))
    f = 0
    mats = [F.random_matrix(f, 10, 7, 9400), F.random_matrix(f, 8, 3, 9401)]
    TwoAdicFriPcs(gpu, f, 1).commit([(TwoAdicDomain(10), mats[0]), (TwoAdicDomain(8), mats[1])], keep=False)
    req = CommitServer(gpu).submit(f, mats, 1)
    req.wait(keep=False)
    req.free()
    lines = [json.loads(l) for l in log.read_text().splitlines()]
    assert [l["kind"] for l in lines] == ["commit", "request"]
    for l in lines:
        assert l["cells"] == (7 << 10) + (3 << 8) and l["lde_cells"] == 2 * l["cells"]
        assert l["field"] == "koalabear" and l["matrices"] == 2 and l["log_blowup"] == 1
        assert l["total_ms"] > 0 and l["launches"] > 0
    assert lines[1]["queued_us"] >= 0 and lines[1]["run_us"] > 0


def test_tune_cache_is_written_then_reused(tmp_path, monkeypatch):
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("PICO_TUNE_CACHE", str(cache))
    with GpuContext(0) as ctx:
        first = ctx.autotune(0, 12, 14)
    text = cache.read_text().splitlines()
    assert len(text) == 4  # three heights and the hash block
    with GpuContext(0) as ctx:
        second = ctx.autotune(0, 12, 14)
        for l in (12, 13, 14):
            assert second[l].get("cached") and second[l]["log_n1"] == first[l]["log_n1"]
            assert ctx.lde_split(0, l) == first[l]["log_n1"]
        assert second.get("hash_block_cached")
    assert cache.read_text().splitlines() == text  # nothing re-timed, nothing appended
