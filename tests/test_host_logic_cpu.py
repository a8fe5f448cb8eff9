"""Host-side logic that needs no GPU: the size-bucket autotuner's choices and
the bench's roofline bookkeeping (algorithmic bytes, issue fraction, ncu
profile entries tied to the grid they were captured with)."""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import ts_b200 as T  # noqa: E402
from ts_b200 import autotune as AT  # noqa: E402


def test_autotuner_keeps_the_fastest_feasible_shape(monkeypatch):
    # synthetic rates: the tile pass is faster from the third bucket up, and
    # cluster 4 never fits -- it must be recorded and never chosen
    def fake_trial(problem, n, kind, cluster, jobs, iters, seed, sweep=T.PASS_AUTO):
        if cluster == 4:
            raise T.TsError(4, "ts_batch_create", "a cluster of 4 CTAs does not fit on the device")
        base = {"csr": 3.0, "hash": 1.0, "csr-bb": 2.0, "wswap": 2.5}[kind] * n
        if sweep == T.PASS_TILE:
            base *= 2.0 if n > 2000 else 0.5
        return base * (1.0 + 0.1 * cluster)

    monkeypatch.setattr(AT, "_trial", fake_trial)
    table = AT.autotune(budget_s=1e9)
    for (problem, b), c in table.choice.items():
        n = int(np.sqrt(AT.DEFAULT_BUCKETS[b][0] * (AT.DEFAULT_BUCKETS[b][1] - 1)))
        assert c.cluster == 2 and c.kind == "csr"
        assert c.sweep == (T.PASS_TILE if n > 2000 else T.PASS_ROWS)
    bad = [t for t in table.trials if "unavailable" in t]
    assert bad and all(t["cluster"] == 4 for t in bad)
    assert all("does not fit" in t["unavailable"] for t in bad)
    assert not any(t.get("structure") == "wswap" and t.get("sweep") == T.PASS_TILE for t in table.trials)
    d = table.as_dict()
    assert len(d) == 2 * len(AT.DEFAULT_BUCKETS) and all(v["sweep"] in ("tile", "rows") for v in d.values())


def test_autotuner_budget_is_shared_between_buckets(monkeypatch):
    calls = []

    def slow_trial(problem, n, kind, cluster, jobs, iters, seed, sweep=T.PASS_AUTO):
        calls.append((problem, n))
        import time
        time.sleep(0.02)
        return 1.0

    monkeypatch.setattr(AT, "_trial", slow_trial)
    table = AT.autotune(budget_s=0.0)  # every bucket still gets one timed candidate
    assert len(table.choice) == 2 * len(AT.DEFAULT_BUCKETS)
    assert len(calls) == 2 * len(AT.DEFAULT_BUCKETS)


def test_algorithmic_bytes_and_issue_fraction():
    import bench
    n, m = 1000, 100
    ldc = (n - m + 3) // 4 * 4
    deg = np.full(m, 10, np.int64)
    cap = np.full(m, 32, np.int64)
    base = m * (4 + 8) + (n - m) * (4 + 4)
    assert bench.algorithmic_bytes("csr", n, m, ldc, 4, deg, cap, 16) == base + 16 * m + 12 * 1000
    assert bench.algorithmic_bytes("hash", n, m, ldc, 4, deg, cap, 16) == base + 4 * (n - m) + 16 * m + 8 * 3200
    assert bench.algorithmic_bytes("wswap", n, m, ldc, 4, deg, cap, 16, w_bytes=2) == base + 2 * m * ldc
    assert bench.algorithmic_bytes("csr-bitset", n, m, ldc, 4, deg, cap, 16) == base + 4 * (n - m) + 8 * m * 16
    # 148 SMs x 4 schedulers x 1 GHz issue 5.92e11 warp instructions per second
    assert bench.issue_fraction(5.92e8, 1e-3, 1000.0) == pytest.approx(1.0)
    assert bench._hash_cap(0) == 8 and bench._hash_cap(5) == 16 and bench._hash_cap(64) == 128


def test_profile_entries_apply_only_to_their_grid(tmp_path, monkeypatch):
    import bench
    prof = tmp_path / "profiles"
    prof.mkdir()
    (prof / "dram_traffic.json").write_text(json.dumps(
        {"config2": {"hash": {"grid": 1563, "bytes": 8.0e7, "warp_inst": 3.0e8}}}))
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    assert bench.profile_entry("config2", "hash", 1563)["bytes"] == 8.0e7
    assert bench.profile_entry("config2", "hash", 3125) is None  # another tile shape: not this kernel
    assert bench.profile_entry("config3", "hash", 1563) is None
    assert bench.profile_entry("config2", "csr", 1563) is None
