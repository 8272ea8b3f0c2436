"""Shard scans (ws_scan_shard) on one GPU with the multi-GPU chain protocol:
every shard of the input scanned with its halo, regex chains resumed from the
previous shard's cursors; the union equals one scan of the whole input."""
import numpy as np
import pytest

import oracle
import workloads as w
from test_multi_gpu_cpu import PATTERNS, _data

pytestmark = pytest.mark.gpu

PLAIN, SPEC = 1, 0


def matcher(patterns, mode=SPEC):
    import warpstate_b200 as ws
    b = ws.PatternSet.builder()
    for kind, p in patterns:
        b = b.literal_bytes(p) if kind == 0 else b.regex(p.decode() if isinstance(p, bytes) else p)
    return ws.GpuMatcher.with_config(b.build(), ws.AutoMatcherConfig().regex_mode(mode))


@pytest.mark.parametrize("mode", [PLAIN, SPEC])
def test_shards_equal_whole_scan_with_crossing_chains(mode):
    from warpstate_b200 import multi_gpu as mg
    data = _data()
    m = matcher(PATTERNS, mode)
    whole = oracle.scan_patterns(PATTERNS, data).astype(np.uint64)
    assert np.array_equal(m.scan_array(data).astype(np.uint64), whole)
    for n in (2, 3, 5):
        assert np.array_equal(mg.sharded_scan_local(m, data, n), whole), n


def test_shards_regex_workload():
    from warpstate_b200 import multi_gpu as mg
    wl = w.regex(size=4 << 20, n=100, seed=51)
    pats = wl.patterns + w.literals_large(size=1 << 10, n=300, seed=52).patterns
    m = matcher(pats)
    whole = oracle.scan_patterns(pats, wl.data).astype(np.uint64)
    assert len(whole) > 100
    for n in (2, 4):
        assert np.array_equal(mg.sharded_scan_local(m, wl.data, n), whole), n


def test_multi_gpu_matcher_concurrent_shards():
    # MultiGpuMatcher (core/src/multi_gpu.rs:33-160): shards scanned at the
    # same time from host threads, then the cursor exchange; here every shard
    # is on device 0 (each thread its own stream), which is how one GPU runs
    # the multi-device driver without any kernel waiting for another
    import warpstate_b200 as ws
    from warpstate_b200 import multi_gpu as mg
    data = _data()
    b = ws.PatternSet.builder()
    for kind, p in PATTERNS:
        b = b.literal_bytes(p) if kind == 0 else b.regex(p.decode() if isinstance(p, bytes) else p)
    ps = b.build()
    whole = oracle.scan_patterns(PATTERNS, data).astype(np.uint64)
    for n in (1, 2, 4):
        mm = mg.MultiGpuMatcher(ps, devices=[0] * n)
        assert mm.device_count() == n
        assert np.array_equal(mm.scan_array(data), whole), n
        assert np.array_equal(mm.scan_array(data), whole), n  # scanners are reused
