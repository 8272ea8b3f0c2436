#!/usr/bin/env python
"""Scan-path benchmark: one JSON line on rank 0.

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config NAME]

A "step" is one scan of the configuration's whole input (already resident in
HBM) by the full pattern set.  The default configuration is the 500-regex
scan over 1 GiB of Markov text (learned-speculative DFA walk, with the plain
thread-per-start kernel timed beside it).  Other configurations:
literals_large (10,000 literals over 1 GiB), literals_small (100 literals over
16 MiB), batch (200,000 lognormal items through the device batch scan) and dna
(4 GiB of ACGT through the 64-bit windowed device scan).  Under torchrun every
rank scans its own copy of the workload (weak scaling, no collective on the
data path); the reported time is the max over ranks.

--impl reference times the oracle port of the reference's CPU algorithm for
the same configuration on the host cores (the reference is a Rust crate with
un-vendored dependencies and a wgpu GPU path, neither runnable here).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import workloads as W  # noqa: E402

CONFIGS = {
    "regex": "500 regexes (2-4 literal alternations joined by [class]{1,8}), 1 GiB order-1 Markov printable ASCII",
    "literals_large": "10,000 literals (8-32 B, printable Zipf 1.1), 1 GiB order-1 Markov printable ASCII",
    "literals_small": "100 literals (4-16 B, a-z), 16 MiB iid a-z",
    "batch": "200,000 lognormal items (median 4 KiB, sigma 1.5), 1,500 literals + 500 regexes",
    "dna": "4 GiB ACGT with 1% N runs, 50,000 k-mers + 200 IUPAC regexes",
}
METRIC = "scan GB/s, learned-speculative vs plain DFA kernel, exact match sets, 1 B200"
CAP = 8 << 20  # device match capacity of the benchmark


def make_workload(name: str, size: int | None):
    if name == "regex":
        return W.regex(size=size or W.GiB)
    if name == "literals_large":
        return W.literals_large(size=size or W.GiB)
    if name == "literals_small":
        return W.literals_small(size=size or 16 * W.MiB)
    if name == "batch":
        return W.batch(n_items=size or 200_000)
    if name == "dna":
        return W.dna(size=size or 4 * W.GiB)
    raise SystemExit(f"unknown config {name}")


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def read_traffic(kernel: str, config: str):
    """DRAM bytes per launch from the committed ncu summary, if one exists."""
    p = ROOT / "profiles" / f"{kernel}_{config}.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.device), "-lms", "100", "-f", self.path],
                                         stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in Path(self.path).read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------- CPU baseline
def cpu_baseline(wl, seconds: float = 12.0):
    """Oracle port of the reference's CPU algorithm on a bounded sample of the
    same workload, all host threads.  Each call compiles the pattern set (a
    fixed cost of a few tenths of a second); the sample is sized from the rate
    between two probes, which cancels that cost, so that the timed scan runs
    about `seconds` and the compile is a small part of it."""
    import oracle
    threads = oracle.hw_threads()

    def size_for(run, p1, p2, total):
        t = time.perf_counter()
        run(p1)
        d1 = time.perf_counter() - t
        t = time.perf_counter()
        run(p2)
        d2 = time.perf_counter() - t
        rate = (p2 - p1) / max(d2 - d1, 1e-3) if p2 > p1 else p1 / max(d1, 1e-6)
        return int(min(total, max(p2, rate * seconds)))

    if wl.items is not None:
        items = wl.items

        def run_items(k, th=threads):
            oracle.batch_scan(wl.patterns, wl.data, items[:k], threads=th)

        k = size_for(run_items, min(len(items), 2000), min(len(items), 8000), len(items))
        t = time.perf_counter()
        run_items(k)
        dt = time.perf_counter() - t
        nbytes = sum(ln for _, ln in items[:k])
        return {"value": round(nbytes / dt / 1e9, 4), "unit": "GB/s", "cores": threads, "kind": "port",
                "sample": f"first {k} of {len(items)} items ({nbytes} bytes) scanned per item in {dt:.1f} s"}
    data = wl.data

    def run_bytes(n, th=threads):
        oracle.scan_patterns(wl.patterns, data[:n], th)

    n = size_for(run_bytes, min(len(data), 1 << 20), min(len(data), 16 << 20), min(len(data), 0xFFFFFFFF))
    t = time.perf_counter()
    run_bytes(n)
    dt = time.perf_counter() - t
    # one thread on a tenth of that sample
    n1 = max(min(len(data), 1 << 20), n // 10)
    t = time.perf_counter()
    run_bytes(n1, 1)
    dt1 = time.perf_counter() - t
    return {"value": round(n / dt / 1e9, 4), "unit": "GB/s", "cores": threads, "kind": "port",
            "sample": f"first {n} bytes of the same input ({n / dt / 1e6:.1f} MB/s over {dt:.1f} s)",
            "single_thread": {"value": round(n1 / dt1 / 1e9, 4), "unit": "GB/s", "sample": f"first {n1} bytes"}}


# ----------------------------------------------------------------- parity
MATCH64 = np.dtype([("pid", "<u4"), ("res", "<u4"), ("start", "<u8"), ("end", "<u8")])
TAGGED = np.dtype([("sid", "<u8"), ("pid", "<u4"), ("start", "<u4"), ("end", "<u4"), ("res", "<u4")])


def device_rows(d_out, count: int, kind: str) -> np.ndarray:
    """The device output of one scan as rows in the oracle's canonical order:
    (pattern_id, start, end) by (start, pattern_id, end), or for batches
    (source_id, pattern_id, start, end) by (source_id, start, pattern_id, end)."""
    import oracle
    if kind == "match":
        a = d_out.view(-1).view(__import__("torch").int32)[: count * 3].cpu().numpy().view(np.uint32)
        return oracle.sort_matches(a.reshape(-1, 3).copy())
    raw = d_out.view(-1).view(__import__("torch").uint8)[: count * 24].cpu().numpy()
    if kind == "match64":
        o = raw.view(MATCH64)
        a = np.empty((count, 3), dtype=np.uint64)
        a[:, 0], a[:, 1], a[:, 2] = o["pid"], o["start"], o["end"]
        return a[np.lexsort((a[:, 2], a[:, 0], a[:, 1]))]
    o = raw.view(TAGGED)
    a = np.empty((count, 4), dtype=np.uint64)
    a[:, 0], a[:, 1], a[:, 2], a[:, 3] = o["sid"], o["pid"], o["start"], o["end"]
    return a[np.lexsort((a[:, 3], a[:, 1], a[:, 2], a[:, 0]))]


def mismatches(a: np.ndarray, b: np.ndarray) -> int:
    """Size of the symmetric difference of two match multisets."""
    if a.shape == b.shape and np.array_equal(a, b):
        return 0
    from collections import Counter
    ca = Counter(map(tuple, a.astype(np.uint64).tolist()))
    cb = Counter(map(tuple, b.astype(np.uint64).tolist()))
    return sum(((ca - cb) + (cb - ca)).values())


def oracle_rows(wl, nbytes: int, threads: int) -> np.ndarray:
    import oracle
    if wl.items is not None:
        return oracle.batch_scan(wl.patterns, wl.data, wl.items, threads=threads)
    return oracle.scan_patterns(wl.patterns, wl.data[:nbytes], threads)


def run_reference(args, rank):
    if rank != 0:
        return
    wl = make_workload(args.config, args.size)
    base = cpu_baseline(wl, seconds=max(2.0, 60.0 / max(args.steps + args.warmup, 1)))
    line = {"metric": METRIC, "value": base["value"], "unit": "GB/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": {"workload": args.config, "description": CONFIGS[args.config]},
            "impl": "reference", "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "oracle port of the reference CPU algorithm (the Rust crate and its wgpu path cannot run here)"}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ ours
def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="regex", choices=sorted(CONFIGS))
    ap.add_argument("--size", type=int, default=None, help="input bytes (items for batch)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the oracle comparison of the full match set")
    ap.add_argument("--no-literal", action="store_true",
                    help="skip the literals_large sub-record of the regex configuration")
    ap.add_argument("--no-arms", action="store_true", help="skip the second boundary-guess arm of the regex walk")
    ap.add_argument("--parity-bytes", type=int, default=(4 << 30) - (16 << 20),
                    help="dna: bytes of the input prefix compared with the oracle (its offsets are 32-bit)")
    ap.add_argument("--walk-chunk", type=int, default=None, help="speculative walk chunk bytes")
    ap.add_argument("--no-proposer", action="store_true", help="guess the unanchored start at every boundary")
    ap.add_argument("--dfa-max-states", type=int, default=None, help="states per merged group DFA")
    return ap.parse_args()


class Runner:
    """Device-resident inputs and outputs of one configuration and the timed
    step over them (one scan of the whole input by the full pattern set)."""

    def __init__(self, wl, config, dev, stream, dist, torch):
        self.wl, self.config, self.dev, self.stream, self.dist, self.torch = wl, config, dev, stream, dist, torch
        self.batch = wl.items is not None
        self.big = config == "dna" or wl.data.nbytes > 0xFFFFFFFF
        if self.batch:
            self.lens = np.array([ln for _, ln in wl.items], dtype=np.uint64)
            self.n_bytes = int(self.lens.sum())
            self.n_items = len(self.lens)
            self.d_in = torch.from_numpy(wl.data[: self.n_bytes]).to(dev)
            self.d_ends = torch.from_numpy(np.cumsum(self.lens).astype(np.uint32).view(np.int32)).to(dev)
            self.d_ids = torch.arange(self.n_items, dtype=torch.int64, device=dev)
        else:
            self.n_bytes = int(wl.data.nbytes)
            self.n_items = 1
            self.d_in = torch.from_numpy(wl.data).to(dev)
        # ws_match (12 B), ws_match64 or ws_tagged_match (24 B)
        self.d_out = torch.empty(CAP * 3, dtype=torch.int64, device=dev)
        self.d_cnt = torch.zeros(1, dtype=torch.int64, device=dev)
        self.kind = "tagged" if self.batch else "match64" if self.big else "match"
        # inputs smaller than L2 are re-read cold: a 512 MiB write between steps
        self.flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev) if self.n_bytes < (256 << 20) else None

    def step(self, matcher, n_bytes=None):
        s = self.stream.cuda_stream
        if self.batch:
            matcher.scan_batch_device(self.d_in.data_ptr(), self.n_bytes, self.d_ends.data_ptr(),
                                      self.d_ids.data_ptr(), self.n_items, self.d_out.data_ptr(), CAP,
                                      self.d_cnt.data_ptr(), s)
        elif self.big:
            matcher.scan_device64(self.d_in.data_ptr(), n_bytes or self.n_bytes, self.d_out.data_ptr(), CAP,
                                  self.d_cnt.data_ptr(), s)
        else:
            matcher.scan_device(self.d_in.data_ptr(), n_bytes or self.n_bytes, self.d_out.data_ptr(), CAP,
                                self.d_cnt.data_ptr(), s)

    def count(self) -> int:
        c = int(self.d_cnt.item()) & 0xFFFFFFFFFFFFFFFF
        if c > CAP:
            raise SystemExit(f"match overflow or unknown count ({c} > {CAP})")
        return c

    def timed_steps(self, matcher, steps, warmup):
        torch, dist = self.torch, self.dist
        for _ in range(warmup):
            self.step(matcher)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        total, infos = 0.0, []
        # per step: device time, and host time of the scan call (the enqueue)
        self.step_ms, self.enqueue_ms = [], []
        torch.cuda.nvtx.range_push("timed")  # lets a profiler capture only the timed steps
        for _ in range(steps):
            if self.flush is not None:
                self.flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(self.stream)
            h0 = time.perf_counter()
            self.step(matcher)
            self.enqueue_ms.append((time.perf_counter() - h0) * 1e3)
            e1.record(self.stream)
            e1.synchronize()
            total += e0.elapsed_time(e1)
            self.step_ms.append(e0.elapsed_time(e1))
            infos.append(matcher.info())
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        return total / steps, infos

    def parity(self, matcher, parity_bytes: int):
        """One more scan (untimed), its full match set against the oracle's on
        the same input: the whole input, or for the 4 GiB nucleotide input a
        prefix (the oracle's offsets are 32-bit)."""
        import oracle
        n = self.n_bytes
        if self.big:
            n = min(n, parity_bytes)
        self.step(matcher, n_bytes=n)
        self.torch.cuda.synchronize()
        got = device_rows(self.d_out, self.count(), self.kind)
        t = time.perf_counter()
        exp = oracle_rows(self.wl, n, oracle.hw_threads())
        dt = time.perf_counter() - t
        rec = {"mismatches": mismatches(got, exp), "compared_matches": int(len(exp)), "gpu_matches": int(len(got)),
               "compared_bytes": n, "oracle_s": round(dt, 2), "oracle_threads": oracle.hw_threads()}
        if n < self.n_bytes:
            rec["scope"] = f"first {n} bytes of the {self.n_bytes}-byte input"
        return rec


def boundary_guess(info, tune) -> str:
    """How the speculative walk chose each chunk's start state."""
    spec = info["n_groups"] - info["n_context_groups"]
    if spec and info["exact_groups"] == spec:
        return "exact: each chunk's start state from the bytes before it (every regex of bounded length)"
    if tune and tune["proposer_used"]:
        return "learned proposer (top-1)"
    return "unanchored start state (the autotuner turned the proposer off)"


def build_matchers(ws, wl, config, walk_chunk=None, proposer=True, dfa_max_states=None, plain_too=True):
    ps = ws.PatternSet.builder()
    for kind, p in wl.patterns:
        ps = ps.literal_bytes(p) if kind == 0 else ps.regex(p.decode())
    ps = ps.build()
    cfg = ws.AutoMatcherConfig().max_matches(CAP).profile(True).regex_mode(ws.REGEX_SPECULATIVE)
    if walk_chunk:
        cfg.walk_chunk(walk_chunk)
    if dfa_max_states:
        cfg.dfa_max_states(dfa_max_states)
    if not proposer:
        cfg.proposer(ws.PROPOSER_NONE)
    m = ws.GpuMatcher.with_config(ps, cfg)
    plain = None
    has_regex = any(k == 1 for k, _ in wl.patterns)
    if plain_too and has_regex and config in ("regex", "batch", "dna"):
        pcfg = ws.AutoMatcherConfig().max_matches(CAP).profile(True).regex_mode(ws.REGEX_PLAIN)
        plain = ws.GpuMatcher.with_config(ps, pcfg)
    tune = None
    if has_regex:
        # a separately seeded 256 MiB corpus of the same distribution: the
        # autotuner picks group size, hot rows, proposer and chunk on it (knobs
        # given on the command line stay fixed)
        corpus = W.dna_training_corpus() if config == "dna" else W.regex_training_corpus()
        flags = (0 if dfa_max_states else ws.GpuMatcher.TUNE_GROUPS) | (0 if walk_chunk else ws.GpuMatcher.TUNE_CHUNK)
        tune = m.tune(corpus, flags=flags)
        del corpus
    return m, plain, tune


def roofline_of(config, infos, n_bytes, count, n_items, batch, has_regex, peak, peak_kind):
    """The dominant kernel's achieved algorithmic bandwidth against the
    measured HBM peak (N input bytes + 12 B per match + 16 B per item)."""
    # the literal phase (index 0) spans the filter and the verify kernel; the
    # 10,000-literal set takes the large-set layout (stage-1b table, no literals
    # under 4 bytes), whose filter is literal_lean_kernel
    lit_name = "literal_lean_kernel" if config == "literals_large" else "literal_filter_kernel"

    def phase(k):
        return statistics.mean(i["last_kernel_ms"][k] for i in infos) if infos else 0.0

    # the dominant of the literal phase and the regex walk (the nucleotide
    # configuration spends more time on its 50,000 k-mers than on its walk)
    kidx, kname = (0, lit_name)
    if has_regex and (phase(1) >= phase(0) or not infos):
        kidx, kname = (1, "dfa_walk_kernel")
    kms = phase(kidx) if infos else None
    alg_bytes = n_bytes + 12 * count + (16 * n_items if batch else 0)
    achieved = alg_bytes / (kms * 1e-3) / 1e9 if kms else None
    return {"bound": "hbm", "achieved": round(achieved, 2) if achieved else None, "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4) if achieved else None,
            "traffic": read_traffic(kname, config), "kernel": kname,
            "kernel_ms": round(kms, 4) if kms else None,
            "peak_source": (f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured"
                            else "fallback 6.65 TB/s"),
            "algorithmic_bytes_per_launch": alg_bytes}


def walk_record(info, n_bytes, ms):
    """Counters of the speculative walk of one profiled scan."""
    g = info["n_groups"]
    walk_ms = info["last_kernel_ms"][1]
    guesses = info["last_guesses"]
    return {"gbs": round(n_bytes / (ms * 1e-3) / 1e9, 3), "ms_per_step": round(ms, 4),
            "walk_ms": round(walk_ms, 4),
            "lookups_per_s": round(g * n_bytes / (walk_ms * 1e-3), 1) if walk_ms else None,
            "guess_hit_rate": round(info["last_guess_hits"] / guesses, 5) if guesses else None,
            "fixup_chunks": info["last_fixup_chunks"], "chunks": info["last_chunks"],
            "rewalk_bytes": info["last_rewalk_bytes"],
            "rewalk_frac": round(info["last_rewalk_bytes"] / (g * n_bytes), 6) if g else None,
            "events": info["last_events"], "candidates": info["last_kcandidates"],
            "phase_ms": [round(x, 4) for x in info["last_kernel_ms"]]}


def literal_subrecord(ws, args, dev, stream, dist, torch, peak, peak_kind):
    """The literal prefilter + verify path (10,000 literals over 1 GiB) timed
    in the same run, with its own roofline and oracle comparison."""
    wl = make_workload("literals_large", None)
    m, _, _ = build_matchers(ws, wl, "literals_large", plain_too=False)
    r = Runner(wl, "literals_large", dev, stream, dist, torch)
    ms, infos = r.timed_steps(m, args.steps, args.warmup)
    count = r.count()
    rec = {"workload": "literals_large", "description": CONFIGS["literals_large"],
           "value": round(r.n_bytes / (ms * 1e-3) / 1e9, 3), "unit": "GB/s", "ms_per_step": round(ms, 4),
           "matches": count,
           "roofline": roofline_of("literals_large", infos, r.n_bytes, count, 1, False, False, peak, peak_kind)}
    if not args.no_parity:
        rec["parity"] = r.parity(m, args.parity_bytes)
    m.close()
    del r, wl
    torch.cuda.empty_cache()
    return rec


def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    torch.cuda.set_device(local)
    dev = f"cuda:{local}"
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    import warpstate_b200 as ws

    wl = make_workload(args.config, args.size)
    m, plain, tune = build_matchers(ws, wl, args.config, args.walk_chunk, not args.no_proposer,
                                    args.dfa_max_states, plain_too=not args.no_plain)
    stream = torch.cuda.current_stream()
    r = Runner(wl, args.config, dev, stream, dist, torch)
    n_bytes, n_items, batch = r.n_bytes, r.n_items, r.batch

    def max_over_ranks(x):
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        if dist:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # the speculative (or only) path
    with ClockSampler(local) as clk:
        ms, infos = r.timed_steps(m, args.steps, args.warmup)
    clocks = clk.summary()
    step_ms = [round(x, 4) for x in r.step_ms]
    enqueue_ms = round(sum(r.enqueue_ms) / max(1, len(r.enqueue_ms)), 4)
    count = r.count()
    ms_max = max_over_ranks(ms)
    value = world * n_bytes / (ms_max * 1e-3) / 1e9
    has_regex = any(k == 1 for k, _ in wl.patterns)

    # the other boundary guess of the speculative walk, timed the same way:
    # the trained proposer when the tuner chose the unanchored start, and the
    # reverse; same chunk, same matches
    arms = None
    if has_regex and tune and not args.no_arms and not args.no_proposer and tune["proposer_top1"] > 0:
        used = tune["proposer_used"]
        arms = {("proposer" if used else "unanchored"): walk_record(infos[-1], n_bytes, ms)}
        m.set_walk(0, ws.PROPOSER_NONE if used else ws.PROPOSER_MLP)
        ams, ainfos = r.timed_steps(m, args.steps, args.warmup)
        acount = r.count()
        if acount != count:
            raise SystemExit(f"match counts differ between boundary guesses: {acount} vs {count}")
        arms[("unanchored" if used else "proposer")] = walk_record(ainfos[-1], n_bytes, max_over_ranks(ams))
        m.set_walk(0, ws.PROPOSER_MLP if used else ws.PROPOSER_NONE)

    plain_gbs = plain_ms = None
    if plain is not None:
        pms, _ = r.timed_steps(plain, max(1, min(2, args.steps)), 1)
        plain_ms = max_over_ranks(pms)
        plain_gbs = world * n_bytes / (plain_ms * 1e-3) / 1e9
        plain_count = r.count()
        if plain_count != count:
            raise SystemExit(f"plain/speculative match counts differ: {plain_count} vs {count}")

    # batch: per-item dispatch of the plain kernel from host memory (one scan
    # call, one H2D copy and one readback per item), the shape of the
    # reference's per-call GPU round trips, on the first items
    per_item = None
    if batch and plain is not None:
        import ctypes
        import warpstate_b200._native as N
        k = min(n_items, 2000)
        lens = r.lens
        offs = np.concatenate([[0], np.cumsum(lens[:k])]).astype(np.int64)
        host = np.ascontiguousarray(wl.data[: int(offs[k])])
        out1 = (N.WsMatch * (1 << 20))()
        cnt1 = ctypes.c_uint64()
        err1 = N.WsErrorInfo()
        lib = N.lib()
        t0 = time.perf_counter()
        for i in range(k):
            st = lib.ws_scan(plain._h, host.ctypes.data + int(offs[i]), int(lens[i]), out1, 1 << 20,
                             ctypes.byref(cnt1), ctypes.byref(err1))
            if st != 0:
                raise SystemExit(f"per-item scan failed with status {st}")
        dt_items = time.perf_counter() - t0
        per_item = {"items": k, "bytes": int(offs[k]), "ms": round(dt_items * 1e3, 3),
                    "gbs": round(int(offs[k]) / dt_items / 1e9, 4),
                    "api": "GpuMatcher.scan (ws_scan), plain kernel, one call per item from host memory"}
    if plain is not None:
        plain.close()

    # roofline of the dominant kernel
    peak, peak_kind = load_peaks()
    roofline = roofline_of(args.config, infos, n_bytes, count, n_items, batch, has_regex, peak, peak_kind)

    # end to end through the public API from pinned host memory
    e2e = None
    if not args.no_e2e:
        pinned = torch.empty(n_bytes, dtype=torch.uint8, pin_memory=True)
        pinned.numpy()[:] = wl.data[:n_bytes]
        hv = pinned.numpy()
        if batch:
            lens = r.lens

            def call():
                return ws.scan_batch_packed(m, pinned, lens)
            d2h = lambda n: 24 * n + 8  # noqa: E731
        elif r.big:
            sp = ws.StreamPipeline(m)

            def call():
                return sp.scan_array(pinned)
            d2h = lambda n: 24 * n + 8  # noqa: E731
        else:
            def call():
                return m.scan_array(hv)
            d2h = lambda n: 12 * n + 8  # noqa: E731
        res = call()
        torch.cuda.synchronize()
        k = max(2, min(args.steps, 5)) if n_bytes < (2 << 30) else 2
        t0 = time.perf_counter()
        call_ms = []
        for _ in range(k):
            c0 = time.perf_counter()
            res = call()
            call_ms.append(round((time.perf_counter() - c0) * 1e3, 3))
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / k
        if len(res) != count:
            raise SystemExit(f"e2e count {len(res)} != device count {count}")
        # the link ceiling: a plain pinned host-to-device copy of the same bytes
        dbuf = torch.empty(n_bytes, dtype=torch.uint8, device=dev)
        dbuf.copy_(pinned, non_blocking=True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(k):
            dbuf.copy_(pinned, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        h2d_gbs = n_bytes * k / (e0.elapsed_time(e1) * 1e-3) / 1e9
        del dbuf
        e2e = {"value": round(world * n_bytes / dt / 1e9, 3), "unit": "GB/s", "h2d_bytes_per_step": n_bytes,
               "d2h_bytes_per_step": d2h(count), "ms_per_step": round(dt * 1e3, 3), "call_ms": call_ms,
               "h2d_copy_gbs": round(h2d_gbs, 2),
               "api": ("scan_batch_packed (ws_scan_batch)" if batch else
                       "StreamPipeline.scan (ws_stream_*)" if r.big else "GpuMatcher.scan (ws_scan)")}
        del pinned, hv

    # the full match set of one more scan against the oracle on the same input
    parity = None
    if rank == 0 and not args.no_parity:
        parity = r.parity(m, args.parity_bytes)

    base = None
    if rank == 0 and not args.no_cpu:
        base = cpu_baseline(wl)

    launches = infos[-1]["last_launches"] if infos else 0
    line = {
        "metric": METRIC,
        "value": round(value, 3),
        "unit": "GB/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_max, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u8",
        "data": "synthetic",
        "config": {"workload": args.config, "description": CONFIGS[args.config], "bytes_per_rank": n_bytes,
                   "items": n_items if batch else None, "patterns": len(wl.patterns), "matches": count,
                   "l2": "input larger than L2" if r.flush is None else "L2 flushed (512 MiB write) between steps",
                   "parallelism": f"replicas x{world}"},
        "roofline": roofline,
        "cpu_baseline": base,
        "e2e": e2e,
        "gpu_launches": int(launches) * args.steps,
        "clocks": clocks,
        "parity": parity,
    }
    if has_regex:
        last = infos[-1]
        rec = {"speculative_gbs": round(value, 3),
               "plain_gbs": round(plain_gbs, 3) if plain_gbs else None,
               "speedup_vs_plain": round(value / plain_gbs, 3) if plain_gbs else None,
               "plain_ms_per_step": round(plain_ms, 4) if plain_ms else None,
               "boundary_guess": boundary_guess(last, tune),
               "proposer_top1_heldout": last["proposer_top1"], "proposer_top4_heldout": last["proposer_top4"],
               "tune": tune, "groups": last["n_groups"], "states": last["total_states"]}
        rec.update(walk_record(last, n_bytes, ms_max))
        rec["step_ms"] = step_ms
        rec["enqueue_ms"] = enqueue_ms
        if arms:
            rec["arms"] = arms
        line["regex"] = rec
    if per_item is not None:
        line["batch"] = {"per_item_plain_dispatch": per_item,
                         "batched_gbs": round(value, 3)}
    del r
    torch.cuda.empty_cache()
    if args.config == "regex" and not args.no_literal and rank == 0 and world == 1:
        line["literal"] = literal_subrecord(ws, args, dev, stream, dist, torch, peak, peak_kind)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
