"""ctypes binding of include/warpstate.h (libwarpstate_b200.so).

The library is loaded from the package directory.  There is no fallback: if
the shared library is missing, importing the package raises, telling the user
to run the build (``python -m warpstate_b200.build``).
"""
from __future__ import annotations

import ctypes
from pathlib import Path

_DIR = Path(__file__).resolve().parent
LIB_PATH = _DIR / "libwarpstate_b200.so"

c_u8p = ctypes.POINTER(ctypes.c_uint8)
c_u32p = ctypes.POINTER(ctypes.c_uint32)
c_u64p = ctypes.POINTER(ctypes.c_uint64)


class WsMatch(ctypes.Structure):
    _fields_ = [("pattern_id", ctypes.c_uint32), ("start", ctypes.c_uint32), ("end", ctypes.c_uint32)]


class WsTaggedMatch(ctypes.Structure):
    _fields_ = [("source_id", ctypes.c_uint64), ("pattern_id", ctypes.c_uint32), ("start", ctypes.c_uint32),
                ("end", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class WsMatch64(ctypes.Structure):
    _fields_ = [("pattern_id", ctypes.c_uint32), ("reserved", ctypes.c_uint32),
                ("start", ctypes.c_uint64), ("end", ctypes.c_uint64)]


class WsItem(ctypes.Structure):
    _fields_ = [("id", ctypes.c_uint64), ("data", ctypes.c_void_p), ("len", ctypes.c_uint64)]


class WsErrorInfo(ctypes.Structure):
    _fields_ = [("index", ctypes.c_uint64), ("count", ctypes.c_uint64), ("max", ctypes.c_uint64),
                ("message", ctypes.c_char * 512)]


class WsPatternSpec(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_uint32), ("bytes", ctypes.c_void_p), ("len", ctypes.c_uint64)]


class WsPatternTables(ctypes.Structure):
    _fields_ = [("packed_bytes", c_u8p), ("packed_len", ctypes.c_uint64),
                ("offsets", c_u32p), ("literal_pattern_ids", c_u32p), ("n_literals", ctypes.c_uint32),
                ("hash_window_len", ctypes.c_uint32), ("prefix_meta", c_u32p), ("bucket_ranges", c_u32p),
                ("n_buckets", ctypes.c_uint32), ("entries", c_u32p),
                ("regex_sources", ctypes.POINTER(ctypes.c_char_p)), ("regex_pattern_ids", c_u32p),
                ("n_regex", ctypes.c_uint32), ("n_patterns", ctypes.c_uint32),
                ("case_insensitive", ctypes.c_uint32)]


class WsConfig(ctypes.Structure):
    _fields_ = [("gpu_threshold", ctypes.c_uint64), ("gpu_max_input_size", ctypes.c_uint64),
                ("max_matches", ctypes.c_uint64), ("chunk_size", ctypes.c_uint64),
                ("chunk_overlap", ctypes.c_uint64), ("regex_mode", ctypes.c_uint32),
                ("dfa_max_states", ctypes.c_uint32), ("walk_chunk", ctypes.c_uint32),
                ("proposer", ctypes.c_uint32), ("proposer_train_bytes", ctypes.c_uint64),
                ("proposer_seed", ctypes.c_uint64), ("flags", ctypes.c_uint32),
                ("batch_mib", ctypes.c_uint32), ("window_mib", ctypes.c_uint32), ("reserved", ctypes.c_uint32 * 5)]


class WsMatcherInfo(ctypes.Structure):
    _fields_ = [("n_literals", ctypes.c_uint32), ("n_regex", ctypes.c_uint32), ("n_groups", ctypes.c_uint32),
                ("total_states", ctypes.c_uint32), ("max_classes", ctypes.c_uint32),
                ("filter_q", ctypes.c_uint32), ("filter_period", ctypes.c_uint32),
                ("filter_bits", ctypes.c_uint32), ("proposer_top1", ctypes.c_double),
                ("proposer_top4", ctypes.c_double), ("last_fixup_chunks", ctypes.c_uint64),
                ("last_chunks", ctypes.c_uint64), ("last_kcandidates", ctypes.c_uint64),
                ("last_kernel_ms", ctypes.c_double * 8), ("last_launches", ctypes.c_uint32),
                ("max_literal_len", ctypes.c_uint32), ("max_regex_len", ctypes.c_int64),
                ("last_events", ctypes.c_uint64), ("last_rewalk_bytes", ctypes.c_uint64),
                ("last_guess_hits", ctypes.c_uint64), ("last_guesses", ctypes.c_uint64),
                ("regex_context", ctypes.c_uint32), ("n_context_groups", ctypes.c_uint32),
                ("last_graph_replay", ctypes.c_uint32), ("exact_groups", ctypes.c_uint32)]


class WsTuneReport(ctypes.Structure):
    _fields_ = [("dfa_max_states", ctypes.c_uint32), ("n_groups", ctypes.c_uint32), ("walk_chunk", ctypes.c_uint32),
                ("proposer_used", ctypes.c_uint32), ("group_candidates", ctypes.c_uint32 * 4),
                ("group_ms", ctypes.c_double * 4), ("chunk_candidates", ctypes.c_uint32 * 4),
                ("chunk_ms", (ctypes.c_double * 2) * 4), ("proposer_top1", ctypes.c_double),
                ("proposer_top4", ctypes.c_double), ("tune_seconds", ctypes.c_double)]


# Every symbol of include/warpstate.h, with its ctypes signature.
SIGNATURES = {
    "ws_ctx_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(WsErrorInfo)]),
    "ws_ctx_destroy": (None, [ctypes.c_void_p]),
    "ws_device_count": (ctypes.c_int, []),
    "ws_ir_build": (ctypes.c_int, [ctypes.POINTER(WsPatternSpec), ctypes.c_uint64, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(WsErrorInfo)]),
    "ws_ir_destroy": (None, [ctypes.c_void_p]),
    "ws_ir_tables": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(WsPatternTables)]),
    "ws_ir_set_name": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_uint64]),
    "ws_ir_name": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_uint64, c_u64p]),
    "ws_index_load": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p),
                                     ctypes.POINTER(WsErrorInfo)]),
    "ws_index_save": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, c_u64p,
                                     ctypes.POINTER(WsErrorInfo)]),
    "ws_config_default": (None, [ctypes.POINTER(WsConfig)]),
    "ws_matcher_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(WsPatternTables), ctypes.POINTER(WsConfig),
                                         ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(WsErrorInfo)]),
    "ws_matcher_destroy": (None, [ctypes.c_void_p]),
    "ws_scan": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(WsMatch),
                               ctypes.c_uint64, c_u64p, ctypes.POINTER(WsErrorInfo)]),
    "ws_scan_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                      ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(WsErrorInfo)]),
    "ws_scan_literals_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                                ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p,
                                                ctypes.POINTER(WsErrorInfo)]),
    "ws_scan_batch": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(WsItem), ctypes.c_uint64,
                                     ctypes.POINTER(WsTaggedMatch), ctypes.c_uint64, c_u64p, ctypes.POINTER(WsErrorInfo)]),
    "ws_scan_batch_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                            ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64,
                                            ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(WsErrorInfo)]),
    "ws_scan_device64": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                        ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(WsErrorInfo)]),
    "ws_scan_shard": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                     ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(WsErrorInfo)]),
    "ws_stream_begin": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(WsErrorInfo)]),
    "ws_stream_feed": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(WsMatch64),
                                      ctypes.c_uint64, c_u64p, ctypes.POINTER(WsErrorInfo)]),
    "ws_stream_end": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(WsMatch64), ctypes.c_uint64, c_u64p,
                                     ctypes.POINTER(WsErrorInfo)]),
    "ws_stream_destroy": (None, [ctypes.c_void_p]),
    "ws_zero_copy_begin": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p),
                                          ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(WsErrorInfo)]),
    "ws_zero_copy_finish": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(WsMatch), ctypes.c_uint64, c_u64p,
                                           ctypes.POINTER(WsErrorInfo)]),
    "ws_zero_copy_abort": (None, [ctypes.c_void_p]),
    "ws_hotswap_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p),
                                         ctypes.POINTER(WsErrorInfo)]),
    "ws_hotswap_swap": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "ws_hotswap_scan": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(WsMatch),
                                       ctypes.c_uint64, c_u64p, ctypes.POINTER(WsErrorInfo)]),
    "ws_hotswap_destroy": (None, [ctypes.c_void_p]),
    "ws_matcher_train_proposer": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                                 ctypes.POINTER(WsErrorInfo)]),
    "ws_matcher_tune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                       ctypes.c_uint32, ctypes.POINTER(WsTuneReport), ctypes.POINTER(WsErrorInfo)]),
    "ws_matcher_set_walk": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32,
                                           ctypes.POINTER(WsErrorInfo)]),
    "ws_matcher_get_info":(ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(WsMatcherInfo)]),
    "ws_regex_candidates": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32,
                                           ctypes.POINTER(WsMatch), ctypes.c_uint64, c_u64p, ctypes.POINTER(WsErrorInfo)]),
    "ws_status_name": (ctypes.c_char_p, [ctypes.c_int]),
}

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m warpstate_b200.build` "
                              "(the scan path has no CPU fallback)")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib
