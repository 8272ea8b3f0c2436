/*
 * warpstate_b200 -- C ABI of the B200-native scan path.
 *
 * The reference (a Rust crate) drives its GPU scan through GpuMatcher
 * (core/src/gpu/mod.rs), the batch helpers (core/src/batch.rs) and
 * StreamPipeline (core/src/pipeline.rs).  This header is what a Rust shim binds
 * in their place: plain pointers and sizes, caller-owned output buffers, no
 * allocation handed across the boundary, status codes that map 1:1 onto the
 * reference's Error enum (core/src/error.rs:6-91).
 *
 * Semantics of a scan (the parity contract):
 *   - literal patterns: every occurrence, overlapping, duplicates reported under
 *     each id (what the reference's GPU literal kernels compute,
 *     core/src/gpu/shader.rs:56-98,174-227);
 *   - regex patterns: per regex, regex::bytes find_iter with multi_line(true) and
 *     unicode(false): leftmost-first, non-overlapping (what GpuMatcher::scan
 *     returns for regexes, core/src/gpu/dispatch.rs:357-378 ->
 *     core/src/dfa/scan.rs:433-456);
 *   - output sorted by (start, pattern_id, end) (core/src/cpu/mod.rs:56-78).
 *
 * Threading: a ws_matcher is immutable after creation; ws_scan* may be called
 * concurrently from many host threads (each call takes its own stream and
 * scratch from the matcher's pool), as GpuMatcher is shared across threads in
 * the reference (tests/adversarial/adversarial_gpu.rs:537-580).
 */
#ifndef WARPSTATE_B200_H
#define WARPSTATE_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes; each maps to one variant of core/src/error.rs:6-91. */
typedef enum {
  WS_OK = 0,
  WS_ERR_EMPTY_PATTERN_SET = 1,     /* Error::EmptyPatternSet */
  WS_ERR_EMPTY_PATTERN = 2,         /* Error::EmptyPattern{index} */
  WS_ERR_NO_DEVICE = 3,             /* Error::NoGpuAdapter */
  WS_ERR_DEVICE = 4,                /* Error::GpuDeviceError{reason} */
  WS_ERR_BUFFER_MAP = 5,            /* Error::BufferMapFailed */
  WS_ERR_COMPILE = 6,               /* Error::PatternCompilationFailed{reason} */
  WS_ERR_DFA_OOB = 7,               /* Error::DfaOutOfBounds */
  WS_ERR_PATTERN_TOO_LARGE = 8,     /* Error::PatternTooLarge */
  WS_ERR_PATTERN_SET_TOO_LARGE = 9, /* Error::PatternSetTooLarge */
  WS_ERR_INPUT_TOO_LARGE = 10,      /* Error::InputTooLarge{bytes,max_bytes} */
  WS_ERR_OVERFLOW = 11,             /* Error::MatchBufferOverflow{count,max} */
  WS_ERR_PATHOLOGICAL = 12,         /* Error::PathologicalRegex{index} */
  WS_ERR_TIMEOUT = 13,              /* Error::GpuDeviceError{"... timed out"} */
  WS_ERR_INVALID_ARGUMENT = 14      /* caller bug (null pointer, bad size) */
} ws_status;

/* Match { pattern_id, start, end } -- three u32, 12 bytes, the reference's
 * layout (asserted at core/src/dfa/mod.rs:416-419). */
typedef struct { uint32_t pattern_id, start, end; } ws_match;

/* batch::TaggedMatch (core/src/batch.rs:22-27): offsets relative to the item. */
typedef struct { uint64_t source_id; uint32_t pattern_id, start, end, reserved; } ws_tagged_match;

/* batch::ScanItem (core/src/batch.rs:13-18). */
typedef struct { uint64_t id; const uint8_t* data; uint64_t len; } ws_item;

/* Matches of a stream carry 64-bit offsets (a stream may exceed 4 GiB). */
typedef struct { uint32_t pattern_id, reserved; uint64_t start, end; } ws_match64;

/* Extra error detail filled by calls that can fail with a payload. */
typedef struct {
  uint64_t index;      /* EmptyPattern / PatternTooLarge / PathologicalRegex */
  uint64_t count;      /* MatchBufferOverflow.count, InputTooLarge.bytes */
  uint64_t max;        /* MatchBufferOverflow.max, InputTooLarge.max_bytes */
  char message[512];   /* reason text for GpuDeviceError / PatternCompilationFailed */
} ws_error_info;

typedef struct ws_ctx ws_ctx;
typedef struct ws_ir ws_ir;
typedef struct ws_matcher ws_matcher;
typedef struct ws_stream ws_stream;

/* ------------------------------------------------------------------ context */
/* One context per device: holds the CUDA context binding and the caching
 * allocator.  Replaces acquire_device / GpuBufferPool
 * (core/src/gpu/device.rs:9-84,158-189). */
ws_status ws_ctx_create(int device, ws_ctx** out, ws_error_info* err);
void ws_ctx_destroy(ws_ctx* ctx);
int ws_device_count(void);

/* --------------------------------------------------------------- pattern IR */
/* Pattern kinds for ws_ir_build. */
enum { WS_PATTERN_LITERAL = 0, WS_PATTERN_REGEX = 1 };
typedef struct {
  uint32_t kind;            /* WS_PATTERN_LITERAL or WS_PATTERN_REGEX */
  const uint8_t* bytes;     /* literal bytes, or the regex source (UTF-8) */
  uint64_t len;
} ws_pattern_spec;

/* PatternSetBuilder::build (core/src/pattern/compiler.rs:97-340), host only:
 * literal packing, FNV-1a prefix hashes with hash_window_len = 8, regex parse
 * and validation, pathological-repetition rejection, literal demotion, and the
 * LiteralPrefilterTable.  Pattern ids are the insertion indices. */
ws_status ws_ir_build(const ws_pattern_spec* patterns, uint64_t n, int case_insensitive,
                      ws_ir** out, ws_error_info* err);
void ws_ir_destroy(ws_ir* ir);

/* A read-only view of the IR, laid out as the reference's PatternIR
 * (core/src/pattern/ir.rs:6-34) and LiteralPrefilterTable
 * (core/src/literal_prefilter.rs:10-19).  A Rust shim fills this struct from
 * its own PatternIR and passes it to ws_matcher_create. */
typedef struct {
  const uint8_t* packed_bytes; uint64_t packed_len;
  const uint32_t* offsets;             /* 2 per literal: (start, len) */
  const uint32_t* literal_pattern_ids; /* user pattern id per literal */
  uint32_t n_literals;
  uint32_t hash_window_len;            /* 8 in the reference */
  const uint32_t* prefix_meta;         /* 4 per prefix length */
  const uint32_t* bucket_ranges;       /* 2 per bucket */
  uint32_t n_buckets;
  const uint32_t* entries;             /* 2 per literal: (hash, literal index) */
  const char* const* regex_sources;    /* NUL-terminated sources */
  const uint32_t* regex_pattern_ids;
  uint32_t n_regex;
  uint32_t n_patterns;                 /* total patterns (literals + regexes) */
  uint32_t case_insensitive;
} ws_pattern_tables;

ws_status ws_ir_tables(const ws_ir* ir, ws_pattern_tables* out);

/* Pattern names (PatternSetBuilder::named_literal / named_regex,
 * core/src/pattern/compiler.rs:50-93), kept with the IR so that a compiled
 * index carries them.  ws_ir_name writes the name's UTF-8 bytes (not
 * NUL-terminated) and sets *n_out to its length, or to UINT64_MAX when the
 * pattern has no name. */
ws_status ws_ir_set_name(ws_ir* ir, uint64_t pattern_id, const char* name, uint64_t len);
ws_status ws_ir_name(const ws_ir* ir, uint64_t pattern_id, char* out, uint64_t cap, uint64_t* n_out);

/* ----------------------------------------------------------- compiled index */
/* CompiledPatternIndex::load (core/src/compiled_index/mod.rs:58-260): parses
 * the reference's on-disk index (magic WPSIDX01, versions 1-3, CRC-32 of
 * version 3) into an IR, with the reference's own validation and errors
 * (PatternCompilationFailed for a corrupt, truncated or inconsistent file,
 * InputTooLarge above 512 MiB).  The literal tables -- packed bytes, offsets,
 * ids and the LiteralPrefilterTable -- are used as stored (after bounds
 * checks); regexes come from their stored sources (version 2 and later), and
 * the stored regex-automata DFAs are checked for shape and not used. */
ws_status ws_index_load(const uint8_t* bytes, uint64_t len, ws_ir** out, ws_error_info* err);

/* CompiledPatternIndex::build (core/src/compiled_index/builder.rs:8-64):
 * serializes an IR in the version 3 format, with names, regex sources and the
 * literal tables, and no serialized regex-automata DFAs (the regex section is
 * rebuilt from the sources on load, here and by the reference's
 * to_pattern_set).  *n_out receives the size; WS_ERR_OVERFLOW when it exceeds
 * cap (call again with a larger buffer). */
ws_status ws_index_save(const ws_ir* ir, uint8_t* out, uint64_t cap, uint64_t* n_out, ws_error_info* err);

/* ------------------------------------------------------------------ matcher */
/* AutoMatcherConfig (core/src/config.rs:39-173) plus the B200 plan knobs. */
typedef struct {
  uint64_t gpu_threshold;          /* default 65536 */
  uint64_t gpu_max_input_size;     /* default 128 MiB */
  uint64_t max_matches;            /* default 1,000,000 */
  uint64_t chunk_size;             /* default 128 MiB */
  uint64_t chunk_overlap;          /* default 4096 */
  uint32_t regex_mode;             /* WS_REGEX_* below */
  uint32_t dfa_max_states;         /* per DFA group; default 8192 */
  uint32_t walk_chunk;             /* speculative chunk bytes; default 4096 */
  uint32_t proposer;               /* WS_PROPOSER_* below */
  uint64_t proposer_train_bytes;   /* default 256 MiB */
  uint64_t proposer_seed;          /* corpus seed for proposer training */
  uint32_t flags;                  /* WS_FLAG_* below */
  uint32_t batch_mib;              /* ws_scan_batch: bytes per launch sequence, MiB (0: 1024) */
  uint32_t window_mib;             /* streams, ws_scan_device64: new bytes per window, MiB (0: 1024) */
  uint32_t reserved[5];
} ws_config;

enum { WS_REGEX_SPECULATIVE = 0, WS_REGEX_PLAIN = 1 };
enum { WS_PROPOSER_MLP = 0, WS_PROPOSER_NONE = 1 };
/* WS_FLAG_PROFILE: record CUDA events around every kernel phase of a scan so
 * ws_matcher_get_info reports per-phase device times (one caller at a time). */
enum { WS_FLAG_PROFILE = 1 };

void ws_config_default(ws_config* cfg);

/* GpuMatcher::with_config (core/src/gpu/mod.rs:113-220): uploads the literal
 * tables, builds the regex DFAs (forward, reverse, per-pattern priority), trains
 * the boundary proposer and keeps everything resident on the device. */
ws_status ws_matcher_create(ws_ctx* ctx, const ws_pattern_tables* tables,
                            const ws_config* cfg, ws_matcher** out, ws_error_info* err);
void ws_matcher_destroy(ws_matcher* m);

/* GpuMatcher::scan (core/src/gpu/mod.rs:223-388).  data/len are host memory
 * (pinned or pageable).  Writes up to cap matches sorted by (start, pattern_id,
 * end); *n_out receives the true count.  When the count exceeds cap or the
 * configured max_matches, returns WS_ERR_OVERFLOW with err->count = true count
 * (re-call with a larger buffer; there is no CPU fallback). */
ws_status ws_scan(ws_matcher* m, const uint8_t* data, uint64_t len,
                  ws_match* out, uint64_t cap, uint64_t* n_out, ws_error_info* err);

/* Match count a device-resident scan reports when its regex candidate buffers
 * (library scratch, sized from the input length and max_matches) overflowed:
 * the true count is not known.  The matcher records how many candidates the
 * scan needed, so the same call made again succeeds.  The synchronous entry
 * points (ws_scan, ws_scan_batch, ws_stream_*) repeat such a scan themselves
 * and always return the true count. */
#define WS_COUNT_UNKNOWN UINT64_MAX
/* Match count a device-resident scan reports when one of its bounded
 * device-side waits ran out (it should not; the synchronous entry points
 * return WS_ERR_TIMEOUT for it). */
#define WS_COUNT_TIMEOUT (UINT64_MAX - 1)

/* Device-resident variant: d_data is a 16-byte aligned device pointer, d_out a
 * device buffer of cap matches, d_count a device u64 that receives the true
 * match count (only min(count, cap) matches are written; count > cap means
 * overflow), or WS_COUNT_UNKNOWN or WS_COUNT_TIMEOUT (see above).  Nothing is copied to the host
 * and the output is unsorted.  All work is enqueued on `stream` (a
 * cudaStream_t, 0 = legacy default stream) and the call returns without
 * synchronising.  The device-resident calls below report counts the same way. */
ws_status ws_scan_device(ws_matcher* m, const uint8_t* d_data, uint64_t len,
                         ws_match* d_out, uint64_t cap, uint64_t* d_count,
                         void* stream, ws_error_info* err);

/* Allocation-free literal scan.  No counterpart in the reference.  For callers
 * that cannot call cudaMalloc while scanning (a framework whose memory manager
 * owns all device memory, or a latency-bound loop that cannot afford
 * cudaMalloc's implicit synchronisation): same inputs, outputs and semantics as
 * ws_scan_device, for matchers whose pattern set has literals only, with the
 * scratch in a static device array inside the library (about 8 MiB, held on
 * every GPU that loads the library until the process exits) instead of an
 * allocation.  Accepts at most 128 MiB per call (WS_ERR_INPUT_TOO_LARGE
 * beyond).  Every call looks up the array's device address
 * (cudaGetSymbolAddress); the first call on a device loads the library's
 * device code there, so make that first call before any stream capture.  A
 * device reset (cudaDeviceReset) discards the array with everything else on
 * the device, including the results of earlier calls.  All calls share the
 * one array: calls whose work overlaps on the GPU race, so serialise them (one
 * stream, or events). */
ws_status ws_scan_literals_noalloc(ws_matcher* m, const uint8_t* d_data, uint64_t len,
                                   ws_match* d_out, uint64_t cap, uint64_t* d_count,
                                   void* stream, ws_error_info* err);

/* scan_batch / scan_batch_gpu (core/src/batch.rs:170-363): every item scanned
 * independently in one launch sequence, matches tagged with the item id and
 * sorted by (source_id, start, pattern_id, end); no cross-item matches. */
ws_status ws_scan_batch(ws_matcher* m, const ws_item* items, uint64_t n_items,
                        ws_tagged_match* out, uint64_t cap, uint64_t* n_out,
                        ws_error_info* err);

/* Device-resident form of ws_scan_batch (no reference counterpart: the
 * reference always coalesces on the host, core/src/batch.rs:65-98).  The items
 * are already coalesced in device memory: d_data (16-byte aligned, len < 4 GiB)
 * holds them back to back, d_item_end[i] is the exclusive end of item i
 * (ascending, the last equal to len) and d_ids[i] its source id.  Tagged
 * matches (item-relative offsets) go to d_out in no particular order;
 * *d_count (device) receives the true count.  Asynchronous on `stream`. */
ws_status ws_scan_batch_device(ws_matcher* m, const uint8_t* d_data, uint64_t len,
                               const uint32_t* d_item_end, const uint64_t* d_ids, uint64_t n_items,
                               ws_tagged_match* d_out, uint64_t cap, uint64_t* d_count,
                               void* stream, ws_error_info* err);

/* Device-resident scan of an input of any size with 64-bit offsets (the
 * stream machinery over a buffer already in device memory: windows of up to
 * 1 GiB with exact state carry).  The reference caps scans at u32 offsets
 * (core/src/gpu/mod.rs:248-262); this has no counterpart there.  Matches go to
 * d_out in no particular order; *d_count (device) receives the true count.
 * Asynchronous on `stream`. */
ws_status ws_scan_device64(ws_matcher* m, const uint8_t* d_data, uint64_t len,
                           ws_match64* d_out, uint64_t cap, uint64_t* d_count,
                           void* stream, ws_error_info* err);

/* One shard of a scan split across GPUs: the multi-GPU form of
 * MultiGpuMatcher::scan (core/src/multi_gpu.rs:126-160), exact for regexes.
 * d_data holds input bytes [base, base + len): the shard's own range
 * [base, own_end) plus a halo long enough for any match starting before
 * own_end.  Literal matches starting in the own range are reported; each regex
 * resumes its find_iter chain at d_cursor[r] (device, one u64 per regex,
 * stream offsets; pass base when nothing before the shard reaches into it) and
 * decides every match starting before own_end, after which d_cursor[r] holds
 * max(end of its last match, own_end): the next shard's incoming cursor.
 * Offsets in d_out are stream offsets.  Asynchronous on `stream`.
 * Look-behind assertions (^ \b \B \A) at d_data[0] read it as the start of
 * the input: for a pattern set with such regexes (ws_matcher_info.
 * regex_context), give a shard after the first one byte before its own range
 * (base one lower) and drop the literal matches that start at that byte. */
ws_status ws_scan_shard(ws_matcher* m, const uint8_t* d_data, uint64_t len, uint64_t base,
                        uint64_t own_end, uint64_t* d_cursor, ws_match64* d_out, uint64_t cap,
                        uint64_t* d_count, void* stream, ws_error_info* err);

/* StreamPipeline (core/src/pipeline.rs:87-153) with state carry: feed bytes in
 * pieces of any size; matches are reported once, with global 64-bit offsets,
 * as soon as they are final.  The union over all feeds plus end equals ws_scan
 * of the concatenation. */
ws_status ws_stream_begin(ws_matcher* m, ws_stream** out, ws_error_info* err);
ws_status ws_stream_feed(ws_stream* s, const uint8_t* data, uint64_t len,
                         ws_match64* out, uint64_t cap, uint64_t* n_out, ws_error_info* err);
ws_status ws_stream_end(ws_stream* s, ws_match64* out, uint64_t cap, uint64_t* n_out,
                        ws_error_info* err);
void ws_stream_destroy(ws_stream* s);

/* Zero-copy scan session: StreamPipeline::scan_zero_copy / ZeroCopyScan
 * (core/src/pipeline.rs:31-83) over DmaStagingBuffer (core/src/dma.rs:17-141).
 * ws_zero_copy_begin returns in *mapped a writable buffer of input_len bytes
 * of pinned, device-mapped host memory owned by the library; the caller fills
 * it and calls ws_zero_copy_finish, which scans it exactly as ws_scan does
 * (same output, sorting and errors) with the device copies reading the
 * caller's bytes in place, and ends the session (the buffer returns to a
 * per-matcher pool and must not be touched afterwards).  ws_zero_copy_abort
 * ends a session without scanning.  Staging buffers are freed with the
 * matcher; end every session before destroying its matcher. */
typedef struct ws_zero_copy ws_zero_copy;
ws_status ws_zero_copy_begin(ws_matcher* m, uint64_t input_len, ws_zero_copy** out, uint8_t** mapped,
                             ws_error_info* err);
ws_status ws_zero_copy_finish(ws_zero_copy* z, ws_match* out, uint64_t cap, uint64_t* n_out, ws_error_info* err);
void ws_zero_copy_abort(ws_zero_copy* z);

/* HotSwapPatternSet (core/src/pattern/mod.rs:17-70): a handle whose active
 * matcher can be replaced while other threads scan through it.
 * ws_hotswap_create and ws_hotswap_swap take ownership of the matcher they
 * are given.  ws_hotswap_swap returns 1 when the active matcher changed, 0
 * when `next` is already active (the reference's swap_arc result), -1 for a
 * null argument; the matcher it replaces is destroyed once no scan that
 * started with it is running.  ws_hotswap_scan is ws_scan with the matcher
 * active when the call starts. */
typedef struct ws_hotswap ws_hotswap;
ws_status ws_hotswap_create(ws_matcher* initial, ws_hotswap** out, ws_error_info* err);
int ws_hotswap_swap(ws_hotswap* h, ws_matcher* next);
ws_status ws_hotswap_scan(ws_hotswap* h, const uint8_t* data, uint64_t len, ws_match* out, uint64_t cap,
                          uint64_t* n_out, ws_error_info* err);
void ws_hotswap_destroy(ws_hotswap* h);

/* Trains the learned boundary-state proposer of the speculative regex walk on
 * a corpus drawn from the same distribution as the inputs to be scanned (host
 * memory, at least 64 KiB; 256 MiB is the intended size).  No counterpart in
 * the reference (its GPU regex path has no chunked walk).  Until it is called,
 * the walk guesses the unanchored start state at every chunk boundary; results
 * are exact either way (mispredicted chunks are re-walked).  Groups whose
 * regexes all match at most 512 bytes (ws_matcher_info.exact_groups) take no
 * guess at all: each chunk starts from the state derived from the bytes before
 * it. */
ws_status ws_matcher_train_proposer(ws_matcher* m, const uint8_t* corpus, uint64_t len, uint64_t seed,
                                    ws_error_info* err);

/* Autotuner of the regex walk on a sample corpus (no counterpart in the
 * reference).  With WS_TUNE_GROUPS it rebuilds the merged group DFAs at
 * several size limits and keeps the plan whose scan of the corpus is fastest;
 * it then learns the hot-row placement from the corpus, trains the proposer
 * (when the config enables it and some group has no exact chunk starts) and,
 * with WS_TUNE_CHUNK, times the speculative
 * walk at several chunk sizes with and without the proposer and keeps the
 * fastest.  Every choice gives the same matches; only speed differs.  The
 * corpus is host memory of at least 64 KiB; the timings scan it tiled to 1 GiB.
 * Call it before scanning, not while scans run. */
enum { WS_TUNE_GROUPS = 1, WS_TUNE_CHUNK = 2 };
typedef struct {
  uint32_t dfa_max_states, n_groups, walk_chunk, proposer_used;
  uint32_t group_candidates[4];      /* size limits tried (0: unused slot) */
  double group_ms[4];                /* corpus scan time per candidate, ms */
  uint32_t chunk_candidates[4];      /* walk chunks tried (0: unused slot) */
  double chunk_ms[4][2];             /* [chunk][0: no proposer, 1: proposer], ms */
  double proposer_top1, proposer_top4;
  double tune_seconds;
} ws_tune_report;
ws_status ws_matcher_tune(ws_matcher* m, const uint8_t* corpus, uint64_t len, uint64_t seed,
                          uint32_t flags, ws_tune_report* report, ws_error_info* err);

/* Pins the speculative walk's chunk (bytes, a multiple of 256; 0 keeps the
 * current one) and whether the trained proposer (WS_PROPOSER_MLP) or the
 * unanchored start (WS_PROPOSER_NONE) supplies each chunk's start state in the
 * groups without exact chunk starts, overriding the autotuner's choice.  Matches never change.  No counterpart in
 * the reference.  Call it between scans, not while scans run. */
ws_status ws_matcher_set_walk(ws_matcher* m, uint32_t walk_chunk, uint32_t proposer, ws_error_info* err);

/* Introspection for tests and the benchmark. */
typedef struct {
  uint32_t n_literals, n_regex, n_groups;
  uint32_t total_states;         /* forward DFA states over all groups */
  uint32_t max_classes;
  uint32_t filter_q, filter_period, filter_bits;
  double proposer_top1, proposer_top4;  /* held-out hit rates after training */
  uint64_t last_fixup_chunks;     /* chunk re-walks of the fix-up (profiled scans) */
  uint64_t last_chunks;           /* (group, chunk) walks of the last scan */
  uint64_t last_kcandidates;      /* regex candidates of the last profiled scan */
  double last_kernel_ms[8];      /* literal, walk, propose, fixup, reverse, resolve, plain, total */
  uint32_t last_launches;
  uint32_t max_literal_len;      /* longest literal (bytes) */
  int64_t max_regex_len;         /* longest regex match (bytes), -1 unbounded */
  /* Counters of the last profiled speculative scan (WS_FLAG_PROFILE): */
  uint64_t last_events;          /* match events of the chunked walk */
  uint64_t last_rewalk_bytes;    /* bytes re-walked by the fix-up (over all groups) */
  uint64_t last_guess_hits;      /* chunk boundaries whose guessed start state was the true one */
  uint64_t last_guesses;         /* chunk boundaries guessed (chunks - 1, per group) */
  uint32_t regex_context;        /* 1 when some regex has a look-around assertion */
  uint32_t n_context_groups;     /* DFA groups of such regexes (walked per start position) */
  uint32_t last_graph_replay;    /* 1 when the last ws_scan_batch_device call replayed a captured CUDA
                                    graph of its launch sequence (the same arguments as the calls before
                                    it, on a stream other than the legacy default stream, not profiled) */
  uint32_t exact_groups;         /* speculative groups whose regexes all match at most 512 bytes: the walk
                                    derives each chunk's start state from the bytes before the chunk (at
                                    chunks of at least four times that length), so no boundary is guessed */
} ws_matcher_info;
ws_status ws_matcher_get_info(const ws_matcher* m, ws_matcher_info* out);

/* Diagnostic entry points used by the parity tests: the K-candidate set
 * (pattern_id, start, end) of every anchored regex match, computed by the plain
 * thread-per-start kernel (mode WS_REGEX_PLAIN) or by the speculative walk plus
 * reverse walk (WS_REGEX_SPECULATIVE).  Host buffers, unsorted.
 * With WS_CAND_DISTINCT or-ed into the mode: the candidates a scan works from,
 * which hold the same distinct (pattern_id, start) pairs, without the repeats
 * that a long run of match ends (a+ over a run of a's) makes quadratic. */
enum { WS_CAND_DISTINCT = 0x100 };
ws_status ws_regex_candidates(ws_matcher* m, const uint8_t* data, uint64_t len, uint32_t mode,
                              ws_match* out, uint64_t cap, uint64_t* n_out, ws_error_info* err);

const char* ws_status_name(ws_status s);

#ifdef __cplusplus
}
#endif
#endif
