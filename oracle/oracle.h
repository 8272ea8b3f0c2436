/*
 * warpstate oracle -- CPU restatement of the reference's matching semantics.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (warpstate_b200/, include/)
 * links, loads or calls this library.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline / reference arm use it, and only as the checker or as
 * the timed CPU baseline.
 *
 * What it restates (paths are inside the reference project):
 *   - FNV-1a prefix hash ............ core/src/pattern/compiler.rs:343-350
 *   - LiteralPrefilterTable::build .. core/src/literal_prefilter.rs:23-88
 *   - literal contract L (every overlapping occurrence, duplicates under their
 *     own ids) as computed by the GPU literal path: per-position FNV-1a probe of
 *     the prefilter table (core/src/gpu/shader.rs:56-98) followed by the exact
 *     verify (core/src/gpu/shader.rs:174-227); equal to scan_overlapping's AC
 *     overlapping pass (core/src/cpu/scan.rs:300-349)
 *   - regex contract R: per regex, regex::bytes find_iter with multi_line(true),
 *     unicode(false) (core/src/regex_engine.rs:7-17, core/src/dfa/scan.rs:433-456):
 *     leftmost-first, non-overlapping, empty-match rule of regex-automata's
 *     iterator.  Restated as a bounded backtracker (the published "BitState"
 *     method: depth-first search in priority order with a visited set over
 *     (instruction, position)), written from the regex crate's documented
 *     semantics because the crate itself is not available here.
 *   - regex -> literal demotion (core/src/pattern/compiler.rs:181-212, 353-373)
 *     and the pathological-repetition check (core/src/pattern/compiler.rs:381-405).
 *
 * Parity of the regex restatement is pinned by the known answers in the
 * reference's tests (tests/unit/harness_regex.rs and others), ported as golden
 * fixtures under tests/golden/.
 */
#ifndef WARPSTATE_ORACLE_H
#define WARPSTATE_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { uint32_t pattern_id, start, end; } or_match;

uint32_t or_fnv1a(const uint8_t* bytes, size_t len, size_t window);

/* LiteralPrefilterTable::build.  offsets = n pairs (start,len); hashes = n.
 * Outputs: prefix_meta[4*window], bucket_ranges[2*nb], entries[2*n].
 * Returns 0 on success.  *n_buckets receives nb; call with bucket_ranges=NULL
 * first to size the buffer. */
int or_prefilter_build(const uint32_t* offsets, const uint32_t* hashes, uint32_t n,
                       uint32_t window, uint32_t* prefix_meta,
                       uint32_t* bucket_ranges, uint32_t* n_buckets, uint32_t* entries);

/* Contract L over the whole input (reference GPU literal algorithm on the CPU).
 * Returns the true match count; writes min(count, cap) matches (unsorted).
 * nthreads <= 0 means all hardware threads. */
uint64_t or_literal_scan(const uint8_t* packed, const uint32_t* offsets,
                         const uint32_t* literal_pattern_ids, uint32_t n_literals,
                         uint32_t window, const uint8_t* data, uint64_t len,
                         or_match* out, uint64_t cap, int nthreads);

/* Regex handles. */
typedef struct or_regex or_regex;
or_regex* or_regex_new(const char* pattern, char* err, size_t err_cap);
void or_regex_free(or_regex* r);
int or_regex_nullable(const or_regex* r);
/* Longest match in bytes, -1 when unbounded. */
long long or_regex_maxlen(const or_regex* r);
/* 1 if the regex would be demoted to a literal; the bytes go to out (cap). */
int or_regex_literal(const char* pattern, uint8_t* out, size_t cap, size_t* out_len);
/* 1 if pathological (nested repetition under an outer repetition with max>1). */
int or_regex_pathological(const char* pattern);

/* find_iter of one regex: writes (start,end) pairs, returns the true count. */
uint64_t or_regex_find_iter(const or_regex* r, const uint8_t* data, uint64_t len,
                            uint32_t* starts, uint32_t* ends, uint64_t cap);

/* find_iter of many regexes (each independently), ids in pattern_ids.
 * Returns the true count, writes min(count,cap) (unsorted). */
uint64_t or_regex_set_scan(or_regex* const* rs, const uint32_t* pattern_ids, uint32_t n,
                           const uint8_t* data, uint64_t len,
                           or_match* out, uint64_t cap, int nthreads);

/* Batch contract: every item scanned independently (L + R inside the item),
 * tagged with its id, sorted by (source_id, start, pattern_id, end) -- the
 * structure of scan_batch_cpu (core/src/batch.rs:170-195).  Items are
 * (item_off[i], item_len[i]) slices of data.  Returns the true count. */
typedef struct { uint64_t source_id; uint32_t pattern_id, start, end, reserved; } or_tagged_match;
uint64_t or_batch_scan(const uint8_t* packed, const uint32_t* offsets, const uint32_t* literal_pattern_ids,
                       uint32_t n_literals, uint32_t window, or_regex* const* rs, const uint32_t* regex_pattern_ids,
                       uint32_t n_regex, const uint8_t* data, const uint64_t* item_off, const uint64_t* item_len,
                       const uint64_t* item_id, uint64_t n_items, or_tagged_match* out, uint64_t cap,
                       int nthreads);

/* Sort matches by (start, pattern_id, end): the CPU path's order
 * (core/src/cpu/mod.rs:56-78). */
void or_sort_matches(or_match* m, uint64_t n);

int or_hw_threads(void);

#ifdef __cplusplus
}
#endif
#endif
