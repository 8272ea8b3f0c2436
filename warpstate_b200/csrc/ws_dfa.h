// Regex DFA path of the B200 scan: host plan + launchers.
//
// Replaces the reference's regex path -- the WGSL ensemble kernel
// (core/src/gpu/ensemble_shader.wgsl:65-130) that only reports one bool per
// regex, followed by a CPU regex::bytes find_iter per flagged regex
// (core/src/gpu/dispatch.rs:331-380) -- with a GPU pipeline that produces the
// same find_iter spans:
//
//   1. candidates K = every (regex, start, end) with input[start..end) in the
//      regex's language, found either by
//        plain:        one thread per start position walking the group's DFA
//                      from its anchored start (the reference's form, with
//                      every match reported instead of a bool), or
//        speculative:  a chunk-parallel walk of the group's unanchored DFA,
//                      each chunk from its exact start state (derived from the
//                      bytes before it when every regex of the group is of
//                      bounded length) or from a proposed one, exact fix-up of
//                      mispredicted chunks, then a reverse-DFA walk from every
//                      match end to enumerate the starts;
//   2. resolution: per regex, starts sorted, and the regex crate's find_iter
//      chain rebuilt: take the leftmost start, end it where the regex's
//      leftmost-first DFA last matched, continue from that end.
//
// Transition words follow the reference's packing (core/src/dfa/mod.rs:19-22):
// bits 0..29 the next state's row, bit 31 match, bit 30 dead.  Rows are
// ordered by estimated visit frequency, so that the hottest rows of each group
// can be staged in shared memory as byte-indexed rows (256 words each: the
// hot path of a walk is one shared-memory load per input byte).
#pragma once
#include "ws_internal.h"

namespace ws {

// Hot rows staged per group in shared memory (a 224 KiB image: the first row
// replicated per lane, 191 more rows column-interleaved; see ws_dfa.cu).
constexpr uint32_t kHotRows = 192;
// Unanchored hot rows of the speculative walk and the fix-up, which stage six
// of the image's seven 32 KiB blocks (the first row and rows 1..159) and keep
// the rest of their shared memory for input stages.
constexpr uint32_t kHotRowsWalk = 160;
// Groups of at most this many byte classes (small alphabets: nucleotides)
// index the walk's image by class: a row takes `classes` words instead of
// 256, so the same 192 KiB hold 32 x (49152 / (32 x classes) - 1) hot rows.
constexpr uint32_t kClassImageMaxClasses = 32;
// Unanchored hot rows of a group with `classes` byte classes.
constexpr uint32_t walk_hot_rows(uint32_t classes) {
  return classes <= kClassImageMaxClasses ? 32 * (49152 / (32 * classes) - 1) : kHotRowsWalk;
}

struct GroupDev {
  uint32_t fwd_off;          // class-indexed forward table (u32 words)
  uint32_t n_states, n_classes;
  uint32_t start_anchored, start_unanchored;  // rows
  uint32_t rev_off, rev_start;                // reverse table and its start row
  uint32_t mptr_off, rmptr_off, cls_off;
  uint32_t hot_off, hot_rows;                 // unanchored hot rows [0, hot_rows), byte-indexed
  uint32_t ahot_off, ahot_base, ahot_rows;    // anchored hot rows [ahot_base, +ahot_rows)
  // Context groups (patterns with look-around assertions): the forward table
  // is a context DFA (build_context_all_dfa) with a start row per left
  // context, and match lists per (row, right context) at mptr[4 * row + k].
  uint32_t context;
  uint32_t cstart[4];
  // The unanchored image of the walk: entries per row (256 byte-indexed, or
  // the group's class count when class-indexed) and the bytes staged.
  uint32_t img_cols, img_bytes;
  // Speculative groups whose regexes all match at most L bytes (L <= kWarmMax):
  // L rounded up to 16, else 0.  The state of the unanchored walk at a
  // position depends only on the L bytes before it (an NFA thread that started
  // earlier has died or matched), so walking those bytes from the unanchored
  // start gives a chunk's exact start state.
  uint32_t warm;
};

// Longest match for which a chunk's start state is derived from the bytes
// before it (the walk reads them once per chunk: at most a quarter of a chunk).
constexpr uint32_t kWarmMax = 512;

struct Proposer;
// Frees a trained proposer (ws_proposer.cu).
struct ProposerDeleter {
  void operator()(Proposer* p) const;
};

struct RegexPlan {
  uint32_t n_regex = 0;
  uint32_t n_groups = 0;
  // Groups [0, n_spec) take the speculative walk (or the plain kernel);
  // groups [n_spec, n_groups) are context groups, walked one anchored walk
  // per start position in both modes.
  uint32_t n_spec = 0;
  bool has_context = false;              // some regex has a look-around assertion
  bool class_image = false;              // the speculative groups' walk images are class-indexed
  uint32_t total_states = 0;
  uint32_t max_classes = 0;
  int64_t max_len = 0;                   // longest match (-1 unbounded)
  // Speculative groups with exact chunk starts (GroupDev::warm > 0), and the
  // largest warm length among them.
  uint32_t n_warm = 0, max_warm = 0;
  bool rev_marks = false;                // reverse walks may share visited-state marks
  std::vector<GroupDev> groups;
  std::vector<uint32_t> regex_group;     // regex index -> group
  // device tables
  DeviceBuffer d_groups, d_fwd, d_hot, d_rev, d_lf, d_cls, d_mptr, d_mlist, d_rmptr, d_rmlist, d_lfinfo, d_pid,
      d_lfx;
  // host copies
  std::vector<uint32_t> fwd, rev, lf, mptr, mlist, rmptr, rmlist, lfinfo, pid;
  // per regex, 8 words: {context, start row per left context (4), offset in
  // `lf` of the end-step flags, 0, 0}; context 0 for regexes without
  // assertions
  std::vector<uint32_t> lfx;
  std::vector<uint32_t> hot;   // shared-memory images, one per (group, part)
  std::vector<uint8_t> cls;
  // host forward DFAs per group (their numbering defines the layout above)
  std::vector<Dfa> fdfa;
  std::vector<ByteClasses> fcls;
  std::vector<std::vector<uint32_t>> gregex;
  std::vector<uint32_t> nhot_u, nhot_a;
  // proposer
  std::unique_ptr<Proposer, ProposerDeleter> proposer;  // trained by ws_matcher_train_proposer
  bool use_proposer = true;               // config: MLP guesses (else the unanchored start)
  double top1 = 0, top4 = 0, start_rate = 0;
  uint32_t walk_chunk = 4096;            // speculative chunk bytes (multiple of 256)
  // last scan
  uint64_t last_chunks = 0;
  uint32_t last_launches = 0;
  // profiled scans: the scan's counters (K candidates, events, fix-up
  // re-walks and bytes, boundary guesses and hits), read back into pinned
  // memory behind the scan's last phase event
  struct PinnedDeleter {
    void operator()(unsigned long long* p) const { cudaFreeHost(p); }
  };
  std::unique_ptr<unsigned long long, PinnedDeleter> prof_ctr;
};

struct RegexLaunch {
  const uint8_t* data;
  uint64_t len;
  ws_match* out;
  uint64_t cap;
  unsigned long long* counter;
  uint32_t mode;
  // Batch scans: ascending exclusive item ends in `data`; every match lies
  // inside one item and each item has its own find_iter chain.
  const uint32_t* item_end = nullptr;
  uint32_t n_items = 0;
  // Stream scans: `data` holds stream bytes [base, base + len).  cursor[r]
  // (device, one u64 per regex) is regex r's find_iter position: matches
  // starting before it were decided by earlier calls.  Only matches starting
  // before `frontier` are decided now; cursor[r] advances to
  // max(last match end, frontier).
  unsigned long long* cursor = nullptr;
  uint64_t base = 0, frontier = 0;
  // Candidate-buffer sizing: `need` (device address of two host-mapped
  // words) receives the candidate and event counts of a scan whose buffers
  // overflowed; k_min and ev_min are the capacities to reserve (what an
  // earlier scan needed).
  unsigned long long* need = nullptr;
  uint64_t k_min = 0, ev_min = 0;
};

// Match count of a scan whose regex candidate buffers overflowed: the true
// count is unknown (repeating the scan succeeds, sized by what it needed).
constexpr unsigned long long kCountUnknown = ~0ull;
// Match count of a scan in which a bounded device-side wait ran out.
constexpr unsigned long long kCountTimeout = ~0ull - 1;

void plan_regex(const ws_pattern_tables& t, const ws_config& cfg, int sm_count, RegexPlan& plan);
// Re-ranks the forward DFA states of every group by how often a walk over
// `d_corpus` visits them and rebuilds the hot-row layout: the placement of
// rows in shared memory versus L2 is learned from the workload.
void regex_rerank_from_corpus(RegexPlan& plan, const uint8_t* d_corpus, uint64_t len);
void regex_fill_info(const RegexPlan& plan, ws_matcher_info& info);
// True when every speculative group starts its chunks (of `chunk` bytes) from
// their exact states, so that boundary guesses (and the proposer) are unused.
bool regex_all_exact(const RegexPlan& plan, uint64_t chunk);
// Enqueues the regex pipeline on `st`.  `events` (8 CUDA events) is non-null
// when phase timing is wanted.  Returns the number of kernel launches.
uint32_t run_regex_scan(RegexPlan& plan, const RegexLaunch& l, cudaStream_t st, DeviceBuffer& scratch,
                        int sm_count, cudaEvent_t* events);
void regex_collect_timing(const RegexPlan& plan, cudaEvent_t* events, ws_matcher_info& info);
// K candidates only (diagnostic entry point), copied to host_out.
uint64_t regex_candidates(RegexPlan& plan, const uint8_t* d_data, uint64_t len, uint32_t mode, cudaStream_t st,
                          DeviceBuffer& scratch, int sm_count, ws_match* host_out, uint64_t cap);

}  // namespace ws
