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
//        speculative:  a chunk-parallel walk of the group's unanchored DFA from
//                      proposed boundary states, exact fix-up of mispredicted
//                      chunks, then a reverse-DFA walk from every match end to
//                      enumerate the starts;
//   2. resolution: per regex, starts sorted, and the regex crate's find_iter
//      chain rebuilt: take the leftmost start, end it where the regex's
//      leftmost-first DFA last matched, continue from that end.
#pragma once
#include "ws_internal.h"

namespace ws {

struct GroupDev {
  uint32_t fwd_off;        // offset of the forward table (u32 words)
  uint32_t n_states, n_classes;
  uint32_t start_anchored, start_unanchored;  // premultiplied (state * classes)
  uint32_t rev_off, rev_start;                // reverse table, premultiplied start
  uint32_t mptr_off;       // forward match pointers (n_states + 1)
  uint32_t rmptr_off;      // reverse match pointers
  uint32_t cls_off;        // 256-byte class map
  uint32_t hot_words;      // leading table words staged in shared memory
  uint32_t pad;
};

struct RegexPlan {
  uint32_t n_regex = 0;
  uint32_t n_groups = 0;
  uint32_t total_states = 0;
  uint32_t max_classes = 0;
  int64_t max_len = 0;                   // longest match (-1 unbounded)
  std::vector<GroupDev> groups;
  std::vector<uint32_t> regex_group;     // regex index -> group
  // device tables
  DeviceBuffer d_groups, d_fwd, d_rev, d_lf, d_cls, d_mptr, d_mlist, d_rmptr, d_rmlist, d_lfinfo, d_pid;
  // host copies (for the proposer's training walk and diagnostics)
  std::vector<uint32_t> fwd, rev, lf, mptr, mlist, rmptr, rmlist, lfinfo, pid;
  std::vector<uint8_t> cls;
  // proposer
  struct Proposer* proposer = nullptr;
  double top1 = 0, top4 = 0;
  // last scan
  uint32_t walk_chunk = 4096;            // speculative chunk bytes (multiple of 256)
  uint64_t last_chunks = 0, last_fixup = 0, last_k = 0;
  uint32_t last_launches = 0;
  ~RegexPlan();
};

struct RegexLaunch {
  const uint8_t* data;
  uint64_t len;
  ws_match* out;
  uint64_t cap;
  unsigned long long* counter;
  uint32_t mode;
};

void plan_regex(const ws_pattern_tables& t, const ws_config& cfg, int sm_count, RegexPlan& plan);
void regex_fill_info(const RegexPlan& plan, ws_matcher_info& info);
// Enqueues the regex pipeline on `st`.  `events` (8 CUDA events) is non-null
// when phase timing is wanted.  Returns the number of kernel launches.
uint32_t run_regex_scan(RegexPlan& plan, const RegexLaunch& l, cudaStream_t st, DeviceBuffer& scratch,
                        int sm_count, cudaEvent_t* events);
// Byte offset, inside the regex scratch, of the error-flag word (non-zero after
// a scan whose candidate or event buffer overflowed).
constexpr size_t kRegexErrorFlagOffset = 16;
void regex_collect_timing(const RegexPlan& plan, cudaEvent_t* events, ws_matcher_info& info);
// K candidates only (diagnostic entry point); returns their device count pointer.
uint64_t regex_candidates(RegexPlan& plan, const uint8_t* d_data, uint64_t len, uint32_t mode, cudaStream_t st,
                          DeviceBuffer& scratch, int sm_count, ws_match* host_out, uint64_t cap);

}  // namespace ws
