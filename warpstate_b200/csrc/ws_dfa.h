// Regex DFA path of the B200 scan (plain thread-per-start and speculative
// chunked walk).  Host plan + launchers.
#pragma once
#include "ws_internal.h"

namespace ws {

struct RegexPlan {
  uint32_t n_regex = 0;
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
void run_regex_scan(RegexPlan& plan, const RegexLaunch& l, cudaStream_t st, DeviceBuffer& scratch, int sm_count,
                    cudaEvent_t* events);
void regex_collect_timing(const RegexPlan& plan, cudaEvent_t* events, ws_matcher_info& info);

}  // namespace ws
