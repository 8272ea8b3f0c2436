#include "ws_dfa.h"

namespace ws {

void plan_regex(const ws_pattern_tables& t, const ws_config& cfg, int sm_count, RegexPlan& plan) {
  (void)cfg; (void)sm_count;
  plan.n_regex = t.n_regex;
  if (t.n_regex) raise(WS_ERR_COMPILE, "regex DFA path not built yet");
}
void regex_fill_info(const RegexPlan& plan, ws_matcher_info& info) { (void)plan; (void)info; }
void run_regex_scan(RegexPlan& plan, const RegexLaunch& l, cudaStream_t st, DeviceBuffer& scratch, int sm_count,
                    cudaEvent_t* events) {
  (void)plan; (void)l; (void)st; (void)scratch; (void)sm_count; (void)events;
}
void regex_collect_timing(const RegexPlan& plan, cudaEvent_t* events, ws_matcher_info& info) {
  (void)plan; (void)events; (void)info;
}

}  // namespace ws
