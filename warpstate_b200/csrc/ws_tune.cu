// Autotuner of the regex walk: group size, hot-row placement, proposer and
// chunk size, chosen by timing scans of a sample corpus on the device.
//
// The knobs change only speed, never matches:
//   - the size limit of the merged group DFAs trades the number of walks over
//     the input (one per group) against how much of each group's walk stays in
//     its 224 KiB shared-memory image of hot rows;
//   - the hot rows themselves are ranked by how often a walk over the corpus
//     visits them (regex_rerank_from_corpus);
//   - the walk chunk trades proposer and fix-up work (per boundary) against
//     the parallelism of the walk;
//   - the proposer is kept only where it beats guessing the unanchored start,
//     and trained only when some group has no exact chunk starts (regexes of
//     unbounded length).
// No counterpart in the reference (its regex path has no tunable walk).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>

#include "ws_matcher.h"
#include "ws_proposer.h"

using namespace ws;

namespace {

// The timings scan the corpus tiled to 1 GiB: the walk's parallelism (chunks
// per group) depends on the input size, so the choice is made at the scale of
// the inputs the matcher is meant for.
constexpr uint64_t kTuneBytes = 1ull << 30;

// Median device time (ms) of the speculative regex scan of `len` bytes.
double time_regex(ws_matcher* m, RegexPlan& P, const uint8_t* d, uint64_t len, int reps) {
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  check_cuda(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
  struct Cleanup {
    cudaStream_t& st; cudaEvent_t& e0; cudaEvent_t& e1;
    ~Cleanup() { if (e0) cudaEventDestroy(e0); if (e1) cudaEventDestroy(e1); if (st) cudaStreamDestroy(st); }
  } cleanup{st, e0, e1};
  check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
  check_cuda(cudaEventCreate(&e1), "cudaEventCreate");
  DeviceBuffer scratch, out, ctr;
  const uint64_t cap = device_capacity(m);
  out.alloc(cap * sizeof(ws_match));
  ctr.alloc(64);
  RegexLaunch rl{d, len, out.as<ws_match>(), cap, ctr.as<unsigned long long>(), WS_REGEX_SPECULATIVE};
  std::vector<float> ts;
  for (int r = -1; r < reps; ++r) {  // r = -1: warm-up (sizes the scratch)
    check_cuda(cudaMemsetAsync(ctr.ptr, 0, 8, st), "memset");
    check_cuda(cudaEventRecord(e0, st), "event");
    run_regex_scan(P, rl, st, scratch, m->ctx->sm_count, nullptr);
    check_cuda(cudaEventRecord(e1, st), "event");
    check_cuda(cudaStreamSynchronize(st), "tune scan");
    float ms = 0;
    check_cuda(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
    if (r >= 0) ts.push_back(ms);
  }
  std::sort(ts.begin(), ts.end());
  return ts.empty() ? 0.0 : ts[ts.size() / 2];
}

ws_pattern_tables regex_tables(const ws_matcher* m, std::vector<const char*>& ptrs) {
  ws_pattern_tables t;
  std::memset(&t, 0, sizeof(t));
  ptrs.clear();
  for (const auto& s : m->rx_src) ptrs.push_back(s.c_str());
  t.regex_sources = ptrs.data();
  t.regex_pattern_ids = m->rx_ids.data();
  t.n_regex = (uint32_t)m->rx_src.size();
  t.n_patterns = m->n_patterns;
  t.hash_window_len = HASH_WINDOW;
  return t;
}

}  // namespace

extern "C" ws_status ws_matcher_tune(ws_matcher* m, const uint8_t* corpus, uint64_t len, uint64_t seed, uint32_t flags,
                                     ws_tune_report* report, ws_error_info* err) {
  return guarded(err, [&] {
    if (!m || (len && !corpus)) raise(WS_ERR_INVALID_ARGUMENT, "null argument");
    ws_tune_report rep;
    std::memset(&rep, 0, sizeof(rep));
    const auto t0 = std::chrono::steady_clock::now();
    if (m->rx.n_regex) {
      if (len < 65536) raise(WS_ERR_INVALID_ARGUMENT, "tuning corpus must hold at least 64 KiB");
      check_cuda(cudaSetDevice(m->ctx->device), "cudaSetDevice");
      DeviceBuffer d;
      d.alloc(len + 64);
      check_cuda(cudaMemcpy(d.ptr, corpus, len, cudaMemcpyHostToDevice), "H2D corpus");
      const uint8_t* dc = d.as<uint8_t>();
      DeviceBuffer tiled;
      tiled.alloc(kTuneBytes + 64);
      for (uint64_t off = 0; off < kTuneBytes; off += len)
        check_cuda(cudaMemcpy(tiled.as<uint8_t>() + off, dc, std::min(len, kTuneBytes - off), cudaMemcpyDeviceToDevice),
                   "D2D tile");
      const uint64_t tlen = kTuneBytes;
      const uint64_t rlen = std::min<uint64_t>(len, 64ull << 20);  // hot-row ranking sample

      // 1. group size: re-plan at each limit, rank hot rows on the corpus, time
      if (flags & WS_TUNE_GROUPS) {
        // larger groups mean fewer lookups per input byte, as long as their
        // visited rows stay hot (the class-indexed image holds up to 1,472)
        std::vector<uint32_t> cands = {16384, 32768, 65536, 131072};
        std::vector<const char*> ptrs;
        const ws_pattern_tables t = regex_tables(m, ptrs);
        double best = 1e300;
        for (size_t k = 0; k < cands.size(); ++k) {
          ws_config c = m->cfg;
          c.dfa_max_states = cands[k];
          c.proposer = WS_PROPOSER_NONE;
          RegexPlan cand;
          try {
            plan_regex(t, c, m->ctx->sm_count, cand);
          } catch (const WsError&) {
            continue;  // a limit too small for some regex: not a candidate
          }
          regex_rerank_from_corpus(cand, dc, rlen);
          const double ms = time_regex(m, cand, tiled.as<uint8_t>(), tlen, 3);
          rep.group_candidates[k] = cands[k];
          rep.group_ms[k] = ms;
          if (ms < best) {
            best = ms;
            cand.use_proposer = m->cfg.proposer == WS_PROPOSER_MLP;
            m->rx = std::move(cand);
            m->cfg.dfa_max_states = cands[k];
          }
        }
      } else {
        regex_rerank_from_corpus(m->rx, dc, rlen);
      }

      // 2. the proposer, in the chosen plan's state numbering
      // (not when every group starts its chunks exactly: the walk would ignore
      // its guesses at every chunk the scans can use, at least half the
      // configured or smallest tuned chunk)
      bool trained = false;
      const uint64_t min_chunk = (flags & WS_TUNE_CHUNK) ? 2048 : m->rx.walk_chunk / 2 / 256 * 256;
      if (m->cfg.proposer == WS_PROPOSER_MLP && !regex_all_exact(m->rx, min_chunk)) {
        ProposerStats st;
        proposer_train(m->rx, dc, len, seed, m->ctx->sm_count, &st);
        m->rx.start_rate = st.start_rate;
        rep.proposer_top1 = st.top1;
        rep.proposer_top4 = st.top4;
        trained = true;
      }

      // 3. walk chunk, with and without the proposer
      m->rx.use_proposer = trained;
      if (flags & WS_TUNE_CHUNK) {
        const uint32_t chunks[3] = {4096, 8192, 16384};
        double best = 1e300;
        uint32_t best_chunk = m->rx.walk_chunk;
        bool best_prop = trained;
        for (int k = 0; k < 3; ++k) {
          rep.chunk_candidates[k] = chunks[k];
          m->rx.walk_chunk = chunks[k];
          for (int p = 0; p < (trained ? 2 : 1); ++p) {
            m->rx.use_proposer = p == 1;
            const double ms = time_regex(m, m->rx, tiled.as<uint8_t>(), tlen, 3);
            rep.chunk_ms[k][p] = ms;
            if (ms < best) { best = ms; best_chunk = chunks[k]; best_prop = p == 1; }
          }
        }
        m->rx.walk_chunk = best_chunk;
        m->rx.use_proposer = best_prop;
        m->cfg.walk_chunk = best_chunk;
      }
      std::lock_guard<std::mutex> g(m->info_mu);
      regex_fill_info(m->rx, m->info);
      m->info.proposer_top1 = rep.proposer_top1;
      m->info.proposer_top4 = rep.proposer_top4;
    }
    rep.dfa_max_states = m->cfg.dfa_max_states;
    rep.n_groups = m->rx.n_groups;
    rep.walk_chunk = m->rx.walk_chunk;
    rep.proposer_used = (m->rx.proposer && m->rx.use_proposer) ? 1 : 0;
    rep.tune_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    m->plan_gen++;
    if (report) *report = rep;
  });
}

extern "C" ws_status ws_matcher_set_walk(ws_matcher* m, uint32_t walk_chunk, uint32_t proposer, ws_error_info* err) {
  return guarded(err, [&] {
    if (!m) raise(WS_ERR_INVALID_ARGUMENT, "null argument");
    if (walk_chunk && (walk_chunk % 256 != 0 || walk_chunk > (1u << 24)))
      raise(WS_ERR_INVALID_ARGUMENT, "walk chunk must be a multiple of 256 bytes, at most 16 MiB");
    if (proposer != WS_PROPOSER_MLP && proposer != WS_PROPOSER_NONE) raise(WS_ERR_INVALID_ARGUMENT, "unknown proposer");
    if (proposer == WS_PROPOSER_MLP && m->rx.n_regex && !m->rx.proposer)
      raise(WS_ERR_INVALID_ARGUMENT, "no trained proposer (call ws_matcher_train_proposer or ws_matcher_tune first)");
    if (walk_chunk) {
      m->rx.walk_chunk = walk_chunk;
      m->cfg.walk_chunk = walk_chunk;
    }
    m->rx.use_proposer = proposer == WS_PROPOSER_MLP;
    m->plan_gen++;
  });
}
