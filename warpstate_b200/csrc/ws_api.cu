// C ABI of the B200 scan path: context, matcher, scan, batch and stream.
//
// Orchestration replaces GpuMatcher::scan / scan_once / scan_chunk
// (core/src/gpu/mod.rs:223-388) and the dispatch helpers
// (core/src/gpu/dispatch.rs:57-301): one device-resident copy of the pattern
// tables per matcher, per-call streams and scratch from a pool, inputs copied
// once, the whole input scanned in one launch sequence (no 128 MiB chunking and
// no 16 MiB regex cap -- those limits came from wgpu buffer bindings and the
// WGSL shader's quadratic worst case), overflow reported with the true count
// and never answered by a CPU fallback.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>

#include "ws_matcher.h"
#include "ws_proposer.h"

using namespace ws;

namespace ws {

void ensure(DeviceBuffer& b, size_t need) {
  if (b.bytes >= need) return;
  size_t n = 1;
  while (n < need) n <<= 1;
  b.alloc(n);
}

void fill_err(ws_error_info* err, const Failure& f) {
  if (!err) return;
  err->index = f.index;
  err->count = f.count;
  err->max = f.max;
  std::snprintf(err->message, sizeof(err->message), "%s", f.message.c_str());
}

bool is_pinned(const void* p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeHost;
}

void sort_matches(ws_match* p, uint64_t n) {
  std::sort(p, p + n, [](const ws_match& a, const ws_match& b) {
    if (a.start != b.start) return a.start < b.start;
    if (a.pattern_id != b.pattern_id) return a.pattern_id < b.pattern_id;
    return a.end < b.end;
  });
}

uint8_t* staging(Scratch& s, size_t piece) {
  if (s.pinned_bytes < 2 * piece) {
    for (int k = 0; k < 2; ++k)
      if (s.pin_busy[k]) check_cuda(cudaEventSynchronize(s.ev[2 + k]), "staging sync");
    s.pin_busy[0] = s.pin_busy[1] = false;
    if (s.pinned) cudaFreeHost(s.pinned);
    s.pinned = nullptr;
    s.pinned_bytes = 0;
    check_cuda(cudaHostAlloc(&s.pinned, 2 * piece, cudaHostAllocDefault), "cudaHostAlloc");
    s.pinned_bytes = 2 * piece;
  }
  return static_cast<uint8_t*>(s.pinned);
}

uint8_t* staging_slot(Scratch& s, int k, size_t piece) {
  uint8_t* pin = staging(s, piece);
  if (s.pin_busy[k]) {
    check_cuda(cudaEventSynchronize(s.ev[2 + k]), "staging sync");
    s.pin_busy[k] = false;
  }
  return pin + (size_t)k * (s.pinned_bytes / 2);
}

void staging_issued(Scratch& s, int k, cudaStream_t st) {
  check_cuda(cudaEventRecord(s.ev[2 + k], st ? st : s.stream), "event record");
  s.pin_busy[k] = true;
}

void stage_copy(Scratch& s, uint8_t* d_dst, const uint8_t* data, uint64_t len) {
  if (len == 0) return;
  if (is_pinned(data)) {
    check_cuda(cudaMemcpyAsync(d_dst, data, len, cudaMemcpyHostToDevice, s.stream), "H2D input");
    return;
  }
  // pageable: double-buffered staging through pinned memory
  const size_t piece = 8u << 20;
  for (uint64_t off = 0, k = 0; off < len; off += piece, ++k) {
    const int slot = (int)(k & 1);
    uint8_t* pin = staging_slot(s, slot, piece);
    size_t n = (size_t)std::min<uint64_t>(piece, len - off);
    std::memcpy(pin, data + off, n);
    check_cuda(cudaMemcpyAsync(d_dst + off, pin, n, cudaMemcpyHostToDevice, s.stream), "H2D input");
    staging_issued(s, slot);
  }
}

void stage_input(ws_matcher* m, Scratch& s, const uint8_t* data, uint64_t len) {
  (void)m;
  ensure(s.input, len + 64);
  stage_copy(s, s.input.as<uint8_t>(), data, len);
}

uint64_t device_capacity(const ws_matcher* m) { return std::max<uint64_t>(m->cfg.max_matches, 1); }

uint32_t enqueue_scan(ws_matcher* m, Scratch& s, cudaStream_t st, const uint8_t* d_data, uint64_t len,
                      ws_match* d_out, uint64_t cap, unsigned long long* d_counter, const ScanExtras& x) {
  const bool prof = m->profile;
  uint32_t launches = 0;
  m->use_summed = false;
  check_cuda(cudaMemsetAsync(d_counter, 0, sizeof(unsigned long long), st), "memset counter");
  if (prof) check_cuda(cudaEventRecord(m->pev[0], st), "event");
  if (m->lit.n_literals && x.literals) {
    uint64_t scap = literal_survivor_cap(len);
    ensure(s.lit, literal_scratch_bytes(scap));
    LiteralLaunch ll{d_data, len, d_out, cap, d_counter, s.lit.ptr, scap};
    ll.item_end = x.item_end;
    ll.n_items = x.n_items;
    ll.min_end = x.lit_min_end;
    ll.max_start = x.lit_max_start;
    launch_literal_scan(m->lit, ll, st, m->ctx->sm_count);
    launches += 2;
  }
  if (prof) check_cuda(cudaEventRecord(m->pev[1], st), "event");
  if (m->rx.n_regex) {
    RegexLaunch rl{d_data, len, d_out, cap, d_counter, m->cfg.regex_mode};
    rl.item_end = x.item_end;
    rl.n_items = x.n_items;
    rl.cursor = x.cursor;
    rl.base = x.base;
    rl.frontier = x.frontier;
    rl.need = m->need_dev;
    if (m->need_host) {
      // a quarter more than was needed: the reverse walks' shared marks are
      // lossy, so a repeated scan can append a few more candidates
      const volatile unsigned long long* need = m->need_host;
      const uint64_t k = need[0], e = need[1];
      rl.k_min = k ? k + k / 4 : 0;
      rl.ev_min = e ? e + e / 4 : 0;
    }
    launches += run_regex_scan(m->rx, rl, st, s.rx, m->ctx->sm_count, prof ? m->rx_events : nullptr);
  }
  if (prof) check_cuda(cudaEventRecord(m->pev[2], st), "event");
  check_cuda(cudaEventRecord(s.busy, st), "event");
  std::lock_guard<std::mutex> g(m->info_mu);
  m->info.last_launches = launches;
  m->info.last_chunks = m->rx.last_chunks;
  return launches;
}

void read_phases(ws_matcher* m, double* ms) {
  check_cuda(cudaEventSynchronize(m->pev[2]), "event sync");
  ws_matcher_info tmp;
  std::memset(&tmp, 0, sizeof(tmp));
  float a = 0, b = 0;
  if (cudaEventElapsedTime(&a, m->pev[0], m->pev[1]) == cudaSuccess) tmp.last_kernel_ms[0] = a;
  if (cudaEventElapsedTime(&b, m->pev[0], m->pev[2]) == cudaSuccess) tmp.last_kernel_ms[7] = b;
  if (m->rx.n_regex) regex_collect_timing(m->rx, m->rx_events, tmp);
  cudaGetLastError();
  for (int k = 0; k < 8; ++k) ms[k] = tmp.last_kernel_ms[k];
}

void raise_candidates_unknown(ws_matcher* m) {
  const uint64_t need = m->need_host ? std::max(m->need_host[0], m->need_host[1]) : 0;
  raise(WS_ERR_OVERFLOW, "regex candidates exceed what the device buffers can hold", 0, need,
        std::min<uint64_t>(need, 0x7FFFFFFFull));
}

bool repeat_scan(ws_matcher* m, unsigned long long count, int attempt) {
  if (count == kCountTimeout) raise(WS_ERR_TIMEOUT, "a device-side wait of the scan ran out");
  if (count != kCountUnknown) return false;
  if (attempt + 1 >= kCandidateRetries) raise_candidates_unknown(m);
  return true;
}

// The windowed form of ws_scan for a large pinned host input (see ws_scan).
void scan_overlapped(ws_matcher* m, Scratch& s, const uint8_t* data, uint64_t len, ws_match* out, uint64_t cap,
                     uint64_t* n_out) {
  const uint64_t W = kOverlapWindow;
  const uint64_t nwin = (len + W - 1) / W;
  ensure(s.input, len + 64);
  if (!s.copy) check_cuda(cudaStreamCreateWithFlags(&s.copy, cudaStreamNonBlocking), "cudaStreamCreate");
  check_cuda(cudaStreamWaitEvent(s.copy, s.busy, 0), "wait");
  std::vector<cudaEvent_t> arrived(nwin, nullptr);
  struct Events {
    std::vector<cudaEvent_t>& e;
    ~Events() { for (auto x : e) if (x) cudaEventDestroy(x); }
  } cleanup{arrived};
  uint8_t* d = s.input.as<uint8_t>();
  for (uint64_t k = 0; k < nwin; ++k) {
    const uint64_t off = k * W, n = std::min(W, len - off);
    check_cuda(cudaEventCreateWithFlags(&arrived[k], cudaEventDisableTiming), "cudaEventCreate");
    check_cuda(cudaMemcpyAsync(d + off, data + off, n, cudaMemcpyHostToDevice, s.copy), "H2D window");
    check_cuda(cudaEventRecord(arrived[k], s.copy), "event");
  }
  const uint64_t dcap = device_capacity(m);
  auto* d_counter = s.counters.as<unsigned long long>();
  unsigned long long count = 0;
  try {
    check_cuda(cudaMemsetAsync(d + len, 0, 64, s.stream), "memset pad");
    ensure(s.out64, dcap * sizeof(ws_match64));
    for (int attempt = 0;; ++attempt) {
      enqueue_windows(m, s, s.stream, d, len, W, s.out64.as<ws_match64>(), dcap, d_counter, [&](uint64_t end) {
        check_cuda(cudaStreamWaitEvent(s.stream, arrived[(end - 1) / W], 0), "wait window");
      });
      check_cuda(cudaMemcpyAsync(&count, d_counter, sizeof(count), cudaMemcpyDeviceToHost, s.stream), "D2H count");
      check_cuda(cudaStreamSynchronize(s.stream), "scan");
      if (!repeat_scan(m, count, attempt)) break;
    }
  } catch (...) {
    cudaStreamSynchronize(s.copy);  // no copy may still read the caller's input
    throw;
  }
  *n_out = count;
  if (count > dcap) raise(WS_ERR_OVERFLOW, "too many matches", 0, count, dcap);
  if (count > cap) raise(WS_ERR_OVERFLOW, "too many matches for the output buffer", 0, count, cap);
  if (count > kMaxDeviceSorted) {
    std::vector<ws_match64> wide(count);
    check_cuda(cudaMemcpy(wide.data(), s.out64.ptr, count * sizeof(ws_match64), cudaMemcpyDeviceToHost),
               "D2H matches");
    for (uint64_t k = 0; k < count; ++k)
      out[k] = ws_match{wide[k].pattern_id, (uint32_t)wide[k].start, (uint32_t)wide[k].end};
    sort_matches(out, count);
    return;
  }
  // the windows' output buffer is free again: narrow into it, then order
  narrow_matches_device(s.out64.as<ws_match64>(), s.out.as<ws_match>(), count, s.stream);
  read_sorted(s, s.out.as<ws_match>(), count, out);
}

void read_sorted(Scratch& s, const ws_match* d_res, uint64_t count, ws_match* out) {
  if (!count) return;
  const bool on_device = count <= kMaxDeviceSorted;
  if (on_device && count > 1) {
    ensure(s.sorted, count * sizeof(ws_match));
    sort_matches_device(s, d_res, s.sorted.as<ws_match>(), count, s.stream);
    d_res = s.sorted.as<ws_match>();
  }
  check_cuda(cudaMemcpyAsync(out, d_res, count * sizeof(ws_match), cudaMemcpyDeviceToHost, s.stream), "D2H matches");
  check_cuda(cudaStreamSynchronize(s.stream), "D2H sync");
  if (!on_device) sort_matches(out, count);
}

}  // namespace ws

std::unique_ptr<Scratch> ws_matcher::take() {
  {
    std::lock_guard<std::mutex> g(pool_mu);
    if (!pool.empty()) {
      auto s = std::move(pool.back());
      pool.pop_back();
      return s;
    }
  }
  check_cuda(cudaSetDevice(ctx->device), "cudaSetDevice");
  auto s = std::make_unique<Scratch>();
  check_cuda(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "cudaStreamCreate");
  for (auto& e : s->ev) check_cuda(cudaEventCreate(&e), "cudaEventCreate");
  check_cuda(cudaEventCreateWithFlags(&s->busy, cudaEventDisableTiming), "cudaEventCreate");
  s->counters.alloc(64);
  return s;
}

void ws_matcher::give(std::unique_ptr<Scratch> s) {
  std::lock_guard<std::mutex> g(pool_mu);
  pool.push_back(std::move(s));
}

extern "C" {

int ws_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) { cudaGetLastError(); return 0; }
  return n;
}

ws_status ws_ctx_create(int device, ws_ctx** out, ws_error_info* err) {
  return guarded(err, [&] {
    if (!out) raise(WS_ERR_INVALID_ARGUMENT, "null out");
    int n = ws_device_count();
    if (n <= 0) raise(WS_ERR_NO_DEVICE, "no GPU adapter available (no CUDA device)");
    if (device < 0 || device >= n) raise(WS_ERR_NO_DEVICE, "device index out of range");
    check_cuda(cudaSetDevice(device), "cudaSetDevice");
    cudaDeviceProp prop;
    check_cuda(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
    if (prop.major < 10) raise(WS_ERR_NO_DEVICE, "device is not sm_100 class (B200 required)");
    auto* c = new ws_ctx();
    c->device = device;
    c->sm_count = prop.multiProcessorCount;
    *out = c;
  });
}

void ws_ctx_destroy(ws_ctx* ctx) { delete ctx; }

void ws_config_default(ws_config* c) {
  std::memset(c, 0, sizeof(*c));
  c->gpu_threshold = 65536;                  // core/src/config.rs:28
  c->gpu_max_input_size = 128ull << 20;       // core/src/config.rs:4
  c->max_matches = 1000000;                  // core/src/config.rs:35
  c->chunk_size = 128ull << 20;               // core/src/config.rs:14
  c->chunk_overlap = 4096;                   // core/src/config.rs:21
  c->regex_mode = WS_REGEX_SPECULATIVE;
  c->dfa_max_states = 8192;
  c->walk_chunk = 4096;
  c->proposer = WS_PROPOSER_MLP;
  c->proposer_train_bytes = 256ull << 20;
  c->proposer_seed = 0x5EEDF00Dull;
}

ws_status ws_matcher_create(ws_ctx* ctx, const ws_pattern_tables* t, const ws_config* cfg,
                            ws_matcher** out, ws_error_info* err) {
  return guarded(err, [&] {
    if (!ctx || !t || !out) raise(WS_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (t->n_literals + t->n_regex == 0) raise(WS_ERR_EMPTY_PATTERN_SET, "pattern set is empty");
    check_cuda(cudaSetDevice(ctx->device), "cudaSetDevice");
    auto m = std::make_unique<ws_matcher>();
    m->ctx = ctx;
    if (cfg) m->cfg = *cfg; else ws_config_default(&m->cfg);
    m->n_patterns = t->n_patterns;
    m->is_regex.assign(t->n_patterns, 0);
    for (uint32_t r = 0; r < t->n_regex; ++r) {
      if (t->regex_pattern_ids[r] < t->n_patterns) m->is_regex[t->regex_pattern_ids[r]] = 1;
      m->rx_src.emplace_back(t->regex_sources[r]);
      m->rx_ids.push_back(t->regex_pattern_ids[r]);
    }
    for (uint32_t i = 0; i < t->n_literals; ++i) m->max_literal_len = std::max(m->max_literal_len, t->offsets[2 * i + 1]);
    std::memset(&m->info, 0, sizeof(m->info));
    plan_literals(*t, m->lit);
    plan_regex(*t, m->cfg, ctx->sm_count, m->rx);
    m->info.n_literals = t->n_literals;
    m->info.n_regex = t->n_regex;
    m->info.filter_q = m->lit.gram_len;
    m->info.max_literal_len = m->max_literal_len;
    m->info.filter_period = m->lit.period;
    m->info.filter_bits = m->lit.table_bits;
    regex_fill_info(m->rx, m->info);
    if (t->n_regex) {
      check_cuda(cudaHostAlloc(reinterpret_cast<void**>(&m->need_host), 2 * sizeof(unsigned long long),
                               cudaHostAllocMapped), "cudaHostAlloc(mapped)");
      m->need_host[0] = m->need_host[1] = 0;
      check_cuda(cudaHostGetDevicePointer(reinterpret_cast<void**>(&m->need_dev), m->need_host, 0),
                 "cudaHostGetDevicePointer");
    }
    m->profile = (m->cfg.flags & WS_FLAG_PROFILE) != 0;
    if (m->profile) {
      for (auto& e : m->pev) check_cuda(cudaEventCreate(&e), "cudaEventCreate");
      for (auto& e : m->rx_events) check_cuda(cudaEventCreate(&e), "cudaEventCreate");
    }
    *out = m.release();
  });
}

void ws_matcher_destroy(ws_matcher* m) {
  if (!m) return;
  cudaSetDevice(m->ctx->device);
  release_staging(m);
  delete m;
}

ws_status ws_scan(ws_matcher* m, const uint8_t* data, uint64_t len, ws_match* out, uint64_t cap,
                  uint64_t* n_out, ws_error_info* err) {
  return guarded(err, [&] {
    if (!m || !n_out || (len && !data) || (cap && !out)) raise(WS_ERR_INVALID_ARGUMENT, "null argument");
    *n_out = 0;
    if (len > 0xFFFFFFFFull)
      raise(WS_ERR_INPUT_TOO_LARGE, "scan input is too large for 32-bit match offsets", 0, len, 0xFFFFFFFFull);
    if (len == 0) return;  // no pattern matches empty input on the GPU path
    check_cuda(cudaSetDevice(m->ctx->device), "cudaSetDevice");
    auto s = m->take();
    struct Return { ws_matcher* m; std::unique_ptr<Scratch>& s; ~Return() { if (s) m->give(std::move(s)); } } ret{m, s};
    check_cuda(cudaStreamWaitEvent(s->stream, s->busy, 0), "wait");
    uint64_t dcap = device_capacity(m);
    auto* d_counter = s->counters.as<unsigned long long>();
    if (len >= 2 * kOverlapWindow && is_pinned(data)) {
      // large pinned input: copy it in windows on a second stream and scan
      // each window as soon as it has arrived, so that the host-to-device
      // copy of window k+1 runs under the scan of window k
      scan_overlapped(m, *s, data, len, out, cap, n_out);
      return;
    }
    stage_input(m, *s, data, len);
    ensure(s->out, dcap * sizeof(ws_match));
    unsigned long long count = 0;
    for (int attempt = 0;; ++attempt) {
      enqueue_scan(m, *s, s->stream, s->input.as<uint8_t>(), len, s->out.as<ws_match>(), dcap, d_counter);
      check_cuda(cudaMemcpyAsync(&count, d_counter, sizeof(count), cudaMemcpyDeviceToHost, s->stream), "D2H count");
      check_cuda(cudaStreamSynchronize(s->stream), "scan");
      if (!repeat_scan(m, count, attempt)) break;
    }
    *n_out = count;
    if (count > dcap) raise(WS_ERR_OVERFLOW, "too many matches", 0, count, dcap);
    if (count > cap) raise(WS_ERR_OVERFLOW, "too many matches for the output buffer", 0, count, cap);
    read_sorted(*s, s->out.as<ws_match>(), count, out);
  });
}

ws_status ws_scan_device(ws_matcher* m, const uint8_t* d_data, uint64_t len, ws_match* d_out, uint64_t cap,
                         uint64_t* d_count, void* stream, ws_error_info* err) {
  return guarded(err, [&] {
    if (!m || !d_count || (len && !d_data)) raise(WS_ERR_INVALID_ARGUMENT, "null argument");
    if (((uintptr_t)d_data & 15) != 0) raise(WS_ERR_INVALID_ARGUMENT, "device input must be 16-byte aligned");
    if (len > 0xFFFFFFFFull)
      raise(WS_ERR_INPUT_TOO_LARGE, "scan input is too large for 32-bit match offsets", 0, len, 0xFFFFFFFFull);
    check_cuda(cudaSetDevice(m->ctx->device), "cudaSetDevice");
    auto s = m->take();
    struct Return { ws_matcher* m; std::unique_ptr<Scratch>& s; ~Return() { if (s) m->give(std::move(s)); } } ret{m, s};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // Reuse of this scratch is ordered after its previous user's work.
    check_cuda(cudaStreamWaitEvent(st, s->busy, 0), "wait");
    auto* d_counter = reinterpret_cast<unsigned long long*>(d_count);
    if (len == 0) {
      check_cuda(cudaMemsetAsync(d_counter, 0, 8, st), "memset");
      return;
    }
    enqueue_scan(m, *s, st, d_data, len, d_out, cap, d_counter);
  });
}

ws_status ws_matcher_get_info(const ws_matcher* m, ws_matcher_info* out) {
  if (!m || !out) return WS_ERR_INVALID_ARGUMENT;
  auto* mm = const_cast<ws_matcher*>(m);
  std::lock_guard<std::mutex> g(mm->info_mu);
  if (mm->profile && mm->use_summed) {
    for (int k = 0; k < 8; ++k) mm->info.last_kernel_ms[k] = mm->summed_ms[k];
  } else if (mm->profile && mm->pev[2] && cudaEventQuery(mm->pev[2]) != cudaErrorNotReady) {
    cudaEventSynchronize(mm->pev[2]);
    float a = 0, b = 0;
    if (cudaEventElapsedTime(&a, mm->pev[0], mm->pev[1]) == cudaSuccess) mm->info.last_kernel_ms[0] = a;
    if (cudaEventElapsedTime(&b, mm->pev[0], mm->pev[2]) == cudaSuccess) mm->info.last_kernel_ms[7] = b;
    regex_collect_timing(mm->rx, mm->rx_events, mm->info);
    cudaGetLastError();
  }
  *out = mm->info;
  return WS_OK;
}

const char* ws_status_name(ws_status s) {
  switch (s) {
    case WS_OK: return "Ok";
    case WS_ERR_EMPTY_PATTERN_SET: return "EmptyPatternSet";
    case WS_ERR_EMPTY_PATTERN: return "EmptyPattern";
    case WS_ERR_NO_DEVICE: return "NoGpuAdapter";
    case WS_ERR_DEVICE: return "GpuDeviceError";
    case WS_ERR_BUFFER_MAP: return "BufferMapFailed";
    case WS_ERR_COMPILE: return "PatternCompilationFailed";
    case WS_ERR_DFA_OOB: return "DfaOutOfBounds";
    case WS_ERR_PATTERN_TOO_LARGE: return "PatternTooLarge";
    case WS_ERR_PATTERN_SET_TOO_LARGE: return "PatternSetTooLarge";
    case WS_ERR_INPUT_TOO_LARGE: return "InputTooLarge";
    case WS_ERR_OVERFLOW: return "MatchBufferOverflow";
    case WS_ERR_PATHOLOGICAL: return "PathologicalRegex";
    case WS_ERR_TIMEOUT: return "Timeout";
    case WS_ERR_INVALID_ARGUMENT: return "InvalidArgument";
  }
  return "Unknown";
}

}  // extern "C"

extern "C" ws_status ws_regex_candidates(ws_matcher* m, const uint8_t* data, uint64_t len, uint32_t mode,
                                         ws_match* out, uint64_t cap, uint64_t* n_out, ws_error_info* err) {
  return guarded(err, [&] {
    if (!m || !n_out || (len && !data) || (cap && !out)) raise(WS_ERR_INVALID_ARGUMENT, "null argument");
    *n_out = 0;
    if (len > 0xFFFFFFFFull)
      raise(WS_ERR_INPUT_TOO_LARGE, "scan input is too large for 32-bit match offsets", 0, len, 0xFFFFFFFFull);
    if (len == 0 || !m->rx.n_regex) return;
    check_cuda(cudaSetDevice(m->ctx->device), "cudaSetDevice");
    auto s = m->take();
    struct Return { ws_matcher* m; std::unique_ptr<Scratch>& s; ~Return() { if (s) m->give(std::move(s)); } } ret{m, s};
    check_cuda(cudaStreamWaitEvent(s->stream, s->busy, 0), "wait");
    stage_input(m, *s, data, len);
    *n_out = regex_candidates(m->rx, s->input.as<uint8_t>(), len, mode, s->stream, s->rx, m->ctx->sm_count, out, cap);
    check_cuda(cudaEventRecord(s->busy, s->stream), "event");
  });
}

namespace ws {
// Used by the allocation-free scan (ws_noalloc.cu), which sees ws_matcher only
// as an opaque type.
const LiteralPlan* matcher_literal_plan(const ws_matcher* m, uint32_t* n_regex, int* device, int* sm_count) {
  *n_regex = m->rx.n_regex;
  *device = m->ctx->device;
  *sm_count = m->ctx->sm_count;
  return &m->lit;
}
}  // namespace ws

extern "C" ws_status ws_matcher_train_proposer(ws_matcher* m, const uint8_t* corpus, uint64_t len, uint64_t seed,
                                               ws_error_info* err) {
  return guarded(err, [&] {
    if (!m || (len && !corpus)) raise(WS_ERR_INVALID_ARGUMENT, "null argument");
    if (!m->rx.n_regex) return;
    check_cuda(cudaSetDevice(m->ctx->device), "cudaSetDevice");
    DeviceBuffer d;
    d.alloc(len + 64);
    check_cuda(cudaMemcpy(d.ptr, corpus, len, cudaMemcpyHostToDevice), "H2D corpus");
    // first place the hottest DFA rows of this workload in shared memory, then
    // learn the boundary states in the resulting numbering
    regex_rerank_from_corpus(m->rx, d.as<uint8_t>(), len);
    ProposerStats st;
    proposer_train(m->rx, d.as<uint8_t>(), len, seed, m->ctx->sm_count, &st);
    m->rx.start_rate = st.start_rate;
    m->plan_gen++;
    std::lock_guard<std::mutex> g(m->info_mu);
    m->info.proposer_top1 = st.top1;
    m->info.proposer_top4 = st.top4;
  });
}
