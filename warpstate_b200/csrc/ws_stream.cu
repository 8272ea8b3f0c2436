// Stream scan: bytes fed in pieces, matches equal to one scan of the whole
// stream, with 64-bit offsets.
//
// Replaces StreamPipeline::scan (core/src/pipeline.rs:87-153), which rescans
// `overlap_window` bytes around every chunk boundary and then keeps, per
// (pattern_id, start), the shortest end -- a heuristic that can report a
// regex match the whole-input find_iter would not.  Here the stream carries
// exact state between pieces:
//   - a device window holding the stream bytes that later matches can still
//     touch: the last max_literal_len - 1 bytes (a literal occurrence that
//     ends in a later piece starts there) and every byte from the regex
//     frontier on;
//   - per regex, the find_iter cursor (u64, device-resident): matches
//     starting before it are decided.
// A regex start s is decided once s + max_len <= bytes seen (no match from s
// can end later), so each piece decides every start below
// frontier = seen - max_len + 1 and the chain resumes from the cursor next
// time.  Literal occurrences are complete as soon as their last byte is seen;
// each piece reports those that end inside it.  Regexes with unbounded
// matches keep the whole undecided stream in the window (decided at the end).
#include <cuda_runtime.h>

#include <algorithm>

#include "ws_matcher.h"

using namespace ws;

struct ws_stream {
  ws_matcher* m = nullptr;
  std::unique_ptr<Scratch> s;
  DeviceBuffer win[2];      // ping-pong windows
  int cur = 0;
  uint64_t win_base = 0;    // stream offset of the window's first byte
  uint64_t win_len = 0;
  uint64_t seen = 0;        // bytes fed so far
  uint64_t frontier = 0;    // regex starts below it are decided
  DeviceBuffer cursor;      // per-regex find_iter position (u64)
  DeviceBuffer cursor_bak;  // the cursors before the window scan in flight (restored to repeat it)
  std::vector<ws_match64> pending;  // decided, not yet delivered
  size_t delivered = 0;
  std::vector<ws_match> host;       // per-step readback
  unsigned long long count = 0;     // the step's match count, read back
  bool failed = false;
  bool ended = false;
  ~ws_stream() {
    if (s && m) m->give(std::move(s));
  }
};

namespace {

// New data per step: the window plus the step must stay below 4 GiB (32-bit
// offsets inside a launch).
uint64_t step_bytes(const ws_matcher* m) { return (uint64_t)(m->cfg.window_mib ? m->cfg.window_mib : 1024) << 20; }

int64_t regex_max_len(const ws_matcher* m) { return m->rx.n_regex ? m->rx.max_len : 0; }

// Enqueues one scan of the current window; false when there is nothing to scan.
bool enqueue_window(ws_stream* st, bool literals, uint64_t lit_min_end, uint64_t frontier) {
  ws_matcher* m = st->m;
  Scratch& s = *st->s;
  const uint64_t dcap = device_capacity(m);
  ensure(s.out, dcap * sizeof(ws_match));
  auto* d_counter = s.counters.as<unsigned long long>();
  ScanExtras x;
  x.literals = literals;
  x.lit_min_end = lit_min_end;
  x.cursor = m->rx.n_regex ? st->cursor.as<unsigned long long>() : nullptr;
  x.base = st->win_base;
  x.frontier = frontier;
  if (!literals && !m->rx.n_regex) return false;
  if (m->rx.n_regex)
    check_cuda(cudaMemcpyAsync(st->cursor_bak.ptr, st->cursor.ptr, (size_t)m->rx.n_regex * 8,
                               cudaMemcpyDeviceToDevice, s.stream), "D2D cursor");
  enqueue_scan(m, s, s.stream, st->win[st->cur].as<uint8_t>(), st->win_len, s.out.as<ws_match>(), dcap, d_counter, x);
  check_cuda(cudaMemcpyAsync(&st->count, d_counter, sizeof(st->count), cudaMemcpyDeviceToHost, s.stream),
             "D2H count");
  return true;
}

// Waits for the window scan just enqueued; false when its regex candidates
// overflowed (the cursors are then back where the scan found them, so the
// window can be scanned again).
bool window_done(ws_stream* st, int attempt) {
  ws_matcher* m = st->m;
  Scratch& s = *st->s;
  check_cuda(cudaStreamSynchronize(s.stream), "stream scan");
  if (!repeat_scan(m, st->count, attempt)) return true;
  check_cuda(cudaMemcpyAsync(st->cursor.ptr, st->cursor_bak.ptr, (size_t)m->rx.n_regex * 8,
                             cudaMemcpyDeviceToDevice, s.stream), "D2D cursor");
  return false;
}

// Appends the decided matches of the window scan that window_done accepted.
void finish_window(ws_stream* st) {
  ws_matcher* m = st->m;
  Scratch& s = *st->s;
  const uint64_t dcap = device_capacity(m);
  const unsigned long long count = st->count;
  if (count > dcap) raise(WS_ERR_OVERFLOW, "too many matches in one stream piece", 0, count, dcap);
  if (count) {
    st->host.resize(count);
    read_sorted(s, s.out.as<ws_match>(), count, st->host.data());
    for (const ws_match& mm : st->host) {
      ws_match64 o;
      o.pattern_id = mm.pattern_id;
      o.reserved = 0;
      o.start = st->win_base + mm.start;
      o.end = st->win_base + mm.end;
      st->pending.push_back(o);
    }
  }
}

// Runs one scan of the current window and appends the decided matches.
void scan_window(ws_stream* st, bool literals, uint64_t lit_min_end, uint64_t frontier) {
  for (int attempt = 0;; ++attempt) {
    if (!enqueue_window(st, literals, lit_min_end, frontier)) return;
    if (window_done(st, attempt)) break;
  }
  finish_window(st);
}

}  // namespace

namespace ws {

StepPlan plan_step(const ws_matcher* m, uint64_t win_base, uint64_t old_seen, uint64_t seen, uint64_t frontier,
                   bool last) {
  StepPlan p;
  // bytes [keep, old_seen) stay in the window: the literal tail and every
  // undecided regex start
  uint64_t keep = old_seen;
  if (m->lit.n_literals && m->max_literal_len > 1)
    keep = std::min(keep, old_seen - std::min<uint64_t>(old_seen, m->max_literal_len - 1));
  if (m->rx.n_regex) keep = std::min(keep, frontier);
  // look-behind assertions read the byte before a start: keep it too
  if (m->rx.has_context && keep > 0 && keep == frontier) keep -= 1;
  p.keep = std::max(keep, win_base);
  const int64_t mx = regex_max_len(m);
  if (last) {
    frontier = seen;
  } else if (mx >= 0 && seen + 1 > (uint64_t)mx) {
    frontier = std::max(frontier, seen + 1 - (uint64_t)mx);
  }
  p.frontier = std::min(frontier, seen);
  if (seen - p.keep > 0xFFFFFFFFull - 64)
    raise(WS_ERR_INPUT_TOO_LARGE, "scan window exceeds 32-bit offsets (a regex with unbounded matches keeps the "
          "whole undecided input in the window)", 0, seen - p.keep, 0xFFFFFFFFull - 64);
  return p;
}

}  // namespace ws

namespace {

// Plans the step that appends `len` bytes (len <= step_bytes) and enqueues its
// window on `cs`: the carried tail of the current window, then the new bytes
// (a stream other than the scratch's own takes pinned input only).
StepPlan copy_step(ws_stream* st, const uint8_t* data, uint64_t len, cudaStream_t cs) {
  ws_matcher* m = st->m;
  Scratch& s = *st->s;
  const uint64_t old_seen = st->seen;
  const StepPlan plan = plan_step(m, st->win_base, old_seen, old_seen + len, st->frontier, false);
  const uint64_t carry = old_seen - plan.keep;
  DeviceBuffer& dst = st->win[st->cur ^ 1];
  ensure(dst, carry + len + 64);
  if (carry)
    check_cuda(cudaMemcpyAsync(dst.ptr, st->win[st->cur].as<uint8_t>() + (plan.keep - st->win_base), carry,
                               cudaMemcpyDeviceToDevice, cs), "D2D carry");
  if (cs == s.stream)
    stage_copy(s, dst.as<uint8_t>() + carry, data, len);
  else
    check_cuda(cudaMemcpyAsync(dst.as<uint8_t>() + carry, data, len, cudaMemcpyHostToDevice, cs), "H2D step");
  check_cuda(cudaMemsetAsync(dst.as<uint8_t>() + carry + len, 0, 64, cs), "memset pad");
  return plan;
}

// Makes the window that copy_step filled current; returns the literal
// min-end of its scan (occurrences ending before it were reported).
uint64_t advance_step(ws_stream* st, uint64_t len, const StepPlan& plan) {
  const uint64_t old_seen = st->seen;
  st->cur ^= 1;
  st->win_base = plan.keep;
  st->win_len = old_seen - plan.keep + len;
  st->seen = old_seen + len;
  st->frontier = plan.frontier;
  return old_seen - plan.keep;
}

// Appends `len` bytes (len <= step_bytes) to the stream and decides what it can.
void feed_step(ws_stream* st, const uint8_t* data, uint64_t len) {
  const StepPlan plan = copy_step(st, data, len, st->s->stream);
  const uint64_t lit_min_end = advance_step(st, len, plan);
  scan_window(st, st->m->lit.n_literals != 0, lit_min_end, plan.frontier);
}

// Feeds a pinned input of several steps with the copy of step k+1 (on the
// scratch's copy stream) running while step k is scanned.  The schedule is
// the one feed_step follows, so the windows and results are the same.
void feed_pipelined(ws_stream* st, const uint8_t* data, uint64_t len) {
  Scratch& s = *st->s;
  const uint64_t step = step_bytes(st->m);
  if (!s.copy) check_cuda(cudaStreamCreateWithFlags(&s.copy, cudaStreamNonBlocking), "cudaStreamCreate");
  // the copy stream follows everything enqueued on the scratch's stream
  check_cuda(cudaEventRecord(s.busy, s.stream), "event");
  check_cuda(cudaStreamWaitEvent(s.copy, s.busy, 0), "wait");
  try {
    uint64_t n = std::min(step, len);
    StepPlan plan = copy_step(st, data, n, s.copy);
    check_cuda(cudaEventRecord(s.ev[0], s.copy), "event");
    for (uint64_t off = 0, k = 0; off < len; ++k) {
      check_cuda(cudaStreamWaitEvent(s.stream, s.ev[k & 1], 0), "wait step");
      const uint64_t lit_min_end = advance_step(st, n, plan);
      const uint64_t next = off + n, n_next = std::min(step, len - next);
      // the next window is the other buffer, whose last scan has finished
      if (n_next) {
        plan = copy_step(st, data + next, n_next, s.copy);
        check_cuda(cudaEventRecord(s.ev[(k + 1) & 1], s.copy), "event");
      }
      scan_window(st, st->m->lit.n_literals != 0, lit_min_end, st->frontier);
      off = next;
      n = n_next;
    }
  } catch (...) {
    cudaStreamSynchronize(s.copy);  // no copy may still read the caller's input
    throw;
  }
}

// Appends one window's matches to a 64-bit output: offsets shifted by the
// window's stream offset, the step's true count added to the running total
// (so a total above `cap` reports the overflow with the true count).
__global__ void __launch_bounds__(1024) widen_kernel(const ws_match* in, const unsigned long long* step_count,
                                                     uint64_t step_cap, uint64_t base, ws_match64* out, uint64_t cap,
                                                     unsigned long long* total) {
  const unsigned long long n = *step_count;
  const unsigned long long at = *total;
  if (n >= kCountTimeout || at >= kCountTimeout) {  // a timeout or an unknown count stays in the total
    if (threadIdx.x == 0) *total = (n == kCountTimeout || at == kCountTimeout) ? kCountTimeout : kCountUnknown;
    return;
  }
  const unsigned long long avail = n < step_cap ? n : step_cap;
  for (unsigned long long k = threadIdx.x; k < avail; k += blockDim.x) {
    if (at + k >= cap) break;
    ws_match mm = in[k];
    ws_match64 o;
    o.pattern_id = mm.pattern_id;
    o.reserved = 0;
    o.start = base + mm.start;
    o.end = base + mm.end;
    out[at + k] = o;
  }
  __syncthreads();
  if (threadIdx.x == 0) *total = at + n;
}

// Copies up to `cap` undelivered matches out; overflow when some remain.
void deliver(ws_stream* st, ws_match64* out, uint64_t cap, uint64_t* n_out) {
  const uint64_t avail = st->pending.size() - st->delivered;
  const uint64_t n = std::min<uint64_t>(avail, cap);
  if (n) std::memcpy(out, st->pending.data() + st->delivered, n * sizeof(ws_match64));
  st->delivered += n;
  *n_out = n;
  if (st->delivered == st->pending.size()) {
    st->pending.clear();
    st->delivered = 0;
  }
  if (n < avail)
    raise(WS_ERR_OVERFLOW, "more stream matches than the output buffer holds; call again with no data to drain", 0,
          avail, cap);
}

}  // namespace

namespace ws {

uint32_t enqueue_windows(ws_matcher* m, Scratch& s, cudaStream_t cs, const uint8_t* d_data, uint64_t len,
                         uint64_t window, ws_match64* d_out, uint64_t cap, unsigned long long* total,
                         const std::function<void(uint64_t)>& before_window) {
  // the whole schedule is known on the host: windows are slices of d_data
  check_cuda(cudaMemsetAsync(total, 0, 8, cs), "memset count");
  const uint64_t scap = std::max<uint64_t>(cap, 1);
  ensure(s.out, scap * sizeof(ws_match));
  const size_t cursor_bytes = ((size_t)m->rx.n_regex * 8 + 255) & ~(size_t)255;
  ensure(s.aux, cursor_bytes + 256);
  auto* cursor = s.aux.as<unsigned long long>();
  auto* step_count = reinterpret_cast<unsigned long long*>(s.aux.as<uint8_t>() + cursor_bytes);
  if (m->rx.n_regex) check_cuda(cudaMemsetAsync(cursor, 0, (size_t)m->rx.n_regex * 8, cs), "memset cursor");
  uint64_t seen = 0, win_base = 0, frontier = 0;
  uint32_t launches = 0;
  double summed[8] = {};
  while (seen < len) {
    const uint64_t n = std::min<uint64_t>(window, len - seen);
    const bool last = seen + n == len;
    const StepPlan plan = plan_step(m, win_base, seen, seen + n, frontier, last);
    // windows are slices of d_data: start them on a 16-byte boundary (the
    // kernels load 16-byte vectors); the extra leading bytes hold only
    // literal occurrences already reported and regex starts already decided
    const uint64_t keep = plan.keep & ~15ull;
    ScanExtras x;
    x.literals = m->lit.n_literals != 0;
    x.lit_min_end = seen - keep;
    x.cursor = m->rx.n_regex ? cursor : nullptr;
    x.base = keep;
    x.frontier = plan.frontier;
    before_window(seen + n);
    launches += enqueue_scan(m, s, cs, d_data + keep, seen + n - keep, s.out.as<ws_match>(), scap, step_count, x);
    widen_kernel<<<1, 1024, 0, cs>>>(s.out.as<ws_match>(), step_count, scap, keep, d_out, cap, total);
    check_cuda(cudaGetLastError(), "widen_kernel");
    launches += 1;
    if (m->profile) {  // profiling: phase times summed over the windows
      double ms[8];
      read_phases(m, ms);
      for (int k = 0; k < 8; ++k) summed[k] += ms[k];
    }
    seen += n;
    win_base = keep;
    frontier = plan.frontier;
  }
  check_cuda(cudaEventRecord(s.busy, cs), "event");
  std::lock_guard<std::mutex> g(m->info_mu);
  m->info.last_launches = launches;
  if (m->profile) {
    for (int k = 0; k < 8; ++k) m->summed_ms[k] = summed[k];
    m->use_summed = true;
  }
  return launches;
}

}  // namespace ws

extern "C" {

ws_status ws_stream_begin(ws_matcher* m, ws_stream** out, ws_error_info* err) {
  return guarded(err, [&] {
    if (!m || !out) raise(WS_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    check_cuda(cudaSetDevice(m->ctx->device), "cudaSetDevice");
    auto st = std::make_unique<ws_stream>();
    st->m = m;
    st->s = m->take();
    check_cuda(cudaStreamWaitEvent(st->s->stream, st->s->busy, 0), "wait");
    if (m->rx.n_regex) {
      st->cursor.alloc((size_t)m->rx.n_regex * 8);
      st->cursor_bak.alloc((size_t)m->rx.n_regex * 8);
      check_cuda(cudaMemsetAsync(st->cursor.ptr, 0, (size_t)m->rx.n_regex * 8, st->s->stream), "memset cursor");
    }
    *out = st.release();
  });
}

ws_status ws_stream_feed(ws_stream* st, const uint8_t* data, uint64_t len, ws_match64* out, uint64_t cap,
                         uint64_t* n_out, ws_error_info* err) {
  return guarded(err, [&] {
    if (!st || !n_out || (len && !data) || (cap && !out)) raise(WS_ERR_INVALID_ARGUMENT, "null argument");
    *n_out = 0;
    if (st->failed) raise(WS_ERR_DEVICE, "stream is unusable after an earlier error");
    if (st->ended && len) raise(WS_ERR_INVALID_ARGUMENT, "stream already ended");
    check_cuda(cudaSetDevice(st->m->ctx->device), "cudaSetDevice");
    try {
      if (len > step_bytes(st->m) && is_pinned(data)) {
        feed_pipelined(st, data, len);
      } else {
        for (uint64_t off = 0; off < len;) {
          uint64_t n = std::min<uint64_t>(step_bytes(st->m), len - off);
          feed_step(st, data + off, n);
          off += n;
        }
      }
    } catch (...) {
      st->failed = true;
      throw;
    }
    deliver(st, out, cap, n_out);
  });
}

ws_status ws_stream_end(ws_stream* st, ws_match64* out, uint64_t cap, uint64_t* n_out, ws_error_info* err) {
  return guarded(err, [&] {
    if (!st || !n_out || (cap && !out)) raise(WS_ERR_INVALID_ARGUMENT, "null argument");
    *n_out = 0;
    if (st->failed) raise(WS_ERR_DEVICE, "stream is unusable after an earlier error");
    check_cuda(cudaSetDevice(st->m->ctx->device), "cudaSetDevice");
    if (!st->ended) {
      st->ended = true;
      // every remaining regex start is decided now; literals were all reported
      if (st->m->rx.n_regex && st->win_len && st->frontier < st->seen) {
        try {
          scan_window(st, false, 0, st->seen);
        } catch (...) {
          st->failed = true;
          throw;
        }
      }
      st->frontier = st->seen;
      check_cuda(cudaEventRecord(st->s->busy, st->s->stream), "event");
    }
    deliver(st, out, cap, n_out);
  });
}

ws_status ws_scan_device64(ws_matcher* m, const uint8_t* d_data, uint64_t len, ws_match64* d_out, uint64_t cap,
                           uint64_t* d_count, void* stream, ws_error_info* err) {
  return guarded(err, [&] {
    if (!m || !d_count || (len && !d_data)) raise(WS_ERR_INVALID_ARGUMENT, "null argument");
    if (((uintptr_t)d_data & 15) != 0) raise(WS_ERR_INVALID_ARGUMENT, "device input must be 16-byte aligned");
    check_cuda(cudaSetDevice(m->ctx->device), "cudaSetDevice");
    ScratchLease s(m);
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    check_cuda(cudaStreamWaitEvent(cs, s->busy, 0), "wait");
    auto* total = reinterpret_cast<unsigned long long*>(d_count);
    check_cuda(cudaMemsetAsync(total, 0, 8, cs), "memset count");
    if (len == 0) {
      check_cuda(cudaEventRecord(s->busy, cs), "event");
      return;
    }
    enqueue_windows(m, *s, cs, d_data, len, step_bytes(m), d_out, cap, total, [](uint64_t) {});
  });
}

ws_status ws_scan_shard(ws_matcher* m, const uint8_t* d_data, uint64_t len, uint64_t base, uint64_t own_end,
                        uint64_t* d_cursor, ws_match64* d_out, uint64_t cap, uint64_t* d_count, void* stream,
                        ws_error_info* err) {
  return guarded(err, [&] {
    if (!m || !d_count || (len && !d_data) || (m->rx.n_regex && !d_cursor))
      raise(WS_ERR_INVALID_ARGUMENT, "null argument");
    if (((uintptr_t)d_data & 15) != 0) raise(WS_ERR_INVALID_ARGUMENT, "device input must be 16-byte aligned");
    if (own_end < base || own_end > base + len) raise(WS_ERR_INVALID_ARGUMENT, "own range outside the shard buffer");
    if (len > 0xFFFFFFFFull - 64)
      raise(WS_ERR_INPUT_TOO_LARGE, "shard buffer is too large for 32-bit offsets", 0, len, 0xFFFFFFFFull - 64);
    check_cuda(cudaSetDevice(m->ctx->device), "cudaSetDevice");
    ScratchLease s(m);
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    check_cuda(cudaStreamWaitEvent(cs, s->busy, 0), "wait");
    auto* total = reinterpret_cast<unsigned long long*>(d_count);
    check_cuda(cudaMemsetAsync(total, 0, 8, cs), "memset count");
    if (len == 0 || own_end == base) {
      check_cuda(cudaEventRecord(s->busy, cs), "event");
      return;
    }
    const uint64_t scap = std::max<uint64_t>(cap, 1);
    ensure(s->out, scap * sizeof(ws_match));
    ensure(s->aux, 256);
    auto* step_count = s->aux.as<unsigned long long>();
    ScanExtras x;
    x.literals = m->lit.n_literals != 0;
    x.lit_max_start = own_end - base;
    x.cursor = m->rx.n_regex ? reinterpret_cast<unsigned long long*>(d_cursor) : nullptr;
    x.base = base;
    x.frontier = own_end;
    uint32_t launches = enqueue_scan(m, *s, cs, d_data, len, s->out.as<ws_match>(), scap, step_count, x);
    widen_kernel<<<1, 1024, 0, cs>>>(s->out.as<ws_match>(), step_count, scap, base, d_out, cap, total);
    check_cuda(cudaGetLastError(), "widen_kernel");
    check_cuda(cudaEventRecord(s->busy, cs), "event");
    std::lock_guard<std::mutex> g(m->info_mu);
    m->info.last_launches = launches + 1;
  });
}

void ws_stream_destroy(ws_stream* st) {
  if (!st) return;
  cudaSetDevice(st->m->ctx->device);
  if (st->s) cudaStreamSynchronize(st->s->stream);
  delete st;
}

}  // extern "C"
