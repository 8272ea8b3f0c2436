// Batch scan of many items in one launch sequence.
//
// Replaces scan_batch / scan_batch_gpu / scan_batch_auto
// (core/src/batch.rs:252-363).  The reference coalesces up to 4,096 items or
// 256 MiB into one buffer (coalesce, batch.rs:65-98), runs a full GpuMatcher
// round trip per batch, and afterwards drops matches that cross item
// boundaries (decoalesce, batch.rs:106-167).  Here the items are gathered
// into one device buffer per launch sequence (1 GiB by default) together with
// a table of item end offsets, and the kernels are item-aware:
//   - literal verify rejects an occurrence that runs past its item's end;
//   - the regex reverse walk stops at the start of the item holding the match
//     end, the leftmost-first end walk and the plain walk stop at the end of
//     the item holding the start, so K holds only in-item candidates and each
//     item gets its own find_iter chain (the chain cursor never crosses an
//     item because every match ends inside its item);
// which makes the result the per-item scan of scan_batch_cpu
// (batch.rs:170-195): L + R inside each item, no cross-item matches.  A tag
// kernel converts coalesced offsets to (source_id, item-relative offsets);
// the host sorts by (source_id, start, pattern_id, end) as batch.rs:157-163.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <numeric>

#include "ws_matcher.h"

using namespace ws;

namespace {

// Every match of a coalesced launch, tagged with its item's id and shifted to
// item-relative offsets.
__global__ void tag_kernel(const ws_match* in, const unsigned long long* count, uint64_t cap, const uint32_t* ends,
                           const uint64_t* ids, uint32_t n_items, ws_tagged_match* out) {
  unsigned long long n = *count;
  if (n > cap) n = cap;
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
    ws_match mm = in[k];
    uint32_t lo = 0, hi = n_items;  // first item whose end is above the start
    while (lo < hi) {
      uint32_t mid = (lo + hi) >> 1;
      if (ends[mid] > mm.start) hi = mid; else lo = mid + 1;
    }
    const uint32_t base = lo ? ends[lo - 1] : 0;
    ws_tagged_match t;
    t.source_id = ids[lo];
    t.pattern_id = mm.pattern_id;
    t.start = mm.start - base;
    t.end = mm.end - base;
    t.reserved = 0;
    out[k] = t;
  }
}

// Gathers host byte runs into one contiguous device range through two pinned
// staging pieces (the host copy of one piece overlaps the DMA of the other);
// large pinned runs are copied directly.
class Gather {
 public:
  Gather(Scratch& s, uint8_t* d_dst, cudaStream_t st) : s_(s), d_dst_(d_dst), st_(st) {}

  void push(const uint8_t* src, uint64_t n) {
    if (n >= kDirect && is_pinned(src)) {
      flush();
      check_cuda(cudaMemcpyAsync(d_dst_ + off_, src, n, cudaMemcpyHostToDevice, st_), "H2D item");
      off_ += n;
      return;
    }
    while (n) {
      if (!pin_) {
        pin_ = staging_slot(s_, slot_, kPiece);
        piece_off_ = off_;
      }
      size_t k = (size_t)std::min<uint64_t>(n, kPiece - fill_);
      std::memcpy(pin_ + fill_, src, k);
      fill_ += k;
      off_ += k;
      src += k;
      n -= k;
      if (fill_ == kPiece) flush();
    }
  }

  void flush() {
    if (!pin_) return;
    if (fill_) {
      check_cuda(cudaMemcpyAsync(d_dst_ + piece_off_, pin_, fill_, cudaMemcpyHostToDevice, st_),
                 "H2D batch piece");
      staging_issued(s_, slot_, st_);
      slot_ ^= 1;
    }
    fill_ = 0;
    pin_ = nullptr;
  }

 private:
  static constexpr size_t kPiece = 8u << 20;
  static constexpr uint64_t kDirect = 1u << 20;
  Scratch& s_;
  uint8_t* d_dst_;
  cudaStream_t st_;
  uint8_t* pin_ = nullptr;  // current slot being filled
  int slot_ = 0;
  size_t fill_ = 0;
  uint64_t off_ = 0, piece_off_ = 0;
};

}  // namespace

extern "C" ws_status ws_scan_batch_device(ws_matcher* m, const uint8_t* d_data, uint64_t len,
                                          const uint32_t* d_item_end, const uint64_t* d_ids, uint64_t n_items,
                                          ws_tagged_match* d_out, uint64_t cap, uint64_t* d_count, void* stream,
                                          ws_error_info* err) {
  return guarded(err, [&] {
    if (!m || !d_count || (len && (!d_data || !d_item_end || !d_ids))) raise(WS_ERR_INVALID_ARGUMENT, "null argument");
    if (((uintptr_t)d_data & 15) != 0) raise(WS_ERR_INVALID_ARGUMENT, "device input must be 16-byte aligned");
    if (len > 0xFFFFFFFFull - 64)
      raise(WS_ERR_INPUT_TOO_LARGE, "coalesced batch is too large for 32-bit offsets", 0, len, 0xFFFFFFFFull - 64);
    if (n_items > 0xFFFFFFFFull) raise(WS_ERR_INVALID_ARGUMENT, "too many items");
    check_cuda(cudaSetDevice(m->ctx->device), "cudaSetDevice");
    ScratchLease s(m);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    check_cuda(cudaStreamWaitEvent(st, s->busy, 0), "wait");
    auto* d_counter = reinterpret_cast<unsigned long long*>(d_count);
    if (len == 0 || n_items == 0) {
      check_cuda(cudaMemsetAsync(d_counter, 0, 8, st), "memset");
      check_cuda(cudaEventRecord(s->busy, st), "event");
      return;
    }
    const uint64_t dcap = std::max<uint64_t>(cap, 1);
    ensure(s->out, dcap * sizeof(ws_match));
    auto body = [&]() -> uint32_t {
      ScanExtras x;
      x.item_end = d_item_end;
      x.n_items = (uint32_t)n_items;
      const uint32_t n = enqueue_scan(m, *s, st, d_data, len, s->out.as<ws_match>(), dcap, d_counter, x);
      tag_kernel<<<m->ctx->sm_count * 4, 256, 0, st>>>(s->out.as<ws_match>(), d_counter, std::min(dcap, cap),
                                                        d_item_end, d_ids, (uint32_t)n_items, d_out);
      check_cuda(cudaGetLastError(), "tag_kernel");
      return n + 1;
    };
    // The launch sequence of a call is replayed from a CUDA graph when the
    // previous calls on this scratch had the same arguments and plan: the
    // first runs eagerly (it sizes every buffer), the second is captured.
    BatchGraphKey key;
    key.data = d_data;
    key.len = len;
    key.item_end = d_item_end;
    key.ids = d_ids;
    key.n_items = n_items;
    key.out = d_out;
    key.cap = cap;
    key.count = d_count;
    key.stream = stream;
    key.plan_gen = m->plan_gen.load();
    if (m->need_host) {
      key.need[0] = m->need_host[0];
      key.need[1] = m->need_host[1];
    }
    key.profile = m->profile ? 1 : 0;
    BatchGraph& bg = s->batch_graph;
    if (std::memcmp(&bg.key, &key, sizeof(key)) != 0) {
      bg.reset();
      bg.key = key;
    }
    uint32_t launches = 0;
    bool replayed = false;
    if (bg.exec) {
      check_cuda(cudaGraphLaunch(bg.exec, st), "cudaGraphLaunch(batch)");
      launches = bg.launches;
      replayed = true;
    } else if (bg.seen >= 1 && !bg.broken && !m->profile && st != nullptr && st != cudaStreamLegacy &&
               cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed) == cudaSuccess) {
      // (the legacy default stream cannot be captured, and profiled scans time
      // each phase with events: their calls stay eager)
      cudaGraph_t graph = nullptr;
      try {
        launches = body();
      } catch (...) {
        cudaStreamEndCapture(st, &graph);
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        bg.broken = true;
        throw;
      }
      const cudaError_t ce = cudaStreamEndCapture(st, &graph);
      const cudaError_t ie = ce == cudaSuccess ? cudaGraphInstantiate(&bg.exec, graph, 0) : ce;
      if (graph) cudaGraphDestroy(graph);
      if (ie != cudaSuccess) {  // no graph: run this call eagerly and stay eager for this key
        cudaGetLastError();
        bg.exec = nullptr;
        bg.broken = true;
        launches = body();
      } else {
        bg.launches = launches;
        check_cuda(cudaGraphLaunch(bg.exec, st), "cudaGraphLaunch(batch)");
        replayed = true;
      }
    } else {
      cudaGetLastError();  // a refused capture leaves its error behind
      launches = body();
      bg.seen++;
    }
    check_cuda(cudaEventRecord(s->busy, st), "event");
    std::lock_guard<std::mutex> g(m->info_mu);
    m->info.last_launches = launches;
    m->info.last_graph_replay = replayed ? 1u : 0u;
  });
}

extern "C" ws_status ws_scan_batch(ws_matcher* m, const ws_item* items, uint64_t n_items, ws_tagged_match* out,
                                   uint64_t cap, uint64_t* n_out, ws_error_info* err) {
  return guarded(err, [&] {
    if (!m || !n_out || (n_items && !items) || (cap && !out)) raise(WS_ERR_INVALID_ARGUMENT, "null argument");
    *n_out = 0;
    // batch.rs:65-98: every item must be addressable with 32-bit offsets
    std::vector<uint64_t> order;
    order.reserve(n_items);
    for (uint64_t i = 0; i < n_items; ++i) {
      if (items[i].len > 0xFFFFFFFFull)
        raise(WS_ERR_INPUT_TOO_LARGE, "batch item is too large for 32-bit match offsets", i, items[i].len,
              0xFFFFFFFFull);
      if (items[i].len && !items[i].data) raise(WS_ERR_INVALID_ARGUMENT, "batch item with null data", i);
      if (items[i].len) order.push_back(i);  // an empty item has no matches
    }
    if (order.empty()) return;
    // items in source-id order (stable), packed greedily into launch sequences
    std::stable_sort(order.begin(), order.end(), [&](uint64_t a, uint64_t b) { return items[a].id < items[b].id; });
    const uint64_t budget = std::min<uint64_t>((uint64_t)(m->cfg.batch_mib ? m->cfg.batch_mib : 1024) << 20,
                                               0xFFFFFFFFull);
    std::vector<std::pair<size_t, size_t>> groups;  // [first, last) in order
    {
      size_t a = 0;
      uint64_t bytes = 0;
      for (size_t k = 0; k < order.size(); ++k) {
        uint64_t len = items[order[k]].len;
        if (k > a && bytes + len > budget) {
          groups.emplace_back(a, k);
          a = k;
          bytes = 0;
        }
        bytes += len;
      }
      groups.emplace_back(a, order.size());
    }

    check_cuda(cudaSetDevice(m->ctx->device), "cudaSetDevice");
    ScratchLease s(m);
    check_cuda(cudaStreamWaitEvent(s->stream, s->busy, 0), "wait");
    const uint64_t dcap = device_capacity(m);
    ensure(s->out, dcap * sizeof(ws_match));
    auto* d_counter = s->counters.as<unsigned long long>();
    uint64_t total = 0;
    if (!s->copy) check_cuda(cudaStreamCreateWithFlags(&s->copy, cudaStreamNonBlocking), "cudaStreamCreate");
    check_cuda(cudaStreamWaitEvent(s->copy, s->busy, 0), "wait");
    // launch group k is gathered into input buffer k & 1 on the copy stream,
    // group k + 1 while group k is scanned
    struct Group {
      std::vector<uint32_t> ends;
      std::vector<uint64_t> ids;
      uint64_t bytes = 0;
    } grp[2];
    DeviceBuffer* inbuf[2] = {&s->input, &s->input_alt};
    auto gather = [&](size_t gi) {
      const auto& gr = groups[gi];
      Group& G = grp[gi & 1];
      const size_t ni = gr.second - gr.first;
      G.ends.resize(ni);
      G.ids.resize(ni);
      G.bytes = 0;
      for (size_t k = 0; k < ni; ++k) {
        const ws_item& it = items[order[gr.first + k]];
        G.bytes += it.len;
        G.ends[k] = (uint32_t)G.bytes;
        G.ids[k] = it.id;
      }
      DeviceBuffer& in = *inbuf[gi & 1];  // its last scan (group gi - 2) has finished
      ensure(in, G.bytes + 64);
      // items adjacent in host memory (slices of one arena) move as one run
      Gather g(*s, in.as<uint8_t>(), s->copy);
      const uint8_t* run = nullptr;
      uint64_t run_len = 0;
      for (size_t k = 0; k < ni; ++k) {
        const ws_item& it = items[order[gr.first + k]];
        if (run && it.data == run + run_len) {
          run_len += it.len;
          continue;
        }
        if (run) g.push(run, run_len);
        run = it.data;
        run_len = it.len;
      }
      if (run) g.push(run, run_len);
      g.flush();
      check_cuda(cudaMemsetAsync(in.as<uint8_t>() + G.bytes, 0, 64, s->copy), "memset pad");
      check_cuda(cudaEventRecord(s->ev[gi & 1], s->copy), "event");
    };
    try {
      gather(0);
      for (size_t gi = 0; gi < groups.size(); ++gi) {
        const Group& G = grp[gi & 1];
        const size_t ni = G.ends.size();
        // device layout of aux: [item ends u32][item ids u64][tagged matches]
        const size_t ends_off = 0, ids_off = (ni * 4 + 255) & ~(size_t)255,
                     tag_off = ids_off + ((ni * 8 + 255) & ~(size_t)255);
        ensure(s->aux, tag_off + dcap * sizeof(ws_tagged_match));
        uint8_t* aux = s->aux.as<uint8_t>();
        stage_copy(*s, aux + ends_off, reinterpret_cast<const uint8_t*>(G.ends.data()), ni * 4);
        stage_copy(*s, aux + ids_off, reinterpret_cast<const uint8_t*>(G.ids.data()), ni * 8);
        check_cuda(cudaStreamWaitEvent(s->stream, s->ev[gi & 1], 0), "wait group");
        ScanExtras x;
        x.item_end = reinterpret_cast<const uint32_t*>(aux + ends_off);
        x.n_items = (uint32_t)ni;
        auto* d_tag = reinterpret_cast<ws_tagged_match*>(aux + tag_off);
        unsigned long long count = 0;
        for (int attempt = 0;; ++attempt) {
          enqueue_scan(m, *s, s->stream, inbuf[gi & 1]->as<uint8_t>(), G.bytes, s->out.as<ws_match>(), dcap,
                       d_counter, x);
          tag_kernel<<<m->ctx->sm_count * 4, 256, 0, s->stream>>>(s->out.as<ws_match>(), d_counter, dcap,
                                                                    reinterpret_cast<const uint32_t*>(aux + ends_off),
                                                                    reinterpret_cast<const uint64_t*>(aux + ids_off),
                                                                    (uint32_t)ni, d_tag);
          check_cuda(cudaGetLastError(), "tag_kernel");
          if (attempt == 0 && gi + 1 < groups.size()) gather(gi + 1);
          check_cuda(cudaMemcpyAsync(&count, d_counter, sizeof(count), cudaMemcpyDeviceToHost, s->stream),
                     "D2H count");
          check_cuda(cudaStreamSynchronize(s->stream), "batch scan");
          if (!repeat_scan(m, count, attempt)) break;  // else the regex candidates overflowed: scan again
        }
        if (count > dcap) raise(WS_ERR_OVERFLOW, "too many matches in one batch launch", 0, count, dcap);
        if (total + count <= cap && count) {
          const ws_tagged_match* res = d_tag;
          if (count > 1 && count <= kMaxDeviceSorted) {  // this group's matches in their final order
            ensure(s->sorted, count * sizeof(ws_tagged_match));
            sort_tagged_device(*s, d_tag, s->sorted.as<ws_tagged_match>(), count, s->stream);
            res = s->sorted.as<ws_tagged_match>();
          }
          check_cuda(cudaMemcpyAsync(out + total, res, count * sizeof(ws_tagged_match), cudaMemcpyDeviceToHost,
                                     s->stream), "D2H tagged matches");
          check_cuda(cudaStreamSynchronize(s->stream), "D2H sync");
        }
        total += count;
      }
    } catch (...) {
      cudaStreamSynchronize(s->copy);  // no copy may still read the caller's items
      throw;
    }
    check_cuda(cudaEventRecord(s->busy, s->stream), "event");
    *n_out = total;
    if (total > cap) raise(WS_ERR_OVERFLOW, "too many matches for the output buffer", 0, total, cap);
    // each launch group came back ordered; groups are in source-id order, so
    // only an id whose items span two groups leaves work for the host
    auto less = [](const ws_tagged_match& a, const ws_tagged_match& b) {
      if (a.source_id != b.source_id) return a.source_id < b.source_id;
      if (a.start != b.start) return a.start < b.start;
      if (a.pattern_id != b.pattern_id) return a.pattern_id < b.pattern_id;
      return a.end < b.end;
    };
    if (!std::is_sorted(out, out + total, less)) std::sort(out, out + total, less);
  });
}
