// Pattern IR: the host half of PatternSetBuilder::build that the GPU path needs,
// and the literal-scan plan derived from it.
#include <algorithm>
#include <cstring>

#include "ws_internal.h"

namespace ws {

void raise(ws_status s, const std::string& msg, uint64_t index, uint64_t count, uint64_t max) {
  Failure f;
  f.status = s;
  f.message = msg;
  f.index = index;
  f.count = count;
  f.max = max;
  throw WsError(std::move(f));
}

void check_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  cudaGetLastError();  // a failed call's error is not left behind for the caller's next check
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
    raise(WS_ERR_NO_DEVICE, std::string(what) + ": " + cudaGetErrorString(e));
  raise(WS_ERR_DEVICE, std::string(what) + ": " + cudaGetErrorString(e));
}

uint32_t fnv1a(const uint8_t* p, size_t len, size_t window) {
  // core/src/pattern/compiler.rs:343-350: bytes.iter().take(window.max(1))
  uint32_t h = FNV_BASIS;
  size_t n = std::min(len, std::max<size_t>(window, 1));
  for (size_t k = 0; k < n; ++k) { h ^= p[k]; h *= FNV_PRIME; }
  return h;
}

void build_prefilter_table(const std::vector<uint32_t>& offsets, const std::vector<uint32_t>& hashes,
                           uint32_t window, std::vector<uint32_t>& meta,
                           std::vector<uint32_t>& ranges, std::vector<uint32_t>& entries) {
  // core/src/literal_prefilter.rs:23-88: one partition per effective prefix
  // length min(len, window), each a power-of-two bucket table (2n rounded up)
  // with contiguous collision chains.
  const size_t n = hashes.size();
  std::vector<std::vector<uint32_t>> groups(window);  // literal indices
  for (size_t li = 0; li < n; ++li) {
    uint32_t len = offsets[2 * li + 1];
    uint32_t pl = std::max<uint32_t>(std::min(len, window), 1);
    groups[pl - 1].push_back((uint32_t)li);
  }
  meta.assign(4 * (size_t)window, 0);
  ranges.clear();
  entries.clear();
  entries.reserve(2 * n);
  for (uint32_t g = 0; g < window; ++g) {
    const auto& grp = groups[g];
    if (grp.empty()) continue;
    uint64_t buckets = 1;
    while (buckets < 2 * (uint64_t)grp.size()) buckets <<= 1;
    if (buckets > 0xFFFFFFFFull) raise(WS_ERR_PATTERN_SET_TOO_LARGE, "literal prefilter bucket count overflow");
    uint32_t first_bucket = (uint32_t)(ranges.size() / 2);
    // counting sort of the group's literals by bucket keeps insertion order in a chain
    std::vector<uint32_t> count(buckets + 1, 0);
    for (uint32_t li : grp) ++count[(hashes[li] & (buckets - 1)) + 1];
    for (uint64_t b = 0; b < buckets; ++b) count[b + 1] += count[b];
    std::vector<uint32_t> order(grp.size());
    std::vector<uint32_t> fill(count.begin(), count.end() - 1);
    for (uint32_t li : grp) order[fill[hashes[li] & (buckets - 1)]++] = li;
    uint32_t base = (uint32_t)(entries.size() / 2);
    for (uint64_t b = 0; b < buckets; ++b) {
      ranges.push_back(base + count[b]);
      ranges.push_back(count[b + 1] - count[b]);
    }
    for (uint32_t li : order) { entries.push_back(hashes[li]); entries.push_back(li); }
    meta[4 * g + 0] = first_bucket;
    meta[4 * g + 1] = (uint32_t)buckets - 1;
    meta[4 * g + 2] = (uint32_t)buckets;
    meta[4 * g + 3] = 0;
  }
}

DeviceBuffer::~DeviceBuffer() {
  if (ptr) cudaFree(ptr);
}

void DeviceBuffer::alloc(size_t n) {
  if (ptr) { cudaFree(ptr); ptr = nullptr; }
  bytes = n;
  if (n == 0) return;
  check_cuda(cudaMalloc(&ptr, n), "cudaMalloc");
}

void DeviceBuffer::upload(const void* src, size_t n) {
  alloc(n + 16);  // 16 spare bytes: vector loads of the tail stay inside the allocation
  check_cuda(cudaMemset(ptr, 0, n + 16), "cudaMemset");
  // a null source (an empty table given a minimum size) leaves zeros
  if (n && src) check_cuda(cudaMemcpy(ptr, src, n, cudaMemcpyHostToDevice), "cudaMemcpy H2D");
}

void plan_literals(const ws_pattern_tables& given, LiteralPlan& plan) {
  plan.n_literals = given.n_literals;
  if (given.n_literals == 0) return;
  // ASCII case-insensitive sets (PatternSetBuilder::case_insensitive,
  // core/src/pattern/compiler.rs:66-76, an Aho-Corasick automaton with
  // ascii_case_insensitive): every table below is planned on the literals
  // with A-Z folded to a-z, the prefilter table rebuilt on their FNV-1a
  // hashes, and the kernels fold the input the same way.
  ws_pattern_tables t = given;
  std::vector<uint8_t> folded;
  std::vector<uint32_t> foffsets, fhashes, fmeta, franges, fentries;
  plan.fold = given.case_insensitive != 0;
  if (plan.fold) {
    folded.assign(given.packed_bytes, given.packed_bytes + given.packed_len);
    for (uint8_t& c : folded) c = ascii_fold(c);
    foffsets.assign(given.offsets, given.offsets + 2 * (size_t)given.n_literals);
    for (uint32_t li = 0; li < given.n_literals; ++li)
      fhashes.push_back(fnv1a(folded.data() + foffsets[2 * li], foffsets[2 * li + 1], HASH_WINDOW));
    build_prefilter_table(foffsets, fhashes, HASH_WINDOW, fmeta, franges, fentries);
    t.packed_bytes = folded.data();
    t.hash_window_len = HASH_WINDOW;
    t.prefix_meta = fmeta.data();
    t.bucket_ranges = franges.data();
    t.n_buckets = (uint32_t)(franges.size() / 2);
    t.entries = fentries.data();
  }
  uint32_t min_long = UINT32_MAX;
  plan.max_len = 0;
  for (uint32_t li = 0; li < t.n_literals; ++li) {
    uint32_t len = t.offsets[2 * li + 1];
    plan.max_len = std::max(plan.max_len, len);
    if (len >= 4) { plan.has_long = 1; min_long = std::min(min_long, len); }
    else plan.has_short = 1;
  }
  // P grams at offsets 0..P-1 must fit inside every long literal: P + 3 <= len.
  plan.period = !plan.has_long ? 4 : (min_long >= 7) ? 4 : (min_long >= 5) ? 2 : 1;
  plan.table_bits = 18;
  const uint32_t P = plan.period, bits = plan.table_bits;
  plan.filter.assign((size_t)1 << (bits - 3), 0);
  plan.bloom.assign((size_t)1 << (18 - 5), 0);
  plan.short_bits.assign(65536 / 32, 0);
  plan.parts = 0;
  plan.lit_info.assign(4 * (size_t)t.n_literals, 0);
  plan.lit_bytes.clear();
  for (uint32_t li = 0; li < t.n_literals; ++li) {
    uint32_t off = t.offsets[2 * li], len = t.offsets[2 * li + 1];
    const uint8_t* lit = t.packed_bytes + off;
    while (plan.lit_bytes.size() % 4) plan.lit_bytes.push_back(0);
    plan.lit_info[4 * li + 0] = (uint32_t)plan.lit_bytes.size();
    plan.lit_info[4 * li + 1] = len;
    plan.lit_info[4 * li + 2] = t.literal_pattern_ids[li];
    plan.lit_bytes.insert(plan.lit_bytes.end(), lit, lit + len);
    plan.parts16 |= 1u << (std::min<uint32_t>(std::max<uint32_t>(len, 1), 16) - 1);
    {
      // Bloom bitmap of the first min(len, 8) bytes (the kernel's prefix_key)
      uint32_t pl = std::max<uint32_t>(std::min<uint32_t>(len, HASH_WINDOW), 1);
      uint8_t x[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      std::memcpy(x, lit, pl);
      uint32_t lo, hi;
      std::memcpy(&lo, x, 4);
      std::memcpy(&hi, x + 4, 4);
      uint32_t k = (lo * 0x9E3779B1u + hi * 0x85EBCA77u + pl * 0xC2B2AE3Du) >> (32 - 18);
      plan.bloom[k >> 5] |= 1u << (k & 31);
      plan.parts |= 1u << (pl - 1);
    }
    if (len >= 4) {
      for (uint32_t k = 0; k < P; ++k) {
        uint32_t gram;
        std::memcpy(&gram, lit + k, 4);
        uint32_t h = gram_hash(gram, bits);
        plan.filter[h >> 3] |= (1u << (P - 1 - k)) << ((h & 7) * 4);
      }
    } else {
      uint32_t b0 = lit[0];
      if (len == 1) {
        for (uint32_t b1 = 0; b1 < 256; ++b1) {
          uint32_t key = b0 | (b1 << 8);
          plan.short_bits[key >> 5] |= 1u << (key & 31);
        }
      } else {
        uint32_t key = b0 | ((uint32_t)lit[1] << 8);
        plan.short_bits[key >> 5] |= 1u << (key & 31);
      }
    }
  }
  while (plan.lit_bytes.size() % 16) plan.lit_bytes.push_back(0);
  // A low-entropy pattern set (a small alphabet whose 4-grams the literals
  // mostly cover, e.g. nucleotide k-mers) lets most input positions through
  // 4-byte grams: then switch to the longest gram every long literal holds at
  // all P phases, and add the 16-byte-prefix Bloom.
  if (plan.has_long && P == 4) {
    bool seen_byte[256] = {};
    std::vector<uint32_t> grams;
    for (uint32_t li = 0; li < t.n_literals; ++li) {
      const uint32_t len = t.offsets[2 * li + 1];
      const uint8_t* lit = t.packed_bytes + t.offsets[2 * li];
      for (uint32_t k = 0; k < len; ++k) seen_byte[lit[k]] = true;
      for (uint32_t k = 0; len >= 4 && k < P; ++k) {
        uint32_t g;
        std::memcpy(&g, lit + k, 4);
        grams.push_back(g);
      }
    }
    std::sort(grams.begin(), grams.end());
    const double distinct = (double)(std::unique(grams.begin(), grams.end()) - grams.begin());
    double alphabet = 0;
    for (bool b : seen_byte) alphabet += b ? 1.0 : 0.0;
    const double coverage = distinct / std::min(alphabet * alphabet * alphabet * alphabet, 4294967296.0);
    const uint32_t G = min_long >= 19 ? 16 : min_long >= 11 ? 8 : 4;
    if (coverage > 0.25 && G > 4) {
      plan.gram_len = G;
      std::fill(plan.filter.begin(), plan.filter.end(), 0u);
      plan.bloom2.assign((size_t)1 << (kBloom2Bits - 5), 0u);
      for (uint32_t li = 0; li < t.n_literals; ++li) {
        const uint32_t len = t.offsets[2 * li + 1];
        const uint8_t* lit = t.packed_bytes + t.offsets[2 * li];
        for (uint32_t k = 0; len >= 4 && k < P; ++k) {
          uint32_t g[4] = {0, 0, 0, 0};
          std::memcpy(g, lit + k, G);
          uint32_t h = long_gram_hash(g[0], g[1], g[2], g[3], G, bits);
          plan.filter[h >> 3] |= (1u << (P - 1 - k)) << ((h & 7) * 4);
        }
        // every literal (short ones too) is in the prefix Bloom
        uint32_t x[4] = {0, 0, 0, 0};
        const uint32_t pl = std::min<uint32_t>(len, 16);
        std::memcpy(x, lit, pl);
        uint32_t key = prefix16_key(x[0], x[1], x[2], x[3], pl);
        plan.bloom2[key >> 5] |= 1u << (key & 31);
      }
      plan.d_bloom2.upload(plan.bloom2.data(), plan.bloom2.size() * 4);
    }
  }
  // Stage 1b: when more than 0.5% (P = 4) or 0.1% (P = 2: nine grams per
  // 16 bytes, each passing one sends the warp block to compaction) of the
  // shared table's phase bits are set, a 2^kBigBits-byte table in L2 (the
  // same full 32-bit gram hashes, more of their bits) re-checks each passing
  // gram.
  if (plan.has_long && (P == 4 || P == 2)) {
    uint64_t set = 0;
    for (uint32_t w : plan.filter) set += (uint64_t)__builtin_popcount(w);
    if ((double)set / (double)((uint64_t)plan.filter.size() * 32) > (P == 4 ? 0.005 : 0.001)) {
      const uint32_t G = plan.gram_len;
      plan.big.assign((size_t)1 << kBigBits, 0);
      std::vector<uint32_t> lean2(G > 4 ? (size_t)1 << (kLeanBits - 5) : 0, 0u);
      for (uint32_t li = 0; li < t.n_literals; ++li) {
        const uint32_t len = t.offsets[2 * li + 1];
        const uint8_t* lit = t.packed_bytes + t.offsets[2 * li];
        if (len < 4) continue;
        for (uint32_t k = 0; k < P; ++k) {
          uint32_t g[4] = {0, 0, 0, 0};
          std::memcpy(g, lit + k, G);
          const uint32_t hf = G == 4 ? g[0] * 0x9E3779B1u
                              : G == 8 ? mix_words(g[0], g[1], 0, 0, 8)
                                       : mix_words(g[0], g[1], g[2], g[3], 16);
          const uint32_t h = hf >> (32 - kBigBits);
          plan.big[h] |= (uint8_t)(1u << (P - 1 - k));
          if (G > 4) lean2[lean2_word(hf)] |= lean2_mask(hf);
        }
      }
      plan.d_big.upload(plan.big.data(), plan.big.size());
      plan.lean_bits.assign((size_t)1 << (kLeanBits - 3), 0);
      if (G > 4) {
        std::memcpy(plan.lean_bits.data(), lean2.data(), plan.lean_bits.size());
      } else {
        for (size_t h = 0; h < plan.big.size(); ++h)
          if (plan.big[h]) {
            const size_t b = h >> (kBigBits - kLeanBits);
            plan.lean_bits[b >> 3] |= (uint8_t)(1u << (b & 7));
          }
      }
      plan.d_lean_bits.upload(plan.lean_bits.data(), plan.lean_bits.size());
      plan.has_big = true;
      std::vector<uint8_t>().swap(plan.big);
    }
  }
  plan.n_buckets = t.n_buckets;
  plan.d_filter.upload(plan.filter.data(), plan.filter.size() * 4);
  plan.d_bloom.upload(plan.bloom.data(), plan.bloom.size() * 4);
  plan.d_short.upload(plan.short_bits.data(), plan.short_bits.size() * 4);
  plan.d_info.upload(plan.lit_info.data(), plan.lit_info.size() * 4);
  plan.d_bytes.upload(plan.lit_bytes.data(), plan.lit_bytes.size());
  plan.d_meta.upload(t.prefix_meta, 4 * (size_t)t.hash_window_len * 4);
  plan.d_ranges.upload(t.bucket_ranges, 2 * (size_t)t.n_buckets * 4);
  plan.d_entries.upload(t.entries, 2 * (size_t)t.n_literals * 4);
}

}  // namespace ws

using namespace ws;

namespace {

void fill_err(ws_error_info* err, const Failure& f) {
  if (!err) return;
  err->index = f.index;
  err->count = f.count;
  err->max = f.max;
  std::snprintf(err->message, sizeof(err->message), "%s", f.message.c_str());
}

}  // namespace

extern "C" ws_status ws_ir_build(const ws_pattern_spec* patterns, uint64_t n, int case_insensitive,
                                 ws_ir** out, ws_error_info* err) {
  if (err) std::memset(err, 0, sizeof(*err));
  if (!out || (n && !patterns)) {
    if (err) std::snprintf(err->message, sizeof(err->message), "null argument");
    return WS_ERR_INVALID_ARGUMENT;
  }
  *out = nullptr;
  try {
    // core/src/pattern/compiler.rs:97-340
    if (n == 0) raise(WS_ERR_EMPTY_PATTERN_SET, "pattern set is empty. Fix: add at least one literal pattern before building.");
    if (n > 0xFFFFFFFFull) raise(WS_ERR_PATTERN_SET_TOO_LARGE, "too many patterns", 0, n, 0xFFFFFFFFull);
    auto ir = std::make_unique<ws_ir>();
    IrData& d = ir->d;
    d.n_patterns = (uint32_t)n;
    d.case_insensitive = case_insensitive != 0;
    auto add_literal = [&](uint64_t i, const uint8_t* b, uint64_t len) {
      if (len > 0xFFFFFFFFull) raise(WS_ERR_PATTERN_TOO_LARGE, "pattern too large", i, len, 0xFFFFFFFFull);
      if (d.packed_bytes.size() + len > 0xFFFFFFFFull)
        raise(WS_ERR_PATTERN_SET_TOO_LARGE, "packed literal bytes exceed u32", 0, d.packed_bytes.size(), 0xFFFFFFFFull);
      d.offsets.push_back((uint32_t)d.packed_bytes.size());
      d.offsets.push_back((uint32_t)len);
      d.literal_hashes.push_back(fnv1a(b, len, HASH_WINDOW));
      d.literal_pattern_ids.push_back((uint32_t)i);
      d.packed_bytes.insert(d.packed_bytes.end(), b, b + len);
    };
    for (uint64_t i = 0; i < n; ++i) {
      const ws_pattern_spec& p = patterns[i];
      if (p.len == 0) raise(WS_ERR_EMPTY_PATTERN, "pattern " + std::to_string(i) + " is empty. Fix: provide a non-empty byte sequence for every pattern.", i);
      if (!p.bytes) raise(WS_ERR_INVALID_ARGUMENT, "null pattern bytes", i);
      if (p.kind == WS_PATTERN_LITERAL) {
        add_literal(i, p.bytes, p.len);
      } else if (p.kind == WS_PATTERN_REGEX) {
        std::string src((const char*)p.bytes, (size_t)p.len);
        ReTree tree;
        try {
          tree = parse_regex(src);
        } catch (const CompileError& e) {
          raise(WS_ERR_COMPILE, "invalid regex at index " + std::to_string(i) + ": " + e.what(), i);
        }
        if (tree_pathological(tree)) raise(WS_ERR_PATHOLOGICAL, "regex pattern " + std::to_string(i) + " contains nested repetitions (pathological)", i);
        std::vector<uint8_t> lit;
        if (tree_literal(tree, &lit)) {  // compiler.rs:181-212: literal demotion
          add_literal(i, lit.data(), lit.size());
          continue;
        }
        d.regex_sources.push_back(src);
        d.regex_pattern_ids.push_back((uint32_t)i);
      } else {
        raise(WS_ERR_INVALID_ARGUMENT, "unknown pattern kind", i);
      }
    }
    build_prefilter_table(d.offsets, d.literal_hashes, HASH_WINDOW, d.prefix_meta, d.bucket_ranges, d.entries);
    for (auto& s : d.regex_sources) d.regex_ptrs.push_back(s.c_str());
    *out = ir.release();
    return WS_OK;
  } catch (const WsError& e) {
    fill_err(err, e.f);
    return e.f.status;
  } catch (const std::exception& e) {
    if (err) std::snprintf(err->message, sizeof(err->message), "%s", e.what());
    return WS_ERR_COMPILE;
  }
}

extern "C" void ws_ir_destroy(ws_ir* ir) { delete ir; }

extern "C" ws_status ws_ir_tables(const ws_ir* ir, ws_pattern_tables* t) {
  if (!ir || !t) return WS_ERR_INVALID_ARGUMENT;
  const IrData& d = ir->d;
  std::memset(t, 0, sizeof(*t));
  t->packed_bytes = d.packed_bytes.data();
  t->packed_len = d.packed_bytes.size();
  t->offsets = d.offsets.data();
  t->literal_pattern_ids = d.literal_pattern_ids.data();
  t->n_literals = (uint32_t)d.literal_pattern_ids.size();
  t->hash_window_len = HASH_WINDOW;
  t->prefix_meta = d.prefix_meta.data();
  t->bucket_ranges = d.bucket_ranges.data();
  t->n_buckets = (uint32_t)(d.bucket_ranges.size() / 2);
  t->entries = d.entries.data();
  t->regex_sources = d.regex_ptrs.data();
  t->regex_pattern_ids = d.regex_pattern_ids.data();
  t->n_regex = (uint32_t)d.regex_pattern_ids.size();
  t->n_patterns = d.n_patterns;
  t->case_insensitive = d.case_insensitive ? 1 : 0;
  return WS_OK;
}
