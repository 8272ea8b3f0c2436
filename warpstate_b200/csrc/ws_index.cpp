// CompiledPatternIndex: the reference's on-disk pattern index, loaded into the
// tables the device plan is built from, and written back in the same format.
//
// Format (core/src/compiled_index/builder.rs:8-64, read by
// core/src/compiled_index/mod.rs:96-260), little-endian:
//   magic "WPSIDX01", u32 version (1..3), u32 case_insensitive,
//   u32 pattern count, u32 literal count, u32 regex-DFA count,
//   u32 hash_window_len,
//   packed literal bytes (u32 length + bytes),
//   offsets (u32 count + count x (start, len)),
//   names (u32 count + per name u32 length or 0xFFFFFFFF for none, + UTF-8),
//   version >= 2: regex sources (u32 count + per regex u32 pattern id,
//                 u32 length + UTF-8),
//   literal pattern ids (u32 count + u32 each),
//   LiteralPrefilterTable: prefix_meta (u32 count + 4 u32 each),
//                          bucket ranges (u32 count + 2 u32 each),
//                          entries (u32 count + 2 u32 each),
//   per regex DFA: transition table, match-list pointers, match lists,
//                  pattern lengths (u32 vectors), u32 start state, u32 class
//                  count, u32 eoi class, 256 u32 byte classes, serialized
//                  regex-automata DFA (u32 length + bytes), original ids
//                  (u32 vector),
//   version 3: CRC-32 (IEEE) of everything before it.
//
// Loading keeps the reference's literal tables as they are (packed bytes,
// offsets, ids and the prefilter table go to the device unchanged, after
// bounds checks that make every probe the kernels derive from them stay
// inside the tables) and takes the regexes from their sources: the
// serialized DFAs are regex-automata's own per-regex automata, which the
// merged group DFAs of the GPU walk do not use, so they are checked for shape
// and skipped.  Writing produces version 3 with the regex sources and no
// serialized DFAs (only regex-automata can produce those): the reference's
// CompiledPatternIndex::load accepts such a file and to_pattern_set()
// rebuilds every pattern from it.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>

#include "ws_internal.h"

using namespace ws;

namespace {

constexpr uint8_t kMagic[8] = {'W', 'P', 'S', 'I', 'D', 'X', '0', '1'};
constexpr uint32_t kIndexVersion = 3;
constexpr uint64_t kMaxIndexBytes = 512ull << 20;  // mod.rs:19

// CRC-32 with the reflected IEEE 802.3 polynomial 0xEDB88320, initial value
// and final xor all ones (the checksum builder.rs:67-81 appends), a byte at a
// time through a 256-entry table.
struct CrcTable {
  uint32_t t[256];
  CrcTable() {
    for (uint32_t i = 0; i < 256; ++i) {
      uint32_t c = i;
      for (int k = 0; k < 8; ++k) c = (c & 1) ? (c >> 1) ^ 0xEDB88320u : c >> 1;
      t[i] = c;
    }
  }
};

uint32_t crc32_ieee(const uint8_t* p, size_t n) {
  static const CrcTable table;  // built once, thread-safe
  uint32_t crc = 0xFFFFFFFFu;
  for (size_t i = 0; i < n; ++i) crc = table.t[(crc ^ p[i]) & 0xFF] ^ (crc >> 8);
  return ~crc;
}

[[noreturn]] void bad(const std::string& what) {
  raise(WS_ERR_COMPILE, "compiled index " + what + ". Fix: rebuild the index file.");
}

// Bounds-checked little-endian reader (the Cursor of mod.rs:439-700).
struct Reader {
  const uint8_t* d;
  size_t n, off = 0;
  Reader(const uint8_t* data, size_t len) : d(data), n(len) {}
  size_t remaining() const { return n - off; }
  const uint8_t* take(size_t len) {
    if (len > remaining()) bad("is truncated");
    const uint8_t* p = d + off;
    off += len;
    return p;
  }
  uint32_t u32() {
    const uint8_t* p = take(4);
    return (uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24;
  }
  // A count of elements of `size` bytes each that must fit in what is left.
  uint32_t count(size_t size, const char* what) {
    const uint32_t c = u32();
    if ((uint64_t)c * size > remaining()) bad(std::string(what) + " declares more bytes than remain");
    return c;
  }
  std::vector<uint32_t> u32s(uint32_t c) {
    std::vector<uint32_t> v(c);
    for (auto& x : v) x = u32();
    return v;
  }
  std::vector<uint32_t> u32vec(const char* what) { return u32s(count(4, what)); }
  std::string str(uint32_t len) {
    const uint8_t* p = take(len);
    return std::string(reinterpret_cast<const char*>(p), len);
  }
};

// Strict UTF-8 check (names and regex sources are Rust Strings).
bool valid_utf8(const std::string& s) {
  const auto* p = reinterpret_cast<const uint8_t*>(s.data());
  const size_t n = s.size();
  size_t i = 0;
  while (i < n) {
    const uint8_t c = p[i];
    if (c < 0x80) {
      ++i;
      continue;
    }
    size_t k;
    uint32_t cp;
    if ((c & 0xE0) == 0xC0) { k = 1; cp = c & 0x1F; }
    else if ((c & 0xF0) == 0xE0) { k = 2; cp = c & 0x0F; }
    else if ((c & 0xF8) == 0xF0) { k = 3; cp = c & 0x07; }
    else return false;
    if (i + k >= n) return false;
    for (size_t j = 1; j <= k; ++j) {
      if ((p[i + j] & 0xC0) != 0x80) return false;
      cp = (cp << 6) | (p[i + j] & 0x3F);
    }
    const uint32_t min_cp = k == 1 ? 0x80 : k == 2 ? 0x800 : 0x10000;
    if (cp < min_cp || cp > 0x10FFFF || (cp >= 0xD800 && cp <= 0xDFFF)) return false;
    i += k + 1;
  }
  return true;
}

void put32(std::vector<uint8_t>& b, uint32_t v) {
  for (int k = 0; k < 4; ++k) b.push_back((uint8_t)(v >> (8 * k)));
}

uint32_t checked_u32(uint64_t v, const char* what) {
  if (v > 0xFFFFFFFFull)
    raise(WS_ERR_COMPILE, std::string(what) + " exceeds the on-disk 32-bit format. Fix: split the pattern set "
                                              "into smaller indexes.");
  return (uint32_t)v;
}

void fill_err_info(ws_error_info* err, const Failure& f) {
  if (!err) return;
  err->index = f.index;
  err->count = f.count;
  err->max = f.max;
  std::snprintf(err->message, sizeof(err->message), "%s", f.message.c_str());
}

template <class F>
ws_status run_guarded(ws_error_info* err, F&& fn) {
  if (err) std::memset(err, 0, sizeof(*err));
  try {
    fn();
    return WS_OK;
  } catch (const WsError& e) {
    fill_err_info(err, e.f);
    return e.f.status;
  } catch (const std::bad_alloc&) {
    if (err) std::snprintf(err->message, sizeof(err->message), "host allocation failed");
    return WS_ERR_DEVICE;
  } catch (const std::exception& e) {
    if (err) std::snprintf(err->message, sizeof(err->message), "%s", e.what());
    return WS_ERR_COMPILE;
  }
}

}  // namespace

extern "C" ws_status ws_index_load(const uint8_t* bytes, uint64_t len, ws_ir** out, ws_error_info* err) {
  return run_guarded(err, [&] {
    if (!out || (len && !bytes)) raise(WS_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (len > kMaxIndexBytes) raise(WS_ERR_INPUT_TOO_LARGE, "compiled index is too large", 0, len, kMaxIndexBytes);
    // version 3 ends with the CRC-32 of everything before it (mod.rs:99-139)
    size_t end = (size_t)len;
    if (len >= 16) {
      const uint32_t version = (uint32_t)bytes[8] | (uint32_t)bytes[9] << 8 | (uint32_t)bytes[10] << 16 |
                               (uint32_t)bytes[11] << 24;
      if (version == 3) {
        end = (size_t)len - 4;
        const uint32_t stored = (uint32_t)bytes[end] | (uint32_t)bytes[end + 1] << 8 |
                                (uint32_t)bytes[end + 2] << 16 | (uint32_t)bytes[end + 3] << 24;
        const uint32_t computed = crc32_ieee(bytes, end);
        if (stored != computed) {
          char buf[96];
          std::snprintf(buf, sizeof(buf), "integrity check failed (CRC mismatch: stored=0x%08X, computed=0x%08X)",
                        stored, computed);
          bad(buf);
        }
      }
    }
    Reader r(bytes, end);
    if (std::memcmp(r.take(8), kMagic, 8) != 0) bad("header is invalid");
    const uint32_t version = r.u32();
    if (version > kIndexVersion) bad("version " + std::to_string(version) + " is unsupported");
    if (version == 0) bad("version is invalid");
    auto ir = std::make_unique<ws_ir>();
    IrData& d = ir->d;
    d.case_insensitive = r.u32() != 0;
    const uint32_t n_patterns = r.u32();
    const uint32_t n_literals = r.u32();
    const uint32_t n_dfas = r.u32();
    const uint32_t window = r.u32();
    const uint32_t packed_len = r.count(1, "packed byte length");
    const uint8_t* packed = r.take(packed_len);
    d.packed_bytes.assign(packed, packed + packed_len);
    const uint32_t n_offsets = r.count(8, "literal offsets");
    if (n_offsets != n_literals) bad("literal metadata is inconsistent");
    d.offsets = r.u32s(2 * n_offsets);
    // names (mod.rs:530-551)
    const uint32_t n_names = r.count(4, "name table");
    if (n_names != n_patterns) bad("name metadata is inconsistent");
    d.names.resize(n_names);
    d.named.assign(n_names, 0);
    for (uint32_t i = 0; i < n_names; ++i) {
      const uint32_t nl = r.u32();
      if (nl == 0xFFFFFFFFu) continue;
      d.names[i] = r.str(nl);
      if (!valid_utf8(d.names[i])) bad("name is not valid UTF-8");
      d.named[i] = 1;
    }
    // regex sources (mod.rs:553-588), version 2 and later
    std::vector<uint8_t> seen_regex(n_patterns, 0);
    bool has_sources = false;
    if (version >= 2) {
      has_sources = true;
      const uint32_t n_rx = r.count(8, "regex pattern table");
      for (uint32_t k = 0; k < n_rx; ++k) {
        const uint32_t id = r.u32();
        if (id >= n_patterns) bad("regex pattern ID is out of bounds");
        if (seen_regex[id]) bad("contains duplicate regex pattern IDs");
        seen_regex[id] = 1;
        const uint32_t sl = r.count(1, "regex source");
        std::string src = r.str(sl);
        if (!valid_utf8(src)) bad("regex pattern is not valid UTF-8");
        d.regex_sources.push_back(std::move(src));
        d.regex_pattern_ids.push_back(id);
      }
    }
    // literal pattern ids
    const uint32_t n_ids = r.count(4, "literal ID table");
    if (n_ids != n_literals) bad("literal ID table is inconsistent");
    d.literal_pattern_ids = r.u32s(n_ids);
    // LiteralPrefilterTable (mod.rs:590-636)
    const uint32_t n_meta = r.count(16, "prefix meta table");
    std::vector<uint32_t> meta = r.u32s(4 * n_meta);
    const uint32_t n_ranges = r.count(8, "bucket range table");
    std::vector<uint32_t> ranges = r.u32s(2 * n_ranges);
    const uint32_t n_entries = r.count(8, "prefilter entry table");
    std::vector<uint32_t> entries = r.u32s(2 * n_entries);
    for (uint32_t b = 0; b < n_ranges; ++b)  // validate_prefilter_ranges (mod.rs:702-725)
      if ((uint64_t)ranges[2 * b] + ranges[2 * b + 1] > n_entries) bad("prefilter bucket range points past its entries");
    // the regex DFAs: shape-checked and skipped (mod.rs:217-241, dfa/mod.rs:250-283)
    for (uint32_t k = 0; k < n_dfas; ++k) {
      const uint32_t nt = r.count(4, "DFA transition table");
      r.take((size_t)nt * 4);
      r.take((size_t)r.count(4, "DFA match-list pointers") * 4);
      r.take((size_t)r.count(4, "DFA match lists") * 4);
      r.take((size_t)r.count(4, "DFA pattern lengths") * 4);
      r.u32();  // start state
      const uint32_t classes = r.u32(), eoi = r.u32();
      if (classes == 0) bad("DFA has class_count=0");
      if (nt % classes != 0) bad("DFA transition table is not a multiple of its class count");
      if (eoi >= classes) bad("DFA eoi_class is not below its class count");
      r.take(256 * 4);
      r.take(r.count(1, "serialized DFA"));
      r.take((size_t)r.count(4, "DFA original ids") * 4);
    }
    if (r.remaining() != 0) bad("contains trailing bytes");
    if (n_dfas && !has_sources)
      bad("lacks serialized regex patterns (a version 1 index); rebuild it with a release that stores regex sources");

    // every pattern id is a literal or a regex, exactly once (mod.rs:289-377)
    std::vector<uint8_t> seen_lit(n_patterns, 0);
    for (uint32_t li = 0; li < n_literals; ++li) {
      const uint32_t id = d.literal_pattern_ids[li];
      if (id >= n_patterns) bad("literal pattern ID is out of bounds");
      if (seen_lit[id] || seen_regex[id]) bad("contains duplicate literal IDs");
      seen_lit[id] = 1;
      const uint64_t s = d.offsets[2 * li], l = d.offsets[2 * li + 1];
      if (s + l > packed_len) bad("literal offset points outside the packed byte buffer");
      if (l == 0) bad("holds an empty literal");
    }
    for (uint32_t id = 0; id < n_patterns; ++id)
      if (!seen_lit[id] && !seen_regex[id]) bad("has missing pattern metadata");
    if (n_patterns == 0) raise(WS_ERR_EMPTY_PATTERN_SET, "compiled index holds no patterns");
    d.n_patterns = n_patterns;

    // The kernels probe the prefilter table directly.  Keep the file's table
    // when it is one the probe can use safely and exactly (window 8, every
    // entry names a literal with that FNV-1a prefix hash, every partition's
    // buckets inside the range table); otherwise build it from the literals.
    for (uint32_t li = 0; li < n_literals; ++li)
      d.literal_hashes.push_back(fnv1a(d.packed_bytes.data() + d.offsets[2 * li], d.offsets[2 * li + 1], HASH_WINDOW));
    bool usable = window == HASH_WINDOW && n_meta == HASH_WINDOW && n_entries == n_literals;
    for (uint32_t e = 0; usable && e < n_entries; ++e)
      usable = entries[2 * e + 1] < n_literals && entries[2 * e] == d.literal_hashes[entries[2 * e + 1]];
    for (uint32_t g = 0; usable && g < n_meta; ++g) {
      const uint64_t first = meta[4 * g], mask = meta[4 * g + 1];
      bool has = false;
      for (uint32_t li = 0; li < n_literals && !has; ++li)
        has = std::max<uint32_t>(std::min(d.offsets[2 * li + 1], HASH_WINDOW), 1) == g + 1;
      if (has) usable = ((mask + 1) & mask) == 0 && first + mask < n_ranges;
    }
    if (usable) {
      d.prefix_meta = std::move(meta);
      d.bucket_ranges = std::move(ranges);
      d.entries = std::move(entries);
    } else {
      build_prefilter_table(d.offsets, d.literal_hashes, HASH_WINDOW, d.prefix_meta, d.bucket_ranges, d.entries);
    }
    for (auto& s : d.regex_sources) d.regex_ptrs.push_back(s.c_str());
    *out = ir.release();
  });
}

extern "C" ws_status ws_index_save(const ws_ir* ir, uint8_t* out, uint64_t cap, uint64_t* n_out,
                                   ws_error_info* err) {
  return run_guarded(err, [&] {
    if (!ir || !n_out || (cap && !out)) raise(WS_ERR_INVALID_ARGUMENT, "null argument");
    *n_out = 0;
    const IrData& d = ir->d;
    const uint32_t n_lit = (uint32_t)d.literal_pattern_ids.size();
    std::vector<uint8_t> b;
    b.insert(b.end(), kMagic, kMagic + 8);
    put32(b, kIndexVersion);
    put32(b, d.case_insensitive ? 1 : 0);
    put32(b, d.n_patterns);
    put32(b, n_lit);
    put32(b, 0);  // no serialized regex-automata DFAs
    put32(b, HASH_WINDOW);
    put32(b, checked_u32(d.packed_bytes.size(), "packed literal bytes"));
    b.insert(b.end(), d.packed_bytes.begin(), d.packed_bytes.end());
    put32(b, n_lit);
    for (uint32_t v : d.offsets) put32(b, v);
    put32(b, d.n_patterns);
    for (uint32_t i = 0; i < d.n_patterns; ++i) {
      if (i < d.named.size() && d.named[i]) {
        put32(b, checked_u32(d.names[i].size(), "pattern name"));
        b.insert(b.end(), d.names[i].begin(), d.names[i].end());
      } else {
        put32(b, 0xFFFFFFFFu);
      }
    }
    put32(b, (uint32_t)d.regex_sources.size());
    for (size_t k = 0; k < d.regex_sources.size(); ++k) {
      put32(b, d.regex_pattern_ids[k]);
      put32(b, checked_u32(d.regex_sources[k].size(), "regex source"));
      b.insert(b.end(), d.regex_sources[k].begin(), d.regex_sources[k].end());
    }
    put32(b, n_lit);
    for (uint32_t v : d.literal_pattern_ids) put32(b, v);
    put32(b, (uint32_t)(d.prefix_meta.size() / 4));
    for (uint32_t v : d.prefix_meta) put32(b, v);
    put32(b, (uint32_t)(d.bucket_ranges.size() / 2));
    for (uint32_t v : d.bucket_ranges) put32(b, v);
    put32(b, (uint32_t)(d.entries.size() / 2));
    for (uint32_t v : d.entries) put32(b, v);
    put32(b, crc32_ieee(b.data(), b.size()));
    *n_out = b.size();
    if (b.size() > cap) raise(WS_ERR_OVERFLOW, "output buffer is too small for the index", 0, b.size(), cap);
    std::memcpy(out, b.data(), b.size());
  });
}

extern "C" ws_status ws_ir_set_name(ws_ir* ir, uint64_t pattern_id, const char* name, uint64_t len) {
  if (!ir || (len && !name) || pattern_id >= ir->d.n_patterns) return WS_ERR_INVALID_ARGUMENT;
  IrData& d = ir->d;
  d.names.resize(d.n_patterns);
  d.named.resize(d.n_patterns, 0);
  d.names[pattern_id].assign(name ? name : "", (size_t)len);
  if (!valid_utf8(d.names[pattern_id])) return WS_ERR_INVALID_ARGUMENT;
  d.named[pattern_id] = 1;
  return WS_OK;
}

extern "C" ws_status ws_ir_name(const ws_ir* ir, uint64_t pattern_id, char* out, uint64_t cap, uint64_t* n_out) {
  if (!ir || !n_out || (cap && !out) || pattern_id >= ir->d.n_patterns) return WS_ERR_INVALID_ARGUMENT;
  const IrData& d = ir->d;
  if (pattern_id >= d.named.size() || !d.named[pattern_id]) {
    *n_out = UINT64_MAX;  // no name
    return WS_OK;
  }
  const std::string& s = d.names[pattern_id];
  *n_out = s.size();
  if (s.size() > cap) return WS_ERR_OVERFLOW;
  std::memcpy(out, s.data(), s.size());
  return WS_OK;
}
