// Regex front end for the B200 scan path (see ws_regex.h).
#include "ws_regex.h"

#include <algorithm>
#include <cstring>
#include <unordered_map>

namespace ws {

namespace {

enum Look { LK_LINE_START = 1, LK_LINE_END, LK_TEXT_START, LK_TEXT_END, LK_WORD, LK_NOT_WORD };
static_assert((int)LK_LINE_START == (int)LOOK_LINE_START && (int)LK_LINE_END == (int)LOOK_LINE_END &&
                  (int)LK_TEXT_START == (int)LOOK_TEXT_START && (int)LK_TEXT_END == (int)LOOK_TEXT_END &&
                  (int)LK_WORD == (int)LOOK_WORD && (int)LK_NOT_WORD == (int)LOOK_NOT_WORD,
              "parser and NFA look-around kinds agree");

struct Mode {
  bool ci = false;       // (?i)
  bool ml = true;        // (?m): multi_line(true) is the reference's default
  bool dotnl = false;    // (?s)
  bool lazy = false;     // (?U)
};

ByteSet range_set(int lo, int hi) {
  ByteSet s;
  for (int c = lo; c <= hi; ++c) s.set((size_t)c);
  return s;
}

ByteSet ascii_case_fold(ByteSet s) {
  for (int up = 'A'; up <= 'Z'; ++up) {
    int lo = up + 32;
    if (s.test((size_t)up) || s.test((size_t)lo)) { s.set((size_t)up); s.set((size_t)lo); }
  }
  return s;
}

ByteSet perl_class(char c) {
  ByteSet d = range_set('0', '9');
  ByteSet w = d | range_set('a', 'z') | range_set('A', 'Z');
  w.set('_');
  ByteSet sp;
  for (char x : {'\t', '\n', '\v', '\f', '\r', ' '}) sp.set((size_t)(unsigned char)x);
  switch (c) {
    case 'd': return d;
    case 'D': return ~d;
    case 'w': return w;
    case 'W': return ~w;
    case 's': return sp;
    default: return ~sp;  // 'S'
  }
}

bool posix_class(const std::string& name, ByteSet* out) {
  struct P { const char* n; int kind; };
  ByteSet r;
  if (name == "alnum") r = range_set('0', '9') | range_set('a', 'z') | range_set('A', 'Z');
  else if (name == "alpha") r = range_set('a', 'z') | range_set('A', 'Z');
  else if (name == "ascii") r = range_set(0, 127);
  else if (name == "blank") { r.set(' '); r.set('\t'); }
  else if (name == "cntrl") { r = range_set(0, 31); r.set(127); }
  else if (name == "digit") r = range_set('0', '9');
  else if (name == "graph") r = range_set(33, 126);
  else if (name == "lower") r = range_set('a', 'z');
  else if (name == "print") r = range_set(32, 126);
  else if (name == "punct") r = range_set(33, 47) | range_set(58, 64) | range_set(91, 96) | range_set(123, 126);
  else if (name == "space") { r = range_set(9, 13); r.set(' '); }
  else if (name == "upper") r = range_set('A', 'Z');
  else if (name == "word") { r = range_set('0', '9') | range_set('a', 'z') | range_set('A', 'Z'); r.set('_'); }
  else if (name == "xdigit") r = range_set('0', '9') | range_set('a', 'f') | range_set('A', 'F');
  else return false;
  *out = r;
  return true;
}

int hex_digit(char c) {
  if (c >= '0' && c <= '9') return c - '0';
  c = (char)(c | 0x20);
  if (c >= 'a' && c <= 'f') return c - 'a' + 10;
  return -1;
}

class RegexParser {
 public:
  explicit RegexParser(const std::string& s) : src_(s) {}

  ReTree run() {
    Mode m;
    tree_.root = alternation(m);
    if (pos_ != src_.size()) fail("unmatched ')'");
    return std::move(tree_);
  }

 private:
  const std::string& src_;
  size_t pos_ = 0;
  ReTree tree_;

  [[noreturn]] void fail(const std::string& why) const {
    throw CompileError("regex parse error at offset " + std::to_string(pos_) + ": " + why);
  }
  bool more() const { return pos_ < src_.size(); }
  char cur() const { return src_[pos_]; }
  bool accept(char c) {
    if (more() && cur() == c) { ++pos_; return true; }
    return false;
  }
  int node(ReNode n) { tree_.nodes.push_back(std::move(n)); return (int)tree_.nodes.size() - 1; }
  int bytes_node(ByteSet s) { ReNode n; n.type = ReNode::BYTES; n.bytes = s; return node(std::move(n)); }
  int literal_byte(uint8_t b, const Mode& m) {
    ByteSet s; s.set(b);
    return bytes_node(m.ci ? ascii_case_fold(s) : s);
  }

  int alternation(Mode& m) {
    std::vector<int> branches{sequence(m)};
    while (accept('|')) branches.push_back(sequence(m));
    if (branches.size() == 1) return branches[0];
    ReNode n; n.type = ReNode::ALT; n.kids = std::move(branches);
    return node(std::move(n));
  }

  int sequence(Mode& m) {
    std::vector<int> items;
    while (more() && cur() != '|' && cur() != ')') {
      int atom_id = atom(m);
      if (atom_id < 0) continue;  // a bare flag group changed `m`
      items.push_back(repetitions(atom_id, m));
    }
    if (items.empty()) { ReNode n; n.type = ReNode::EMPTY; return node(std::move(n)); }
    if (items.size() == 1) return items[0];
    ReNode n; n.type = ReNode::CAT; n.kids = std::move(items);
    return node(std::move(n));
  }

  bool read_count(int* v) {
    size_t b = pos_;
    long long x = 0;
    while (more() && cur() >= '0' && cur() <= '9') {
      x = x * 10 + (cur() - '0');
      if (x > 1000000) fail("repetition count too large");
      ++pos_;
    }
    *v = (int)x;
    return pos_ > b;
  }

  int repetitions(int atom_id, const Mode& m) {
    bool done_one = false;
    for (;;) {
      if (!more()) break;
      int lo, hi;
      char c = cur();
      if (c == '*') { lo = 0; hi = -1; ++pos_; }
      else if (c == '+') { lo = 1; hi = -1; ++pos_; }
      else if (c == '?') { lo = 0; hi = 1; ++pos_; }
      else if (c == '{') {
        ++pos_;
        if (!read_count(&lo)) fail("repetition quantifier expects a decimal");
        if (accept(',')) {
          if (more() && cur() == '}') hi = -1;
          else if (!read_count(&hi)) fail("repetition quantifier expects a decimal");
        } else {
          hi = lo;
        }
        if (!accept('}')) fail("unclosed counted repetition");
        if (hi >= 0 && hi < lo) fail("invalid repetition range");
      } else {
        break;
      }
      if (done_one) fail("repetition operator missing expression");
      if (tree_.nodes[(size_t)atom_id].type == ReNode::EMPTY) fail("repetition operator missing expression");
      bool greedy = !accept('?');
      if (m.lazy) greedy = !greedy;
      ReNode n; n.type = ReNode::REP; n.kids = {atom_id}; n.lo = lo; n.hi = hi; n.greedy = greedy;
      atom_id = node(std::move(n));
      done_one = true;
    }
    return atom_id;
  }

  // After a backslash.  Returns 0: byte in *b; 1: set in *s; 2: look in *lk.
  int escape(uint8_t* b, ByteSet* s, int* lk, bool in_class) {
    if (!more()) fail("incomplete escape sequence");
    char c = src_[pos_++];
    switch (c) {
      case 'd': case 'D': case 'w': case 'W': case 's': case 'S':
        *s = perl_class(c); return 1;
      case 'n': *b = '\n'; return 0;
      case 't': *b = '\t'; return 0;
      case 'r': *b = '\r'; return 0;
      case 'f': *b = '\f'; return 0;
      case 'v': *b = '\v'; return 0;
      case 'a': *b = 0x07; return 0;
      case 'e': *b = 0x1B; return 0;
      case 'x': {
        unsigned v = 0;
        if (accept('{')) {
          int digits = 0;
          while (more() && cur() != '}') {
            int h = hex_digit(src_[pos_++]);
            if (h < 0 || ++digits > 8) fail("invalid hex escape");
            v = v * 16 + (unsigned)h;
          }
          if (!accept('}') || digits == 0) fail("invalid hex escape");
        } else {
          if (pos_ + 2 > src_.size()) fail("invalid hex escape");
          int h1 = hex_digit(src_[pos_]), h2 = hex_digit(src_[pos_ + 1]);
          if (h1 < 0 || h2 < 0) fail("invalid hex escape");
          v = (unsigned)(h1 * 16 + h2);
          pos_ += 2;
        }
        if (v > 0xFF) fail("escape above \\xFF needs Unicode mode, which is disabled");
        *b = (uint8_t)v;
        return 0;
      }
      case 'b': case 'B': case 'A': case 'z':
        if (in_class) fail("assertion inside a character class");
        *lk = (c == 'b') ? LK_WORD : (c == 'B') ? LK_NOT_WORD : (c == 'A') ? LK_TEXT_START : LK_TEXT_END;
        return 2;
      case 'p': case 'P':
        fail("Unicode classes need Unicode mode, which is disabled");
      default:
        if ((unsigned char)c < 0x80 && !std::isalnum((unsigned char)c)) { *b = (uint8_t)c; return 0; }
        fail(std::string("unrecognized escape sequence \\") + c);
    }
  }

  // One endpoint of a class range: a byte (returns true) or a whole set.
  bool class_item(uint8_t* b, ByteSet* s) {
    if (!more()) fail("unclosed character class");
    unsigned char c = (unsigned char)cur();
    if (c == '\\') {
      ++pos_;
      int lk = 0;
      return escape(b, s, &lk, true) == 0;
    }
    if (c >= 0x80) fail("non-ASCII character in a class needs Unicode mode, which is disabled");
    ++pos_;
    *b = c;
    return true;
  }

  ByteSet bracket(const Mode& m) {
    bool negated = accept('^');
    ByteSet acc;
    bool first = true;
    for (;;) {
      if (!more()) fail("unclosed character class");
      if (cur() == ']' && !first) { ++pos_; break; }
      first = false;
      if (cur() == '[') {
        if (src_.compare(pos_, 2, "[:") == 0) {
          size_t close = src_.find(":]", pos_ + 2);
          if (close != std::string::npos) {
            std::string name = src_.substr(pos_ + 2, close - pos_ - 2);
            bool neg = !name.empty() && name[0] == '^';
            if (neg) name.erase(0, 1);
            ByteSet ps;
            if (posix_class(name, &ps)) {
              acc |= neg ? ~ps : ps;
              pos_ = close + 2;
              continue;
            }
          }
        }
        ++pos_;
        acc |= bracket(m);
        continue;
      }
      if (src_.compare(pos_, 2, "&&") == 0 || src_.compare(pos_, 2, "--") == 0 ||
          src_.compare(pos_, 2, "~~") == 0)
        fail("character class set operations are not supported");
      uint8_t lo = 0;
      ByteSet s;
      if (!class_item(&lo, &s)) { acc |= s; continue; }
      if (more() && cur() == '-' && pos_ + 1 < src_.size() && src_[pos_ + 1] != ']') {
        ++pos_;
        uint8_t hi = 0;
        ByteSet s2;
        if (!class_item(&hi, &s2)) fail("invalid range in character class");
        if (hi < lo) fail("invalid range in character class");
        acc |= range_set(lo, hi);
      } else {
        acc.set(lo);
      }
    }
    if (m.ci) acc = ascii_case_fold(acc);
    return negated ? ~acc : acc;
  }

  // Returns -1 for a flag-only group "(?i)" (which updates m in place).
  int atom(Mode& m) {
    char c = cur();
    switch (c) {
      case '(': {
        ++pos_;
        Mode inner = m;
        bool capture = true;
        if (accept('?')) {
          if (src_.compare(pos_, 2, "P<") == 0 || (more() && cur() == '<')) {
            pos_ += (cur() == 'P') ? 2 : 1;
            size_t close = src_.find('>', pos_);
            if (close == std::string::npos || close == pos_) fail("invalid capture group name");
            pos_ = close + 1;
          } else {
            bool neg = false, colon = false;
            for (;;) {
              if (!more()) fail("unclosed group");
              char f = src_[pos_++];
              if (f == ':') { colon = true; break; }
              if (f == ')') break;
              if (f == '-') { if (neg) fail("repeated negation in flags"); neg = true; continue; }
              bool on = !neg;
              switch (f) {
                case 'i': inner.ci = on; break;
                case 'm': inner.ml = on; break;
                case 's': inner.dotnl = on; break;
                case 'U': inner.lazy = on; break;
                case 'u': if (on) fail("Unicode mode is disabled"); break;
                case 'x': if (on) fail("verbose mode is not supported"); break;
                case 'R': if (on) fail("CRLF mode is not supported"); break;
                default: fail(std::string("unrecognized flag ") + f);
              }
            }
            if (!colon) { m = inner; return -1; }
            capture = false;
          }
        }
        int body = alternation(inner);
        if (!accept(')')) fail("unclosed group");
        if (!capture) return body;  // non-capturing groups leave no node (as in the HIR)
        ReNode n; n.type = ReNode::CAPTURE; n.kids = {body};
        return node(std::move(n));
      }
      case ')': fail("unopened group");
      case '[': { ++pos_; return bytes_node(bracket(m)); }
      case '.': {
        ++pos_;
        ByteSet s; s.set();
        if (!m.dotnl) s.reset('\n');
        return bytes_node(s);
      }
      case '^': case '$': {
        ++pos_;
        ReNode n; n.type = ReNode::LOOK;
        n.look = (c == '^') ? (m.ml ? LK_LINE_START : LK_TEXT_START) : (m.ml ? LK_LINE_END : LK_TEXT_END);
        return node(std::move(n));
      }
      case '*': case '+': case '?': fail("repetition operator missing expression");
      case '\\': {
        ++pos_;
        uint8_t b = 0; ByteSet s; int lk = 0;
        int k = escape(&b, &s, &lk, false);
        if (k == 0) return literal_byte(b, m);
        if (k == 1) return bytes_node(s);
        ReNode n; n.type = ReNode::LOOK; n.look = lk;
        return node(std::move(n));
      }
      default: break;
    }
    unsigned char uc = (unsigned char)c;
    if (uc >= 0x80) {
      // A UTF-8 encoded character matches its encoded byte sequence.
      int n_bytes = uc >= 0xF0 ? 4 : uc >= 0xE0 ? 3 : uc >= 0xC0 ? 2 : 1;
      std::vector<int> seq;
      for (int k = 0; k < n_bytes && more(); ++k) {
        ByteSet s; s.set((unsigned char)src_[pos_++]);
        seq.push_back(bytes_node(s));
      }
      if (seq.size() == 1) return seq[0];
      ReNode n; n.type = ReNode::CAT; n.kids = std::move(seq);
      return node(std::move(n));
    }
    ++pos_;
    return literal_byte(uc, m);
  }
};

// --------------------------------------------------------------- analyses
bool literal_rec(const ReTree& t, int id, std::vector<uint8_t>* out) {
  const ReNode& n = t.nodes[(size_t)id];
  if (n.type == ReNode::BYTES) {
    if (n.bytes.count() != 1) return false;
    for (int c = 0; c < 256; ++c)
      if (n.bytes.test((size_t)c)) out->push_back((uint8_t)c);
    return true;
  }
  if (n.type == ReNode::CAPTURE) return literal_rec(t, n.kids[0], out);
  if (n.type == ReNode::CAT) {
    bool any = false;
    for (int k : n.kids) {
      if (t.nodes[(size_t)k].type == ReNode::EMPTY) continue;  // dropped from a concat
      if (!literal_rec(t, k, out)) return false;
      any = true;
    }
    return any;
  }
  return false;
}

bool contains_rep(const ReTree& t, int id) {
  const ReNode& n = t.nodes[(size_t)id];
  if (n.type == ReNode::REP) return true;
  if (n.type == ReNode::CAT || n.type == ReNode::ALT || n.type == ReNode::CAPTURE)
    for (int k : n.kids) if (contains_rep(t, k)) return true;
  return false;
}

bool patho_rec(const ReTree& t, int id) {
  const ReNode& n = t.nodes[(size_t)id];
  if (n.type == ReNode::REP) {
    bool outer_unbounded = n.hi < 0 || n.hi > 1;
    if (outer_unbounded && contains_rep(t, n.kids[0])) return true;
    return patho_rec(t, n.kids[0]);
  }
  if (n.type == ReNode::CAT || n.type == ReNode::ALT || n.type == ReNode::CAPTURE)
    for (int k : n.kids) if (patho_rec(t, k)) return true;
  return false;
}

// (min, max) match length; max = -1 unbounded
void len_rec(const ReTree& t, int id, int64_t* mn, int64_t* mx) {
  const ReNode& n = t.nodes[(size_t)id];
  switch (n.type) {
    case ReNode::BYTES: *mn = 1; *mx = 1; return;
    case ReNode::LOOK: case ReNode::EMPTY: *mn = 0; *mx = 0; return;
    case ReNode::CAPTURE: len_rec(t, n.kids[0], mn, mx); return;
    case ReNode::CAT: {
      int64_t a = 0, b = 0;
      for (int k : n.kids) {
        int64_t x, y; len_rec(t, k, &x, &y);
        a += x;
        b = (b < 0 || y < 0) ? -1 : b + y;
      }
      *mn = a; *mx = b; return;
    }
    case ReNode::ALT: {
      int64_t a = INT64_MAX, b = 0;
      for (int k : n.kids) {
        int64_t x, y; len_rec(t, k, &x, &y);
        a = std::min(a, x);
        b = (b < 0 || y < 0) ? -1 : std::max(b, y);
      }
      *mn = a; *mx = b; return;
    }
    case ReNode::REP: {
      int64_t x, y; len_rec(t, n.kids[0], &x, &y);
      *mn = x * n.lo;
      if (n.hi < 0) *mx = (y == 0) ? 0 : -1;
      else *mx = (y < 0) ? -1 : y * n.hi;
      return;
    }
  }
}

bool look_rec(const ReTree& t, int id) {
  const ReNode& n = t.nodes[(size_t)id];
  if (n.type == ReNode::LOOK) return true;
  for (int k : n.kids) if (look_rec(t, k)) return true;
  return false;
}

// ------------------------------------------------------------------ NFA build
struct NfaBuilder {
  Nfa& nfa;
  const ReTree& t;
  bool reverse;
  NfaBuilder(Nfa& n, const ReTree& tr, bool rev) : nfa(n), t(tr), reverse(rev) {}

  int add(NfaState s) { nfa.states.push_back(s); return (int)nfa.states.size() - 1; }

  // Compiles node `id` so that it continues into `next`; returns its entry.
  int compile(int id, int next) {
    const ReNode& n = t.nodes[(size_t)id];
    switch (n.type) {
      case ReNode::BYTES: {
        nfa.sets.push_back(n.bytes);
        NfaState s; s.kind = NfaState::CONSUME; s.a = next; s.set = (int)nfa.sets.size() - 1;
        return add(s);
      }
      case ReNode::EMPTY: return next;
      case ReNode::LOOK: {
        // a reversed pattern sees every look-behind as a look-ahead and back
        int look = n.look;
        if (reverse) {
          look = look == LOOK_LINE_START ? LOOK_LINE_END
                 : look == LOOK_LINE_END ? LOOK_LINE_START
                 : look == LOOK_TEXT_START ? LOOK_TEXT_END
                 : look == LOOK_TEXT_END ? LOOK_TEXT_START
                                         : look;
        }
        NfaState s; s.kind = NfaState::ASSERT; s.a = next; s.look = look;
        return add(s);
      }
      case ReNode::CAPTURE: return compile(n.kids[0], next);
      case ReNode::CAT: {
        int entry = next;
        if (!reverse) {
          for (size_t k = n.kids.size(); k-- > 0;) entry = compile(n.kids[k], entry);
        } else {
          for (size_t k = 0; k < n.kids.size(); ++k) entry = compile(n.kids[k], entry);
        }
        return entry;
      }
      case ReNode::ALT: {
        // priority: earlier branches first
        int entry = compile(n.kids.back(), next);
        for (size_t k = n.kids.size() - 1; k-- > 0;) {
          int br = compile(n.kids[k], next);
          NfaState s; s.kind = NfaState::SPLIT; s.a = br; s.b = entry;
          entry = add(s);
        }
        return entry;
      }
      case ReNode::REP: {
        int sub = n.kids[0];
        int tail = next;
        if (n.hi < 0) {
          // loop: split -> (sub -> split) | next
          NfaState sp; sp.kind = NfaState::SPLIT;
          int split = add(sp);
          int body = compile(sub, split);
          if (n.greedy) { nfa.states[(size_t)split].a = body; nfa.states[(size_t)split].b = next; }
          else { nfa.states[(size_t)split].a = next; nfa.states[(size_t)split].b = body; }
          tail = split;
        } else {
          for (int r = n.lo; r < n.hi; ++r) {
            int body = compile(sub, tail);
            NfaState sp; sp.kind = NfaState::SPLIT;
            if (n.greedy) { sp.a = body; sp.b = next; } else { sp.a = next; sp.b = body; }
            tail = add(sp);
          }
        }
        for (int r = 0; r < n.lo; ++r) tail = compile(sub, tail);
        return tail;
      }
    }
    return next;
  }
};

// Note on optional repetitions x{lo,hi}: the chain built above is
//   x^lo (split -> x (split -> x ... | next) | next)
// so every optional copy can exit straight to `next`, with greedy preferring one
// more copy -- the same priority order as nested (x(x(x)?)?)?.

struct VecHash {
  size_t operator()(const std::vector<uint32_t>& v) const {
    uint64_t h = 1469598103934665603ull;
    for (uint32_t x : v) { h ^= x; h *= 1099511628211ull; }
    return (size_t)h;
  }
};

}  // namespace

ReTree parse_regex(const std::string& src) {
  RegexParser p(src);
  return p.run();
}

bool tree_literal(const ReTree& t, std::vector<uint8_t>* out) {
  out->clear();
  return literal_rec(t, t.root, out) && !out->empty();
}
bool tree_pathological(const ReTree& t) { return patho_rec(t, t.root); }
bool tree_nullable(const ReTree& t) { int64_t a = 0, b = 0; len_rec(t, t.root, &a, &b); return a == 0; }
bool tree_has_look(const ReTree& t) { return look_rec(t, t.root); }
int64_t tree_max_len(const ReTree& t) { int64_t a = 0, b = 0; len_rec(t, t.root, &a, &b); return b; }

Nfa build_nfa(const std::vector<const ReTree*>& trees, bool reverse) {
  Nfa nfa;
  for (size_t p = 0; p < trees.size(); ++p) {
    NfaState m; m.kind = NfaState::MATCH; m.pattern = (int)p;
    nfa.states.push_back(m);
    int match = (int)nfa.states.size() - 1;
    NfaBuilder b(nfa, *trees[p], reverse);
    nfa.starts.push_back(b.compile(trees[p]->root, match));
  }
  return nfa;
}

bool look_holds(int look, int left, int right) {
  switch (look) {
    case LOOK_LINE_START: return left == CTX_BEGIN || left == CTX_NL;
    case LOOK_LINE_END: return right == CTX_BEGIN || right == CTX_NL;
    case LOOK_TEXT_START: return left == CTX_BEGIN;
    case LOOK_TEXT_END: return right == CTX_BEGIN;
    case LOOK_WORD: return (left == CTX_WORD) != (right == CTX_WORD);
    case LOOK_NOT_WORD: return (left == CTX_WORD) == (right == CTX_WORD);
  }
  return false;
}

ByteClasses compute_classes(const std::vector<const Nfa*>& nfas) {
  // Refine the single class {0..255} by every set: two bytes stay together only
  // if every set contains both or neither.  With assertions, the byte contexts
  // (line feed, word bytes, others) are sets too.
  std::vector<uint64_t> sig(256, 0);
  std::vector<uint32_t> cls(256, 0);
  uint32_t n_cls = 1;
  std::vector<ByteSet> context_sets;
  for (const Nfa* nfa : nfas)
    for (const NfaState& q : nfa->states)
      if (q.kind == NfaState::ASSERT && context_sets.empty()) {
        ByteSet nl, word;
        nl.set('\n');
        for (int b = 0; b < 256; ++b) if (byte_context((uint8_t)b) == CTX_WORD) word.set((size_t)b);
        context_sets = {nl, word};
      }
  std::vector<const std::vector<ByteSet>*> all;
  for (const Nfa* nfa : nfas) all.push_back(&nfa->sets);
  all.push_back(&context_sets);
  for (const std::vector<ByteSet>* sets : all) {
    for (const ByteSet& s : *sets) {
      std::unordered_map<uint64_t, uint32_t> remap;
      std::vector<uint32_t> next(256);
      uint32_t k = 0;
      for (int b = 0; b < 256; ++b) {
        uint64_t key = (uint64_t)cls[(size_t)b] * 2 + (s.test((size_t)b) ? 1 : 0);
        auto it = remap.find(key);
        if (it == remap.end()) it = remap.emplace(key, k++).first;
        next[(size_t)b] = it->second;
      }
      cls = next;
      n_cls = k;
    }
  }
  ByteClasses bc;
  bc.count = (int)n_cls;
  bc.representative.assign(n_cls, 0);
  std::vector<uint8_t> seen(n_cls, 0);
  for (int b = 0; b < 256; ++b) {
    bc.map[b] = (uint8_t)cls[(size_t)b];
    if (!seen[cls[(size_t)b]]) { seen[cls[(size_t)b]] = 1; bc.representative[cls[(size_t)b]] = (uint8_t)b; }
  }
  (void)sig;
  return bc;
}

namespace {

// Unordered epsilon closure: keeps CONSUME and MATCH states.
void closure_all(const Nfa& nfa, int start, std::vector<uint32_t>& mark, uint32_t stamp,
                 std::vector<uint32_t>& out, std::vector<int>& stack) {
  stack.clear();
  stack.push_back(start);
  while (!stack.empty()) {
    int q = stack.back();
    stack.pop_back();
    if (mark[(size_t)q] == stamp) continue;
    mark[(size_t)q] = stamp;
    const NfaState& s = nfa.states[(size_t)q];
    switch (s.kind) {
      case NfaState::CONSUME: case NfaState::MATCH: out.push_back((uint32_t)q); break;
      case NfaState::SPLIT: stack.push_back(s.b); stack.push_back(s.a); break;
      case NfaState::EPS: stack.push_back(s.a); break;
      case NfaState::ASSERT: throw CompileError("assertion in a DFA without contexts");
    }
  }
}

}  // namespace

Dfa build_all_dfa(const Nfa& nfa, const ByteClasses& cls, bool with_unanchored, int max_states) {
  Dfa d;
  d.n_classes = cls.count;
  const size_t nn = nfa.states.size();
  std::vector<uint32_t> mark(nn, 0);
  uint32_t stamp = 0;
  std::vector<int> stack;

  // closure of all pattern starts
  std::vector<uint32_t> start_set;
  ++stamp;
  for (int s : nfa.starts) closure_all(nfa, s, mark, stamp, start_set, stack);
  std::sort(start_set.begin(), start_set.end());

  // successor closure per CONSUME state, computed once
  std::vector<std::vector<uint32_t>> succ(nn);
  for (size_t q = 0; q < nn; ++q) {
    if (nfa.states[q].kind != NfaState::CONSUME) continue;
    ++stamp;
    closure_all(nfa, nfa.states[q].a, mark, stamp, succ[q], stack);
  }

  // DFA state key: sorted NFA ids; the unanchored flag is part of the key
  // (an unanchored state re-injects the start closure after every byte).
  std::unordered_map<std::vector<uint32_t>, uint32_t, VecHash> index;
  std::vector<std::vector<uint32_t>> sets;
  std::vector<uint8_t> unanch;
  auto intern = [&](std::vector<uint32_t>&& key, bool u) -> uint32_t {
    std::vector<uint32_t> k = key;
    k.push_back(u ? 1u : 0u);
    auto it = index.find(k);
    if (it != index.end()) return it->second;
    uint32_t id = (uint32_t)sets.size();
    index.emplace(std::move(k), id);
    sets.push_back(std::move(key));
    unanch.push_back(u ? 1 : 0);
    return id;
  };
  intern({}, false);  // 0: dead
  d.start_anchored = intern(std::vector<uint32_t>(start_set), false);
  if (with_unanchored) d.start_unanchored = intern(std::vector<uint32_t>(start_set), true);

  const int C = cls.count;
  std::vector<uint32_t> nxt;
  for (size_t cur = 0; cur < sets.size(); ++cur) {
    if ((int)sets.size() > max_states) { d.too_big = true; return d; }
    d.trans.resize((cur + 1) * (size_t)C, 0);
    if (cur == 0) continue;  // dead state loops to itself (0)
    for (int c = 0; c < C; ++c) {
      uint8_t b = cls.representative[(size_t)c];
      ++stamp;
      nxt.clear();
      for (uint32_t q : sets[cur]) {
        const NfaState& s = nfa.states[q];
        if (s.kind != NfaState::CONSUME || !nfa.sets[(size_t)s.set].test(b)) continue;
        for (uint32_t r : succ[q]) if (mark[r] != stamp) { mark[r] = stamp; nxt.push_back(r); }
      }
      if (unanch[cur]) for (uint32_t r : start_set) if (mark[r] != stamp) { mark[r] = stamp; nxt.push_back(r); }
      std::sort(nxt.begin(), nxt.end());
      uint32_t id = (nxt.empty() && !unanch[cur]) ? 0u : intern(std::vector<uint32_t>(nxt), unanch[cur] != 0);
      d.trans[cur * (size_t)C + (size_t)c] = id;
    }
  }
  d.n_states = (int)sets.size();
  // match lists and flags
  d.is_match.assign((size_t)d.n_states, 0);
  d.match_ptr.assign((size_t)d.n_states + 1, 0);
  for (int s = 0; s < d.n_states; ++s) {
    d.match_ptr[(size_t)s] = (uint32_t)d.match_list.size();
    std::vector<uint32_t> pats;
    for (uint32_t q : sets[(size_t)s])
      if (nfa.states[q].kind == NfaState::MATCH) pats.push_back((uint32_t)nfa.states[q].pattern);
    std::sort(pats.begin(), pats.end());
    pats.erase(std::unique(pats.begin(), pats.end()), pats.end());
    if (!pats.empty()) d.is_match[(size_t)s] = 1;
    d.match_list.insert(d.match_list.end(), pats.begin(), pats.end());
  }
  d.match_ptr[(size_t)d.n_states] = (uint32_t)d.match_list.size();
  for (auto& w : d.trans) {
    uint32_t t = w;
    w = t | (d.is_match[t] ? DFA_FLAG_MATCH : 0u) | (t == 0 ? DFA_FLAG_DEAD : 0u);
  }
  return d;
}

Dfa build_leftmost_first_dfa(const Nfa& nfa, const ByteClasses& cls, int max_states) {
  Dfa d;
  d.n_classes = cls.count;
  const size_t nn = nfa.states.size();
  std::vector<uint32_t> mark(nn, 0);
  uint32_t stamp = 0;

  // Ordered closure: depth-first in priority order; stops at the first MATCH,
  // dropping every lower-priority thread.  Returns true if a MATCH was reached.
  auto closure_ordered = [&](int start, std::vector<uint32_t>& out, bool& matched) {
    std::vector<int> st{start};
    while (!st.empty() && !matched) {
      int q = st.back();
      st.pop_back();
      if (mark[(size_t)q] == stamp) continue;
      mark[(size_t)q] = stamp;
      const NfaState& s = nfa.states[(size_t)q];
      switch (s.kind) {
        case NfaState::CONSUME: out.push_back((uint32_t)q); break;
        case NfaState::MATCH: matched = true; break;
        case NfaState::SPLIT: st.push_back(s.b); st.push_back(s.a); break;
        case NfaState::EPS: st.push_back(s.a); break;
        case NfaState::ASSERT: throw CompileError("assertion in a DFA without contexts");
      }
    }
  };

  std::unordered_map<std::vector<uint32_t>, uint32_t, VecHash> index;
  std::vector<std::vector<uint32_t>> sets;
  std::vector<uint8_t> matchf;
  auto intern = [&](std::vector<uint32_t>&& key, bool m) -> uint32_t {
    std::vector<uint32_t> k = key;
    k.push_back(m ? 1u : 0u);
    auto it = index.find(k);
    if (it != index.end()) return it->second;
    uint32_t id = (uint32_t)sets.size();
    index.emplace(std::move(k), id);
    sets.push_back(std::move(key));
    matchf.push_back(m ? 1 : 0);
    return id;
  };
  intern({}, false);  // dead
  {
    ++stamp;
    std::vector<uint32_t> s0;
    bool m0 = false;
    for (int s : nfa.starts) closure_ordered(s, s0, m0);
    d.start_anchored = intern(std::move(s0), m0);
  }
  const int C = cls.count;
  for (size_t cur = 0; cur < sets.size(); ++cur) {
    if ((int)sets.size() > max_states) { d.too_big = true; return d; }
    d.trans.resize((cur + 1) * (size_t)C, 0);
    if (cur == 0) continue;
    for (int c = 0; c < C; ++c) {
      uint8_t b = cls.representative[(size_t)c];
      ++stamp;
      std::vector<uint32_t> nxt;
      bool m = false;
      for (uint32_t q : sets[cur]) {
        const NfaState& s = nfa.states[q];
        if (!nfa.sets[(size_t)s.set].test(b)) continue;
        closure_ordered(s.a, nxt, m);
        if (m) break;  // lower-priority threads are cut
      }
      uint32_t id = (nxt.empty() && !m) ? 0u : intern(std::move(nxt), m);
      d.trans[cur * (size_t)C + (size_t)c] = id;
    }
  }
  d.n_states = (int)sets.size();
  d.is_match.assign(matchf.begin(), matchf.end());
  d.match_ptr.assign((size_t)d.n_states + 1, 0);
  for (auto& w : d.trans) {
    uint32_t t = w;
    w = t | (d.is_match[t] ? DFA_FLAG_MATCH : 0u) | (t == 0 ? DFA_FLAG_DEAD : 0u);
  }
  return d;
}

namespace {

// Context of a byte class (the classes of a context DFA separate contexts).
int class_context(const ByteClasses& cls, int c) { return byte_context(cls.representative[(size_t)c]); }

// Epsilon closure under the contexts (left, right), depth-first in priority
// order: SPLIT, EPS and holding ASSERT edges are followed, CONSUME and MATCH
// states collected in the order reached.  With `first_match`, stops at the
// first MATCH (the leftmost-first cut) and reports it in `matched`.
void closure_ctx(const Nfa& nfa, int start, int left, int right, std::vector<uint32_t>& mark, uint32_t stamp,
                 std::vector<uint32_t>& out, bool first_match, bool& matched) {
  std::vector<int> st{start};
  while (!st.empty() && !(first_match && matched)) {
    const int q = st.back();
    st.pop_back();
    if (mark[(size_t)q] == stamp) continue;
    mark[(size_t)q] = stamp;
    const NfaState& s = nfa.states[(size_t)q];
    switch (s.kind) {
      case NfaState::CONSUME: out.push_back((uint32_t)q); break;
      case NfaState::MATCH:
        if (first_match) matched = true;
        else out.push_back((uint32_t)q);
        break;
      case NfaState::SPLIT: st.push_back(s.b); st.push_back(s.a); break;
      case NfaState::EPS: st.push_back(s.a); break;
      case NfaState::ASSERT:
        if (look_holds(s.look, left, right)) st.push_back(s.a);
        break;
    }
  }
}

// The subset construction shared by both context DFAs.  A state's key is its
// ordered seed list (NFA states whose closure is pending) and left context.
// `step(seeds, left, right_class, next_seeds, match)` computes a transition.
struct ContextBuilder {
  const Nfa& nfa;
  const ByteClasses& cls;
  std::unordered_map<std::vector<uint32_t>, uint32_t, VecHash> index;
  std::vector<std::vector<uint32_t>> seeds;
  std::vector<int> left;
  ContextBuilder(const Nfa& n, const ByteClasses& c) : nfa(n), cls(c) {
    intern({}, CTX_BEGIN);  // 0: dead (no seeds)
  }
  uint32_t intern(std::vector<uint32_t>&& key, int ctx) {
    if (key.empty() && !seeds.empty()) return 0;
    std::vector<uint32_t> k = key;
    k.push_back((uint32_t)ctx);
    auto it = index.find(k);
    if (it != index.end()) return it->second;
    const uint32_t id = (uint32_t)seeds.size();
    index.emplace(std::move(k), id);
    seeds.push_back(std::move(key));
    left.push_back(ctx);
    return id;
  }
};

}  // namespace

Dfa build_context_all_dfa(const Nfa& nfa, const ByteClasses& cls, int max_states) {
  Dfa d;
  d.n_classes = cls.count;
  ContextBuilder B(nfa, cls);
  std::vector<uint32_t> starts;
  for (int s : nfa.starts) starts.push_back((uint32_t)s);
  for (int k = 0; k < 4; ++k) d.ctx_start[k] = B.intern(std::vector<uint32_t>(starts), k);
  d.start_anchored = d.ctx_start[CTX_BEGIN];
  std::vector<uint32_t> mark(nfa.states.size(), 0);
  uint32_t stamp = 0;
  const int C = cls.count;
  // patterns matching at a state's position, per right context
  std::vector<std::vector<uint32_t>> lists;
  auto closure = [&](uint32_t cur, int right, std::vector<uint32_t>& out) {
    ++stamp;
    out.clear();
    bool unused = false;
    for (uint32_t q : B.seeds[cur]) closure_ctx(nfa, (int)q, B.left[cur], right, mark, stamp, out, false, unused);
  };
  std::vector<uint32_t> cl, nxt;
  for (size_t cur = 0; cur < B.seeds.size(); ++cur) {
    if ((int)B.seeds.size() > max_states) { d.too_big = true; return d; }
    d.trans.resize((cur + 1) * (size_t)C, 0);
    lists.resize((cur + 1) * 4);
    for (int k = 0; k < 4; ++k) {
      closure((uint32_t)cur, k, cl);
      std::vector<uint32_t> pats;
      for (uint32_t q : cl)
        if (nfa.states[q].kind == NfaState::MATCH) pats.push_back((uint32_t)nfa.states[q].pattern);
      std::sort(pats.begin(), pats.end());
      pats.erase(std::unique(pats.begin(), pats.end()), pats.end());
      lists[cur * 4 + (size_t)k] = std::move(pats);
    }
    if (cur == 0) continue;
    for (int c = 0; c < C; ++c) {
      const int right = class_context(cls, c);
      const uint8_t b = cls.representative[(size_t)c];
      closure((uint32_t)cur, right, cl);
      nxt.clear();
      for (uint32_t q : cl) {
        const NfaState& s = nfa.states[q];
        if (s.kind == NfaState::CONSUME && nfa.sets[(size_t)s.set].test(b)) nxt.push_back((uint32_t)s.a);
      }
      std::sort(nxt.begin(), nxt.end());
      nxt.erase(std::unique(nxt.begin(), nxt.end()), nxt.end());
      const uint32_t id = B.intern(std::vector<uint32_t>(nxt), right);
      d.trans[cur * (size_t)C + (size_t)c] =
          id | (lists[cur * 4 + (size_t)right].empty() ? 0u : DFA_FLAG_MATCH) | (id == 0 ? DFA_FLAG_DEAD : 0u);
    }
  }
  d.n_states = (int)B.seeds.size();
  d.is_match.assign((size_t)d.n_states, 0);
  d.match_ptr.assign(4 * (size_t)d.n_states + 1, 0);
  for (size_t j = 0; j < 4 * (size_t)d.n_states; ++j) {
    d.match_ptr[j] = (uint32_t)d.match_list.size();
    d.match_list.insert(d.match_list.end(), lists[j].begin(), lists[j].end());
    if (!lists[j].empty()) d.is_match[j / 4] = 1;
  }
  d.match_ptr[4 * (size_t)d.n_states] = (uint32_t)d.match_list.size();
  return d;
}

Dfa build_context_lf_dfa(const Nfa& nfa, const ByteClasses& cls, int max_states) {
  Dfa d;
  d.n_classes = cls.count;
  ContextBuilder B(nfa, cls);
  std::vector<uint32_t> starts;
  for (int s : nfa.starts) starts.push_back((uint32_t)s);
  for (int k = 0; k < 4; ++k) d.ctx_start[k] = B.intern(std::vector<uint32_t>(starts), k);
  d.start_anchored = d.ctx_start[CTX_BEGIN];
  std::vector<uint32_t> mark(nfa.states.size(), 0);
  uint32_t stamp = 0;
  const int C = cls.count;
  // ordered closure of a state's seeds under a right context: the threads in
  // priority order up to the first match (which cuts the rest)
  auto closure = [&](uint32_t cur, int right, std::vector<uint32_t>& out, bool& matched) {
    ++stamp;
    out.clear();
    matched = false;
    for (uint32_t q : B.seeds[cur]) {
      closure_ctx(nfa, (int)q, B.left[cur], right, mark, stamp, out, true, matched);
      if (matched) break;
    }
  };
  std::vector<uint32_t> cl, nxt;
  std::vector<uint8_t> end_match;
  for (size_t cur = 0; cur < B.seeds.size(); ++cur) {
    if ((int)B.seeds.size() > max_states) { d.too_big = true; return d; }
    d.trans.resize((cur + 1) * (size_t)C, 0);
    bool m_end = false;
    closure((uint32_t)cur, CTX_BEGIN, cl, m_end);
    end_match.push_back(m_end ? 1 : 0);
    if (cur == 0) continue;
    for (int c = 0; c < C; ++c) {
      const int right = class_context(cls, c);
      const uint8_t b = cls.representative[(size_t)c];
      bool m = false;
      closure((uint32_t)cur, right, cl, m);
      nxt.clear();
      for (uint32_t q : cl) {  // successors in priority order, first occurrence kept
        const NfaState& s = nfa.states[q];
        if (!nfa.sets[(size_t)s.set].test(b)) continue;
        if (std::find(nxt.begin(), nxt.end(), (uint32_t)s.a) == nxt.end()) nxt.push_back((uint32_t)s.a);
      }
      const uint32_t id = B.intern(std::vector<uint32_t>(nxt), right);
      d.trans[cur * (size_t)C + (size_t)c] = id | (m ? DFA_FLAG_MATCH : 0u) | (id == 0 ? DFA_FLAG_DEAD : 0u);
    }
  }
  d.n_states = (int)B.seeds.size();
  d.is_match.assign(end_match.begin(), end_match.end());
  d.match_ptr.assign((size_t)d.n_states + 1, 0);
  return d;
}

void renumber_dfa(Dfa& d, const std::vector<uint32_t>& order) {
  const int n = d.n_states, C = d.n_classes;
  std::vector<uint32_t> inv((size_t)n);
  for (int k = 0; k < n; ++k) inv[order[(size_t)k]] = (uint32_t)k;
  std::vector<uint32_t> trans((size_t)n * C);
  std::vector<uint8_t> ism((size_t)n);
  std::vector<uint32_t> mptr((size_t)n + 1);
  std::vector<uint32_t> mlist;
  for (int k = 0; k < n; ++k) {
    uint32_t old = order[(size_t)k];
    ism[(size_t)k] = d.is_match[old];
    mptr[(size_t)k] = (uint32_t)mlist.size();
    if (!d.match_ptr.empty())
      for (uint32_t j = d.match_ptr[old]; j < d.match_ptr[old + 1]; ++j) mlist.push_back(d.match_list[j]);
    for (int c = 0; c < C; ++c) {
      uint32_t w = d.trans[(size_t)old * C + c];
      trans[(size_t)k * C + c] = inv[w & DFA_MASK_STATE] | (w & ~DFA_MASK_STATE);
    }
  }
  mptr[(size_t)n] = (uint32_t)mlist.size();
  d.trans.swap(trans);
  d.is_match.swap(ism);
  d.match_ptr.swap(mptr);
  d.match_list.swap(mlist);
  d.start_anchored = inv[d.start_anchored];
  d.start_unanchored = inv[d.start_unanchored];
}

}  // namespace ws
