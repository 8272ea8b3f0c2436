// warpstate oracle -- CPU restatement of the reference's matching semantics.
// TEST INFRASTRUCTURE ONLY (see oracle.h for what is restated and from where).
#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <bitset>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>
#include <unordered_map>

namespace {

constexpr uint32_t FNV_BASIS = 2166136261u;
constexpr uint32_t FNV_PRIME = 16777619u;

int resolve_threads(int n) {
  if (n > 0) return n;
  unsigned h = std::thread::hardware_concurrency();
  return h ? (int)h : 1;
}

// ---------------------------------------------------------------- regex AST
// Mirrors the shape regex-syntax's HIR gives the reference (case folding turns
// letters into two-byte classes; a one-byte class is a literal byte).
enum class K { Set, Concat, Alt, Repeat, Group, Assert, Empty };
enum AssertKind { A_LINE_START, A_LINE_END, A_TEXT_START, A_TEXT_END, A_WORD, A_NOT_WORD };

struct Node {
  K kind;
  std::bitset<256> set;
  std::vector<int> kids;
  int min = 0, max = -1;
  bool greedy = true;
  int akind = 0;
};

struct Flags {
  bool i = false;   // ASCII case-insensitive
  bool m = true;    // multi_line(true) is the reference's builder default
  bool s = false;   // dot matches \n
  bool U = false;   // swap greed
};

struct ParseError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

struct Parser {
  const std::string& p;
  size_t i = 0;
  std::vector<Node> nodes;
  explicit Parser(const std::string& s) : p(s) {}

  int add(Node n) { nodes.push_back(std::move(n)); return (int)nodes.size() - 1; }
  bool eof() const { return i >= p.size(); }
  char peek() const { return p[i]; }

  static void fold(std::bitset<256>& s) {
    for (int c = 'a'; c <= 'z'; ++c) {
      if (s[c] || s[c - 32]) { s[c] = true; s[c - 32] = true; }
    }
  }
  int set_node(std::bitset<256> s, const Flags& f) {
    if (f.i) fold(s);
    Node n; n.kind = K::Set; n.set = s; return add(n);
  }

  int parse_alt(Flags& f) {
    std::vector<int> alts;
    alts.push_back(parse_concat(f));
    while (!eof() && peek() == '|') {
      ++i;
      alts.push_back(parse_concat(f));
    }
    if (alts.size() == 1) return alts[0];
    Node n; n.kind = K::Alt; n.kids = alts; return add(n);
  }

  int parse_concat(Flags& f) {
    std::vector<int> items;
    while (!eof() && peek() != '|' && peek() != ')') {
      int a = parse_atom(f);
      if (a < 0) continue;  // flag-only group
      a = parse_quants(a, f);
      items.push_back(a);
    }
    if (items.empty()) { Node n; n.kind = K::Empty; return add(n); }
    if (items.size() == 1) return items[0];
    Node n; n.kind = K::Concat; n.kids = items; return add(n);
  }

  bool parse_uint(int& v) {
    size_t st = i; long long x = 0;
    while (!eof() && isdigit((unsigned char)peek())) { x = x * 10 + (peek() - '0'); ++i; if (x > 100000) throw ParseError("repetition count too large"); }
    v = (int)x;
    return i > st;
  }

  int parse_quants(int a, Flags& f) {
    bool quantified = false;
    while (!eof()) {
      char c = peek();
      int mn, mx;
      if (c == '*') { mn = 0; mx = -1; ++i; }
      else if (c == '+') { mn = 1; mx = -1; ++i; }
      else if (c == '?') { mn = 0; mx = 1; ++i; }
      else if (c == '{') {
        size_t save = i; ++i;
        int a1 = 0, a2 = 0;
        if (!parse_uint(a1)) { i = save; throw ParseError("invalid repetition"); }
        if (!eof() && peek() == ',') {
          ++i;
          if (!eof() && peek() == '}') { mn = a1; mx = -1; }
          else { if (!parse_uint(a2)) throw ParseError("invalid repetition"); mn = a1; mx = a2; }
        } else { mn = a1; mx = a1; }
        if (eof() || peek() != '}') throw ParseError("unclosed repetition");
        ++i;
        if (mx >= 0 && mx < mn) throw ParseError("invalid repetition range");
      } else break;
      if (quantified) throw ParseError("repetition operator missing expression");
      if (nodes[a].kind == K::Empty) throw ParseError("repetition operator missing expression");
      bool greedy = true;
      if (!eof() && peek() == '?') { greedy = false; ++i; }
      if (f.U) greedy = !greedy;
      Node n; n.kind = K::Repeat; n.kids = {a}; n.min = mn; n.max = mx; n.greedy = greedy;
      a = add(n);
      quantified = true;
    }
    return a;
  }

  static int hexval(char c) {
    if (c >= '0' && c <= '9') return c - '0';
    if (c >= 'a' && c <= 'f') return c - 'a' + 10;
    if (c >= 'A' && c <= 'F') return c - 'A' + 10;
    return -1;
  }

  // Parses an escape after '\'.  Returns: 0 = single byte in *b, 1 = class in *s,
  // 2 = assertion in *ak.
  int parse_escape(int* b, std::bitset<256>* s, int* ak, bool in_class) {
    if (eof()) throw ParseError("incomplete escape");
    char c = p[i++];
    auto digit = [] { std::bitset<256> r; for (int x = '0'; x <= '9'; ++x) r[x] = true; return r; };
    auto word = [&] { std::bitset<256> r = digit(); for (int x = 'a'; x <= 'z'; ++x) { r[x] = true; r[x - 32] = true; } r['_'] = true; return r; };
    auto space = [] { std::bitset<256> r; for (int x : {'\t', '\n', '\v', '\f', '\r', ' '}) r[x] = true; return r; };
    switch (c) {
      case 'd': *s = digit(); return 1;
      case 'D': *s = ~digit(); return 1;
      case 'w': *s = word(); return 1;
      case 'W': *s = ~word(); return 1;
      case 's': *s = space(); return 1;
      case 'S': *s = ~space(); return 1;
      case 'n': *b = '\n'; return 0;
      case 't': *b = '\t'; return 0;
      case 'r': *b = '\r'; return 0;
      case 'f': *b = '\f'; return 0;
      case 'v': *b = '\v'; return 0;
      case 'a': *b = 7; return 0;
      case 'e': *b = 27; return 0;
      case 'x': {
        int v = 0;
        if (!eof() && peek() == '{') {
          ++i; int nd = 0;
          while (!eof() && peek() != '}') { int h = hexval(p[i++]); if (h < 0) throw ParseError("bad hex"); v = v * 16 + h; if (++nd > 8) throw ParseError("bad hex"); }
          if (eof()) throw ParseError("bad hex");
          ++i;
          if (nd == 0) throw ParseError("bad hex");
        } else {
          if (i + 2 > p.size()) throw ParseError("bad hex");
          int h1 = hexval(p[i]), h2 = hexval(p[i + 1]);
          if (h1 < 0 || h2 < 0) throw ParseError("bad hex");
          v = h1 * 16 + h2; i += 2;
        }
        if (v > 255) throw ParseError("non-byte hex escape with unicode disabled");
        *b = v; return 0;
      }
      case 'b': if (in_class) throw ParseError("\\b in class"); *ak = A_WORD; return 2;
      case 'B': if (in_class) throw ParseError("\\B in class"); *ak = A_NOT_WORD; return 2;
      case 'A': if (in_class) throw ParseError("\\A in class"); *ak = A_TEXT_START; return 2;
      case 'z': if (in_class) throw ParseError("\\z in class"); *ak = A_TEXT_END; return 2;
      case 'p': case 'P': throw ParseError("unicode classes disabled");
      default:
        if ((unsigned char)c < 128 && !isalnum((unsigned char)c)) { *b = (unsigned char)c; return 0; }
        throw ParseError(std::string("unrecognized escape \\") + c);
    }
  }

  bool parse_posix(std::bitset<256>& out) {
    // at "[:" inside a class
    static const char* names[] = {"alnum", "alpha", "ascii", "blank", "cntrl", "digit", "graph", "lower", "print", "punct", "space", "upper", "word", "xdigit"};
    size_t save = i;
    if (p.compare(i, 2, "[:") != 0) return false;
    size_t j = i + 2; bool neg = false;
    if (j < p.size() && p[j] == '^') { neg = true; ++j; }
    size_t e = p.find(":]", j);
    if (e == std::string::npos) return false;
    std::string nm = p.substr(j, e - j);
    std::bitset<256> r;
    bool ok = false;
    for (auto n : names) if (nm == n) ok = true;
    if (!ok) { i = save; return false; }
    for (int c = 0; c < 256; ++c) {
      bool in = false;
      if (nm == "alnum") in = isalnum(c) && c < 128;
      else if (nm == "alpha") in = isalpha(c) && c < 128;
      else if (nm == "ascii") in = c < 128;
      else if (nm == "blank") in = c == ' ' || c == '\t';
      else if (nm == "cntrl") in = c < 32 || c == 127;
      else if (nm == "digit") in = c >= '0' && c <= '9';
      else if (nm == "graph") in = c >= 33 && c <= 126;
      else if (nm == "lower") in = c >= 'a' && c <= 'z';
      else if (nm == "print") in = c >= 32 && c <= 126;
      else if (nm == "punct") in = (c >= 33 && c <= 47) || (c >= 58 && c <= 64) || (c >= 91 && c <= 96) || (c >= 123 && c <= 126);
      else if (nm == "space") in = c == ' ' || (c >= 9 && c <= 13);
      else if (nm == "upper") in = c >= 'A' && c <= 'Z';
      else if (nm == "word") in = (c >= '0' && c <= '9') || (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || c == '_';
      else if (nm == "xdigit") in = (c >= '0' && c <= '9') || (c >= 'a' && c <= 'f') || (c >= 'A' && c <= 'F');
      r[c] = in;
    }
    out = neg ? ~r : r;
    i = e + 2;
    return true;
  }

  // class item: returns a byte value, or -1 when *set holds a class.
  int class_atom(std::bitset<256>* set) {
    if (eof()) throw ParseError("unclosed class");
    unsigned char c = (unsigned char)p[i];
    if (c == '\\') {
      ++i; int b = 0, ak = 0;
      int k = parse_escape(&b, set, &ak, true);
      if (k == 0) return b;
      return -1;
    }
    if (c >= 128) throw ParseError("non-ASCII character in class with unicode disabled");
    ++i;
    return c;
  }

  std::bitset<256> parse_class(const Flags& f) {
    // after '['
    bool neg = false;
    if (!eof() && peek() == '^') { neg = true; ++i; }
    std::bitset<256> acc;
    bool first = true;
    while (true) {
      if (eof()) throw ParseError("unclosed class");
      char c = peek();
      if (c == ']' && !first) { ++i; break; }
      first = false;
      if (c == '[') {
        std::bitset<256> pos;
        if (parse_posix(pos)) { acc |= pos; continue; }
        ++i;
        acc |= parse_class(f);  // nested class union
        continue;
      }
      if (p.compare(i, 2, "&&") == 0 || p.compare(i, 2, "--") == 0 || p.compare(i, 2, "~~") == 0)
        throw ParseError("class set operations are not supported");
      std::bitset<256> s;
      int lo = class_atom(&s);
      if (lo < 0) { acc |= s; continue; }
      if (!eof() && peek() == '-' && i + 1 < p.size() && p[i + 1] != ']') {
        ++i;
        std::bitset<256> s2;
        int hi = class_atom(&s2);
        if (hi < 0) throw ParseError("invalid class range");
        if (hi < lo) throw ParseError("invalid class range");
        for (int x = lo; x <= hi; ++x) acc[x] = true;
      } else {
        acc[lo] = true;
      }
    }
    if (f.i) fold(acc);
    if (neg) acc = ~acc;
    return acc;
  }

  void parse_flags(Flags& f, bool* has_colon) {
    bool negate = false;
    while (!eof()) {
      char c = p[i++];
      if (c == ':') { *has_colon = true; return; }
      if (c == ')') { *has_colon = false; return; }
      if (c == '-') { if (negate) throw ParseError("bad flags"); negate = true; continue; }
      bool v = !negate;
      if (c == 'i') f.i = v;
      else if (c == 'm') f.m = v;
      else if (c == 's') f.s = v;
      else if (c == 'U') f.U = v;
      else if (c == 'u') { if (v) throw ParseError("unicode mode disabled"); }
      else if (c == 'x') { if (v) throw ParseError("verbose mode is not supported"); }
      else if (c == 'R') { /* CRLF mode: no effect on the supported grammar */ if (v) throw ParseError("CRLF mode is not supported"); }
      else throw ParseError("unknown flag");
    }
    throw ParseError("unclosed group");
  }

  int parse_atom(Flags& f) {
    char c = p[i];
    if (c == '(') {
      ++i;
      bool capture = true;
      Flags inner = f;
      if (!eof() && peek() == '?') {
        ++i;
        if (!eof() && peek() == 'P' && i + 1 < p.size() && p[i + 1] == '<') { i += 2; size_t e = p.find('>', i); if (e == std::string::npos) throw ParseError("bad group name"); i = e + 1; }
        else if (!eof() && peek() == '<') { ++i; size_t e = p.find('>', i); if (e == std::string::npos) throw ParseError("bad group name"); i = e + 1; }
        else {
          bool colon = false;
          parse_flags(inner, &colon);
          if (!colon) { f = inner; return -1; }  // (?flags) applies to the rest of the group
          capture = false;
        }
      }
      int a = parse_alt(inner);
      if (eof() || peek() != ')') throw ParseError("unclosed group");
      ++i;
      Node n; n.kind = K::Group; n.kids = {a}; n.akind = capture ? 1 : 0;
      return add(n);
    }
    if (c == ')') throw ParseError("unopened group");
    if (c == '[') {
      ++i;
      std::bitset<256> s = parse_class(f);
      Node n; n.kind = K::Set; n.set = s; return add(n);
    }
    if (c == '.') {
      ++i;
      std::bitset<256> s; s.set();
      if (!f.s) s['\n'] = false;
      Node n; n.kind = K::Set; n.set = s; return add(n);
    }
    if (c == '^' || c == '$') {
      ++i;
      Node n; n.kind = K::Assert;
      n.akind = (c == '^') ? (f.m ? A_LINE_START : A_TEXT_START) : (f.m ? A_LINE_END : A_TEXT_END);
      return add(n);
    }
    if (c == '*' || c == '+' || c == '?') throw ParseError("repetition operator missing expression");
    if (c == '\\') {
      ++i;
      int b = 0, ak = 0; std::bitset<256> s;
      int k = parse_escape(&b, &s, &ak, false);
      if (k == 0) { std::bitset<256> one; one[b] = true; return set_node(one, f); }
      if (k == 1) { Node n; n.kind = K::Set; n.set = s; return add(n); }
      Node n; n.kind = K::Assert; n.akind = ak; return add(n);
    }
    unsigned char uc = (unsigned char)c;
    if (uc >= 128) {
      // a UTF-8 encoded character outside a class matches its byte sequence
      int len = (uc >= 0xF0) ? 4 : (uc >= 0xE0) ? 3 : (uc >= 0xC0) ? 2 : 1;
      std::vector<int> items;
      for (int k = 0; k < len && !eof(); ++k) {
        std::bitset<256> one; one[(unsigned char)p[i++]] = true;
        Node n; n.kind = K::Set; n.set = one; items.push_back(add(n));
      }
      if (items.size() == 1) return items[0];
      Node n; n.kind = K::Concat; n.kids = items; return add(n);
    }
    ++i;
    std::bitset<256> one; one[uc] = true;
    return set_node(one, f);
  }

  int parse() {
    Flags f;
    int r = parse_alt(f);
    if (!eof()) throw ParseError("unopened group");
    return r;
  }
};

// -------------------------------------------------- literal / pathological
bool literal_of(const std::vector<Node>& N, int id, std::vector<uint8_t>& out) {
  const Node& n = N[id];
  switch (n.kind) {
    case K::Set:
      if (n.set.count() != 1) return false;
      for (int c = 0; c < 256; ++c) if (n.set[c]) out.push_back((uint8_t)c);
      return true;
    case K::Concat: {
      // regex-syntax drops empty items from a concatenation
      bool any = false;
      for (int k : n.kids) {
        if (N[k].kind == K::Empty) continue;
        if (!literal_of(N, k, out)) return false;
        any = true;
      }
      return any;
    }
    case K::Group:
      return literal_of(N, n.kids[0], out);
    default:
      return false;
  }
}

bool has_rep(const std::vector<Node>& N, int id) {
  const Node& n = N[id];
  switch (n.kind) {
    case K::Repeat: return true;
    case K::Concat: case K::Alt:
      for (int k : n.kids) if (has_rep(N, k)) return true;
      return false;
    case K::Group: return has_rep(N, n.kids[0]);
    default: return false;
  }
}

bool pathological(const std::vector<Node>& N, int id) {
  const Node& n = N[id];
  switch (n.kind) {
    case K::Repeat: {
      bool outer_unbounded = n.max < 0 || n.max > 1;
      if (outer_unbounded && has_rep(N, n.kids[0])) return true;
      return pathological(N, n.kids[0]);
    }
    case K::Concat: case K::Alt:
      for (int k : n.kids) if (pathological(N, k)) return true;
      return false;
    case K::Group: return pathological(N, n.kids[0]);
    default: return false;
  }
}

// ------------------------------------------------------------- program
enum Op : uint8_t { I_SET, I_SPLIT, I_JMP, I_ASSERT, I_MATCH };
struct Inst { Op op; int x = 0, y = 0; };

struct Program {
  std::vector<Inst> code;
  std::vector<std::bitset<256>> sets;
  int maxlen = -1;  // -1 = unbounded
  bool nullable = false;
  bool has_assert = false;
  std::vector<uint64_t> pair_ok;  // 65536 bits: (b0,b1) may begin a match
  std::bitset<256> first;         // b0 may begin a match
  std::bitset<256> one_byte;      // b0 alone is a complete match
  // every match is at least prefix_len (8) bytes long and begins with
  // one of these (little-endian), when there are few enough to list
  int prefix_len = 0;
  std::vector<uint64_t> prefixes;
};

struct Compiler {
  const std::vector<Node>& N;
  Program& P;
  Compiler(const std::vector<Node>& n, Program& p) : N(n), P(p) {}
  int emit(Op op, int x = 0, int y = 0) { P.code.push_back({op, x, y}); return (int)P.code.size() - 1; }

  void gen(int id) {
    const Node& n = N[id];
    switch (n.kind) {
      case K::Set: { P.sets.push_back(n.set); emit(I_SET, (int)P.sets.size() - 1); break; }
      case K::Empty: break;
      case K::Group: gen(n.kids[0]); break;
      case K::Concat: for (int k : n.kids) gen(k); break;
      case K::Assert: P.has_assert = true; emit(I_ASSERT, n.akind); break;
      case K::Alt: {
        std::vector<int> jumps;
        for (size_t a = 0; a < n.kids.size(); ++a) {
          if (a + 1 < n.kids.size()) {
            int sp = emit(I_SPLIT);
            P.code[sp].x = sp + 1;
            gen(n.kids[a]);
            jumps.push_back(emit(I_JMP));
            P.code[sp].y = (int)P.code.size();
          } else {
            gen(n.kids[a]);
          }
        }
        for (int j : jumps) P.code[j].x = (int)P.code.size();
        break;
      }
      case K::Repeat: {
        int sub = n.kids[0];
        for (int r = 0; r < n.min; ++r) gen(sub);
        if (n.max < 0) {
          int sp = emit(I_SPLIT);
          int body = (int)P.code.size();
          gen(sub);
          emit(I_JMP, sp);
          int out = (int)P.code.size();
          if (n.greedy) { P.code[sp].x = body; P.code[sp].y = out; }
          else { P.code[sp].x = out; P.code[sp].y = body; }
        } else {
          std::vector<int> splits;
          for (int r = n.min; r < n.max; ++r) {
            int sp = emit(I_SPLIT);
            splits.push_back(sp);
            P.code[sp].x = (int)P.code.size();  // provisional: body
            gen(sub);
          }
          int out = (int)P.code.size();
          for (int sp : splits) {
            int body = sp + 1;
            if (n.greedy) { P.code[sp].x = body; P.code[sp].y = out; }
            else { P.code[sp].x = out; P.code[sp].y = body; }
          }
        }
        break;
      }
    }
  }
};

// max match length (-1 unbounded) and nullability from the AST
void lengths(const std::vector<Node>& N, int id, long long& mn, long long& mx) {
  const Node& n = N[id];
  switch (n.kind) {
    case K::Set: mn = 1; mx = 1; return;
    case K::Empty: case K::Assert: mn = 0; mx = 0; return;
    case K::Group: lengths(N, n.kids[0], mn, mx); return;
    case K::Concat: {
      mn = 0; mx = 0;
      for (int k : n.kids) {
        long long a, b; lengths(N, k, a, b);
        mn += a;
        if (mx < 0 || b < 0) mx = -1; else mx += b;
      }
      return;
    }
    case K::Alt: {
      mn = -2; mx = 0;
      for (int k : n.kids) {
        long long a, b; lengths(N, k, a, b);
        mn = (mn == -2) ? a : std::min(mn, a);
        if (mx < 0 || b < 0) mx = -1; else mx = std::max(mx, b);
      }
      return;
    }
    case K::Repeat: {
      long long a, b; lengths(N, n.kids[0], a, b);
      mn = a * n.min;
      if (n.max < 0) mx = (b == 0) ? 0 : -1;
      else if (b < 0) mx = -1;
      else mx = b * n.max;
      return;
    }
  }
}

// epsilon closure for the prefix analysis (assertions pass: over-approximation)
void closure(const Program& P, int pc, std::vector<char>& seen, std::vector<int>& out, bool& match) {
  std::vector<int> st{pc};
  while (!st.empty()) {
    int q = st.back(); st.pop_back();
    if (seen[q]) continue;
    seen[q] = 1;
    const Inst& in = P.code[q];
    switch (in.op) {
      case I_SET: out.push_back(q); break;
      case I_SPLIT: st.push_back(in.y); st.push_back(in.x); break;
      case I_JMP: st.push_back(in.x); break;
      case I_ASSERT: st.push_back(q + 1); break;
      case I_MATCH: match = true; break;
    }
  }
}

void analyze_prefixes(Program& P) {
  size_t n = P.code.size();
  std::vector<char> seen(n, 0);
  std::vector<int> s0; bool m0 = false;
  closure(P, 0, seen, s0, m0);
  P.pair_ok.assign(65536 / 64, 0);
  for (int b0 = 0; b0 < 256; ++b0) {
    std::vector<char> seen1(n, 0);
    std::vector<int> s1; bool m1 = false;
    bool any = false;
    for (int q : s0) {
      if (P.sets[P.code[q].x][b0]) { any = true; closure(P, q + 1, seen1, s1, m1); }
    }
    if (!any) continue;
    P.first[b0] = true;
    if (m1) P.one_byte[b0] = true;
    for (int b1 = 0; b1 < 256; ++b1) {
      bool ok = m1;
      if (!ok) for (int q : s1) if (P.sets[P.code[q].x][b1]) { ok = true; break; }
      if (ok) { size_t key = (size_t)b0 << 8 | b1; P.pair_ok[key >> 6] |= 1ull << (key & 63); }
    }
  }
}

// The first K bytes of every match (K = 8 here), listed when the regex
// matches nothing shorter than K bytes and the prefixes number at most
// kMaxPrefixes (assertions pass here: an over-approximation, as for the pair
// index).  Used only to skip start positions where no match can begin.
constexpr size_t kMaxPrefixes = 4096;
bool list_prefixes(const Program& P, int K, std::vector<uint64_t>& out) {
  const size_t n = P.code.size();
  struct Prefix { uint64_t bytes; std::vector<int> pcs; };
  std::vector<Prefix> cur;
  {
    std::vector<char> seen(n, 0);
    std::vector<int> s0;
    bool m0 = false;
    closure(P, 0, seen, s0, m0);
    if (m0) return false;
    cur.push_back({0ull, s0});
  }
  for (int depth = 0; depth < K; ++depth) {
    std::vector<Prefix> nxt;
    for (const Prefix& pf : cur) {
      std::bitset<256> can;
      for (int q : pf.pcs) can |= P.sets[P.code[q].x];
      for (int b = 0; b < 256; ++b) {
        if (!can[b]) continue;
        std::vector<char> seen(n, 0);
        std::vector<int> s1;
        bool m1 = false, any = false;
        for (int q : pf.pcs)
          if (P.sets[P.code[q].x][b]) { any = true; closure(P, q + 1, seen, s1, m1); }
        if (!any) continue;
        if (m1 && depth < K - 1) return false;  // a match shorter than K bytes
        nxt.push_back({pf.bytes | ((uint64_t)b << (8 * depth)), s1});
        if (nxt.size() > kMaxPrefixes) return false;
      }
    }
    cur.swap(nxt);
  }
  for (const Prefix& pf : cur) out.push_back(pf.bytes);
  std::sort(out.begin(), out.end());
  return true;
}

void analyze_long_prefixes(Program& P) {
  if (P.nullable || P.has_assert) return;
  std::vector<uint64_t> v;
  if (list_prefixes(P, 8, v)) {
    P.prefix_len = 8;
    P.prefixes.swap(v);
  }
}

inline bool is_word(uint8_t c) {
  return (c >= '0' && c <= '9') || (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || c == '_';
}

bool assert_holds(int k, const uint8_t* d, uint64_t len, uint64_t pos) {
  switch (k) {
    case A_LINE_START: return pos == 0 || d[pos - 1] == '\n';
    case A_LINE_END: return pos == len || d[pos] == '\n';
    case A_TEXT_START: return pos == 0;
    case A_TEXT_END: return pos == len;
    case A_WORD: case A_NOT_WORD: {
      bool a = pos > 0 && is_word(d[pos - 1]);
      bool b = pos < len && is_word(d[pos]);
      return (k == A_WORD) ? (a != b) : (a == b);
    }
  }
  return false;
}

// Bounded backtracker: leftmost-first end of an anchored match at s, or -1.
struct Backtracker {
  const Program& P;
  std::vector<uint64_t> visited;  // bit (pos - s) * ncode + pc
  std::vector<std::pair<int, uint64_t>> stack;
  explicit Backtracker(const Program& p) : P(p) {}

  int64_t run(const uint8_t* d, uint64_t len, uint64_t s) {
    const size_t nc = P.code.size();
    uint64_t window = len - s;
    if (P.maxlen >= 0 && (uint64_t)P.maxlen < window) window = (uint64_t)P.maxlen;
    uint64_t bits = (window + 1) * nc;
    size_t words = (size_t)((bits + 63) / 64);
    if (visited.size() < words) visited.resize(words);
    uint64_t hi = 0;  // highest pos - s touched
    stack.clear();
    stack.push_back({0, s});
    int64_t result = -1;
    while (!stack.empty() && result < 0) {
      int pc = stack.back().first; uint64_t pos = stack.back().second; stack.pop_back();
      while (true) {
        uint64_t rel = pos - s;
        if (rel > window) break;
        uint64_t key = rel * nc + (uint64_t)pc;
        uint64_t& w = visited[key >> 6];
        uint64_t bit = 1ull << (key & 63);
        if (w & bit) break;
        w |= bit;
        if (rel > hi) hi = rel;
        const Inst& in = P.code[pc];
        if (in.op == I_SET) {
          if (pos < len && P.sets[in.x][d[pos]]) { ++pc; ++pos; continue; }
          break;
        } else if (in.op == I_SPLIT) {
          stack.push_back({in.y, pos});
          pc = in.x;
        } else if (in.op == I_JMP) {
          pc = in.x;
        } else if (in.op == I_ASSERT) {
          if (assert_holds(in.x, d, len, pos)) { ++pc; continue; }
          break;
        } else {  // I_MATCH
          result = (int64_t)pos;
          break;
        }
      }
    }
    uint64_t clear_words = std::min<uint64_t>(words, ((hi + 1) * nc + 63) / 64 + 1);
    std::memset(visited.data(), 0, clear_words * sizeof(uint64_t));
    return result;
  }
};

}  // namespace

struct or_regex {
  std::string pattern;
  Program prog;
};

extern "C" {

uint32_t or_fnv1a(const uint8_t* bytes, size_t len, size_t window) {
  // compiler.rs:343-350 -- iterates bytes.iter().take(window.max(1))
  uint32_t h = FNV_BASIS;
  size_t n = std::min(len, std::max<size_t>(window, 1));
  for (size_t k = 0; k < n; ++k) { h ^= bytes[k]; h *= FNV_PRIME; }
  return h;
}

int or_prefilter_build(const uint32_t* offsets, const uint32_t* hashes, uint32_t n,
                       uint32_t window, uint32_t* prefix_meta,
                       uint32_t* bucket_ranges, uint32_t* n_buckets, uint32_t* entries) {
  // literal_prefilter.rs:23-88
  if (window == 0) return -1;
  std::vector<std::vector<std::pair<uint32_t, uint32_t>>> groups(window);
  for (uint32_t li = 0; li < n; ++li) {
    uint32_t len = offsets[2 * li + 1];
    uint32_t pl = std::max<uint32_t>(std::min(len, window), 1);
    groups[pl - 1].push_back({hashes[li], li});
  }
  std::vector<uint32_t> meta(4 * window, 0);
  std::vector<uint32_t> ranges;
  std::vector<uint32_t> ents;
  for (uint32_t g = 0; g < window; ++g) {
    auto& grp = groups[g];
    if (grp.empty()) continue;
    uint64_t bc = 1;
    while (bc < (uint64_t)grp.size() * 2) bc <<= 1;
    uint32_t off = (uint32_t)(ranges.size() / 2);
    std::vector<std::vector<std::pair<uint32_t, uint32_t>>> buckets(bc);
    for (auto& e : grp) buckets[e.first & (bc - 1)].push_back(e);
    for (auto& b : buckets) {
      ranges.push_back((uint32_t)(ents.size() / 2));
      ranges.push_back((uint32_t)b.size());
      for (auto& e : b) { ents.push_back(e.first); ents.push_back(e.second); }
    }
    meta[4 * g + 0] = off;
    meta[4 * g + 1] = (uint32_t)bc - 1;
    meta[4 * g + 2] = (uint32_t)bc;
    meta[4 * g + 3] = 0;
  }
  *n_buckets = (uint32_t)(ranges.size() / 2);
  if (prefix_meta) std::memcpy(prefix_meta, meta.data(), meta.size() * 4);
  if (bucket_ranges) std::memcpy(bucket_ranges, ranges.data(), ranges.size() * 4);
  if (entries) std::memcpy(entries, ents.data(), ents.size() * 4);
  return 0;
}

uint64_t or_literal_scan(const uint8_t* packed, const uint32_t* offsets,
                         const uint32_t* literal_pattern_ids, uint32_t n_literals,
                         uint32_t window, const uint8_t* data, uint64_t len,
                         or_match* out, uint64_t cap, int nthreads) {
  if (n_literals == 0 || len == 0) return 0;
  std::vector<uint32_t> hashes(n_literals);
  for (uint32_t li = 0; li < n_literals; ++li)
    hashes[li] = or_fnv1a(packed + offsets[2 * li], offsets[2 * li + 1], window);
  std::vector<uint32_t> meta(4 * window);
  uint32_t nb = 0;
  or_prefilter_build(offsets, hashes.data(), n_literals, window, nullptr, nullptr, &nb, nullptr);
  std::vector<uint32_t> ranges(2 * (size_t)nb), ents(2 * (size_t)n_literals);
  or_prefilter_build(offsets, hashes.data(), n_literals, window, meta.data(), ranges.data(), &nb, ents.data());

  int T = resolve_threads(nthreads);
  uint64_t per = (len + T - 1) / T;
  std::vector<std::vector<or_match>> res(T);
  std::vector<std::thread> th;
  for (int t = 0; t < T; ++t) {
    th.emplace_back([&, t] {
      uint64_t a = (uint64_t)t * per, b = std::min(len, a + per);
      auto& r = res[t];
      for (uint64_t pos = a; pos < b; ++pos) {
        // shader.rs:59-98: FNV-1a over up to window bytes, probe at each prefix length
        uint32_t h = FNV_BASIS;
        uint64_t maxp = std::min<uint64_t>(window, len - pos);
        for (uint64_t i = 0; i < maxp; ++i) {
          h = (h ^ data[pos + i]) * FNV_PRIME;
          const uint32_t* m = &meta[4 * i];
          if (m[2] == 0) continue;
          uint32_t bi = m[0] + (h & m[1]);
          uint32_t es = ranges[2 * bi], ec = ranges[2 * bi + 1];
          for (uint32_t e = 0; e < ec; ++e) {
            if (ents[2 * (es + e)] != h) continue;
            uint32_t li = ents[2 * (es + e) + 1];
            uint32_t lo = offsets[2 * li], ll = offsets[2 * li + 1];
            if (pos + ll > len) continue;
            // shader.rs:174-227 exact verify
            if (std::memcmp(data + pos, packed + lo, ll) == 0)
              r.push_back({literal_pattern_ids[li], (uint32_t)pos, (uint32_t)(pos + ll)});
          }
        }
      }
    });
  }
  for (auto& x : th) x.join();
  uint64_t total = 0;
  for (auto& r : res) {
    for (auto& m : r) { if (total < cap) out[total] = m; ++total; }
  }
  return total;
}

or_regex* or_regex_new(const char* pattern, char* err, size_t err_cap) {
  try {
    std::string p(pattern);
    if (p.empty()) throw ParseError("empty pattern");
    Parser ps(p);
    int root = ps.parse();
    auto* r = new or_regex();
    r->pattern = p;
    Compiler c(ps.nodes, r->prog);
    c.gen(root);
    c.emit(I_MATCH);
    long long mn, mx;
    lengths(ps.nodes, root, mn, mx);
    r->prog.maxlen = (int)std::min<long long>(mx, 1 << 30);
    r->prog.nullable = (mn == 0);
    analyze_prefixes(r->prog);
    analyze_long_prefixes(r->prog);
    return r;
  } catch (const std::exception& e) {
    if (err && err_cap) { std::strncpy(err, e.what(), err_cap - 1); err[err_cap - 1] = 0; }
    return nullptr;
  }
}

void or_regex_free(or_regex* r) { delete r; }
int or_regex_nullable(const or_regex* r) { return r->prog.nullable ? 1 : 0; }
long long or_regex_maxlen(const or_regex* r) { return r->prog.maxlen; }

int or_regex_literal(const char* pattern, uint8_t* out, size_t cap, size_t* out_len) {
  try {
    std::string p(pattern);
    Parser ps(p);
    int root = ps.parse();
    std::vector<uint8_t> bytes;
    if (!literal_of(ps.nodes, root, bytes) || bytes.empty()) return 0;
    *out_len = bytes.size();
    if (out) std::memcpy(out, bytes.data(), std::min(cap, bytes.size()));
    return 1;
  } catch (...) {
    return -1;
  }
}

int or_regex_pathological(const char* pattern) {
  try {
    std::string p(pattern);
    Parser ps(p);
    int root = ps.parse();
    return pathological(ps.nodes, root) ? 1 : 0;
  } catch (...) {
    return -1;
  }
}

static void find_iter_one(const or_regex* r, const uint8_t* d, uint64_t len,
                          std::vector<std::pair<uint32_t, uint32_t>>& out) {
  const Program& P = r->prog;
  Backtracker bt(P);
  bool prefilter = !P.nullable && !P.has_assert;
  auto search = [&](uint64_t at, uint64_t& s, uint64_t& e) -> bool {
    for (uint64_t q = at; q <= len; ++q) {
      if (prefilter) {
        if (q >= len) return false;
        if (!P.first[d[q]]) continue;
        if (q + 1 < len) {
          size_t key = (size_t)d[q] << 8 | d[q + 1];
          if (!((P.pair_ok[key >> 6] >> (key & 63)) & 1)) continue;
        }
      }
      int64_t r2 = bt.run(d, len, q);
      if (r2 >= 0) { s = q; e = (uint64_t)r2; return true; }
    }
    return false;
  };
  int64_t last_end = -1;
  uint64_t at = 0;
  while (at <= len) {
    uint64_t s, e;
    if (!search(at, s, e)) break;
    if (s == e && (int64_t)e == last_end) {
      // regex-automata's iterator: an empty match at the end of the previous
      // match is skipped by searching again one position later.
      if (at + 1 > len) break;
      if (!search(at + 1, s, e)) break;
    }
    out.push_back({(uint32_t)s, (uint32_t)e});
    last_end = (int64_t)e;
    at = e;
  }
}

uint64_t or_regex_find_iter(const or_regex* r, const uint8_t* data, uint64_t len,
                            uint32_t* starts, uint32_t* ends, uint64_t cap) {
  std::vector<std::pair<uint32_t, uint32_t>> v;
  find_iter_one(r, data, len, v);
  for (uint64_t k = 0; k < v.size() && k < cap; ++k) { starts[k] = v[k].first; ends[k] = v[k].second; }
  return v.size();
}

uint64_t or_regex_set_scan(or_regex* const* rs, const uint32_t* pattern_ids, uint32_t n,
                           const uint8_t* data, uint64_t len,
                           or_match* out, uint64_t cap, int nthreads) {
  int T = std::max(1, std::min<int>(resolve_threads(nthreads), (int)n));
  std::vector<std::vector<or_match>> res(T);
  std::atomic<uint32_t> next{0};
  std::vector<std::thread> th;
  // at most 32 regexes per block, and a whole number of blocks per thread
  const uint32_t nblocks = ((n + 31) / 32 + (uint32_t)T - 1) / (uint32_t)T * (uint32_t)T;
  const uint32_t BLOCK = std::max<uint32_t>(1, (n + nblocks - 1) / nblocks);
  for (int t = 0; t < T; ++t) {
    th.emplace_back([&, t] {
      // Threads take blocks of regexes; within a block, non-nullable regexes
      // without assertions share one pass over the input driven by an inverted
      // index of their possible first four bytes (or first byte pairs, for
      // regexes whose 4-byte prefixes are not listed); each regex keeps its
      // own find_iter cursor, so results equal per-regex find_iter.
      std::vector<std::pair<uint32_t, uint32_t>> tmp;
      while (true) {
        uint32_t b0 = next.fetch_add(BLOCK);
        if (b0 >= n) break;
        uint32_t b1 = std::min(n, b0 + BLOCK);
        std::vector<uint32_t> simple;
        for (uint32_t k = b0; k < b1; ++k) {
          const Program& P = rs[k]->prog;
          if (P.nullable || P.has_assert) {
            tmp.clear();
            find_iter_one(rs[k], data, len, tmp);
            for (auto& m : tmp) res[t].push_back({pattern_ids[k], m.first, m.second});
          } else {
            simple.push_back(k);
          }
        }
        if (simple.empty()) continue;
        std::vector<std::vector<uint16_t>> index(65536);
        std::vector<std::vector<uint16_t>> last_byte(256);
        // regexes with listed 8-byte prefixes: a 2^20-bit filter of the prefix
        // hashes, then the exact lists
        std::unordered_map<uint64_t, std::vector<uint16_t>> pre_index;
        std::vector<uint64_t> pre_bits((1u << 20) / 64, 0);
        std::vector<uint64_t> pre_pairs(65536 / 64, 0);  // their first two bytes
        auto pre_hash = [](uint64_t x) { return (uint32_t)((x * 0x9E3779B97F4A7C15ull) >> 44); };
        // a listed prefix replaces the pair index only for a regex whose pairs
        // start a search at more than one position in 64 of (a sample of) the
        // input
        const uint64_t sample = std::min<uint64_t>(len, 1u << 20);
        auto pairs_busy = [&](const Program& P) {
          uint64_t hits = 0;
          for (uint64_t q = 0; q + 1 < sample; ++q) {
            const size_t key = (size_t)data[q] << 8 | data[q + 1];
            hits += (P.pair_ok[key >> 6] >> (key & 63)) & 1;
          }
          return hits * 64 > sample;
        };
        for (uint16_t j = 0; j < simple.size(); ++j) {
          const Program& P = rs[simple[j]]->prog;
          if (P.prefix_len && pairs_busy(P)) {
            for (uint64_t x : P.prefixes) {
              pre_index[x].push_back(j);
              const uint32_t h = pre_hash(x);
              pre_bits[h >> 6] |= 1ull << (h & 63);
              const size_t key = (size_t)(x & 0xFF) << 8 | ((x >> 8) & 0xFF);
              pre_pairs[key >> 6] |= 1ull << (key & 63);
            }
            continue;
          }
          for (size_t key = 0; key < 65536; ++key)
            if ((P.pair_ok[key >> 6] >> (key & 63)) & 1) index[key].push_back(j);
          for (int c = 0; c < 256; ++c) if (P.one_byte[c]) last_byte[c].push_back(j);
        }
        std::vector<std::unique_ptr<Backtracker>> bts;
        for (uint32_t k : simple) bts.emplace_back(new Backtracker(rs[k]->prog));
        std::vector<uint64_t> cursor(simple.size(), 0);
        auto attempt = [&](uint16_t j, uint64_t q) {
          if (q < cursor[j]) return;
          int64_t e = bts[j]->run(data, len, q);
          if (e >= 0) {
            res[t].push_back({pattern_ids[simple[j]], (uint32_t)q, (uint32_t)e});
            cursor[j] = (uint64_t)e;
          }
        };
        if (pre_index.empty()) {
          for (uint64_t q = 0; q < len; ++q) {
            const std::vector<uint16_t>* lst;
            if (q + 1 < len) lst = &index[(size_t)data[q] << 8 | data[q + 1]];
            else lst = &last_byte[data[q]];
            for (uint16_t j : *lst) attempt(j, q);
          }
          continue;
        }
        for (uint64_t q = 0; q < len; ++q) {
          if (q + 1 >= len) {
            for (uint16_t j : last_byte[data[q]]) attempt(j, q);
            continue;
          }
          const size_t key = (size_t)data[q] << 8 | data[q + 1];
          for (uint16_t j : index[key]) attempt(j, q);
          if (q + 8 > len || !((pre_pairs[key >> 6] >> (key & 63)) & 1)) continue;
          uint64_t x;
          std::memcpy(&x, data + q, 8);
          const uint32_t h = pre_hash(x);
          if (!((pre_bits[h >> 6] >> (h & 63)) & 1)) continue;
          auto it = pre_index.find(x);
          if (it != pre_index.end())
            for (uint16_t j : it->second) attempt(j, q);
        }
      }
    });
  }
  for (auto& x : th) x.join();
  uint64_t total = 0;
  for (auto& r : res)
    for (auto& m : r) { if (total < cap) out[total] = m; ++total; }
  return total;
}

// scan_batch_cpu (core/src/batch.rs:170-195): every item scanned on its own
// (contract L + contract R inside the item), matches tagged with the item id
// and sorted by (source_id, start, pattern_id, end).  The literal table and
// the regexes' first-byte-pair indexes are built once; items are spread over
// the threads.
uint64_t or_batch_scan(const uint8_t* packed, const uint32_t* offsets, const uint32_t* literal_pattern_ids,
                       uint32_t n_literals, uint32_t window, or_regex* const* rs, const uint32_t* regex_pattern_ids,
                       uint32_t n_regex, const uint8_t* data, const uint64_t* item_off, const uint64_t* item_len,
                       const uint64_t* item_id, uint64_t n_items, or_tagged_match* out, uint64_t cap,
                       int nthreads) {
  // literal prefilter table, as or_literal_scan builds it
  std::vector<uint32_t> hashes(n_literals), meta(4 * window), ranges, ents;
  if (n_literals) {
    for (uint32_t li = 0; li < n_literals; ++li)
      hashes[li] = or_fnv1a(packed + offsets[2 * li], offsets[2 * li + 1], window);
    uint32_t nb = 0;
    or_prefilter_build(offsets, hashes.data(), n_literals, window, nullptr, nullptr, &nb, nullptr);
    ranges.resize(2 * (size_t)nb);
    ents.resize(2 * (size_t)n_literals);
    or_prefilter_build(offsets, hashes.data(), n_literals, window, meta.data(), ranges.data(), &nb, ents.data());
  }
  // regexes: general ones use find_iter_one, the rest share first-pair indexes
  // in blocks of 32 (as or_regex_set_scan)
  struct Block {
    std::vector<uint32_t> members;
    std::vector<std::vector<uint16_t>> index, last_byte;
  };
  std::vector<uint32_t> general;
  std::vector<Block> blocks;
  for (uint32_t k = 0; k < n_regex; ++k) {
    const Program& P = rs[k]->prog;
    if (P.nullable || P.has_assert) { general.push_back(k); continue; }
    if (blocks.empty() || blocks.back().members.size() == 32) blocks.emplace_back();
    blocks.back().members.push_back(k);
  }
  for (auto& b : blocks) {
    b.index.assign(65536, {});
    b.last_byte.assign(256, {});
    for (uint16_t j = 0; j < b.members.size(); ++j) {
      const Program& P = rs[b.members[j]]->prog;
      for (size_t key = 0; key < 65536; ++key)
        if ((P.pair_ok[key >> 6] >> (key & 63)) & 1) b.index[key].push_back(j);
      for (int c = 0; c < 256; ++c) if (P.one_byte[c]) b.last_byte[c].push_back(j);
    }
  }
  int T = std::max(1, std::min<int>(resolve_threads(nthreads), (int)std::max<uint64_t>(n_items, 1)));
  std::vector<std::vector<or_tagged_match>> res(T);
  std::atomic<uint64_t> next{0};
  std::vector<std::thread> th;
  for (int t = 0; t < T; ++t) {
    th.emplace_back([&, t] {
      std::vector<std::unique_ptr<Backtracker>> bts;
      for (uint32_t k = 0; k < n_regex; ++k) bts.emplace_back(new Backtracker(rs[k]->prog));
      std::vector<std::pair<uint32_t, uint32_t>> tmp;
      std::vector<uint64_t> cursor;
      auto& r = res[t];
      while (true) {
        uint64_t it = next.fetch_add(1);
        if (it >= n_items) break;
        const uint8_t* d = data + item_off[it];
        const uint64_t len = item_len[it], sid = item_id[it];
        // contract L inside the item
        for (uint64_t pos = 0; n_literals && pos < len; ++pos) {
          uint32_t h = FNV_BASIS;
          uint64_t maxp = std::min<uint64_t>(window, len - pos);
          for (uint64_t i = 0; i < maxp; ++i) {
            h = (h ^ d[pos + i]) * FNV_PRIME;
            const uint32_t* m = &meta[4 * i];
            if (m[2] == 0) continue;
            uint32_t bi = m[0] + (h & m[1]);
            uint32_t es = ranges[2 * bi], ec = ranges[2 * bi + 1];
            for (uint32_t e = 0; e < ec; ++e) {
              if (ents[2 * (es + e)] != h) continue;
              uint32_t li = ents[2 * (es + e) + 1];
              uint32_t lo = offsets[2 * li], ll = offsets[2 * li + 1];
              if (pos + ll > len) continue;
              if (std::memcmp(d + pos, packed + lo, ll) == 0)
                r.push_back({sid, literal_pattern_ids[li], (uint32_t)pos, (uint32_t)(pos + ll), 0});
            }
          }
        }
        // contract R inside the item
        for (uint32_t k : general) {
          tmp.clear();
          find_iter_one(rs[k], d, len, tmp);
          for (auto& m : tmp) r.push_back({sid, regex_pattern_ids[k], m.first, m.second, 0});
        }
        for (const auto& b : blocks) {
          cursor.assign(b.members.size(), 0);
          for (uint64_t q = 0; q < len; ++q) {
            const std::vector<uint16_t>& lst =
                (q + 1 < len) ? b.index[(size_t)d[q] << 8 | d[q + 1]] : b.last_byte[d[q]];
            for (uint16_t j : lst) {
              if (q < cursor[j]) continue;
              int64_t e = bts[b.members[j]]->run(d, len, q);
              if (e >= 0) {
                r.push_back({sid, regex_pattern_ids[b.members[j]], (uint32_t)q, (uint32_t)e, 0});
                cursor[j] = (uint64_t)e;
              }
            }
          }
        }
      }
    });
  }
  for (auto& x : th) x.join();
  std::vector<or_tagged_match> all;
  for (auto& r : res) all.insert(all.end(), r.begin(), r.end());
  std::sort(all.begin(), all.end(), [](const or_tagged_match& a, const or_tagged_match& b) {
    if (a.source_id != b.source_id) return a.source_id < b.source_id;
    if (a.start != b.start) return a.start < b.start;
    if (a.pattern_id != b.pattern_id) return a.pattern_id < b.pattern_id;
    return a.end < b.end;
  });
  for (uint64_t k = 0; k < all.size() && k < cap; ++k) out[k] = all[k];
  return all.size();
}

void or_sort_matches(or_match* m, uint64_t n) {
  std::sort(m, m + n, [](const or_match& a, const or_match& b) {
    if (a.start != b.start) return a.start < b.start;
    if (a.pattern_id != b.pattern_id) return a.pattern_id < b.pattern_id;
    return a.end < b.end;
  });
}

int or_hw_threads(void) { return resolve_threads(0); }

}  // extern "C"
