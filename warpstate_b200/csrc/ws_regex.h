// Host-side regex front end of the B200 scan path: parser, Thompson NFA and the
// three DFA constructions the kernels walk.
//
// Syntax and flags follow what the reference compiles its regexes with:
// regex-syntax with unicode(false), utf8(false) and multi_line(true)
// (core/src/pattern/compiler.rs:167-174, core/src/regex_engine.rs:7-17,
// core/src/dfa/builder.rs:36-54).  Patterns that can match the empty string
// are rejected for the GPU path with PatternCompilationFailed; everything
// else in that syntax is supported, look-around assertions (^ $ \b \B \A \z)
// through the context DFAs below.
#pragma once
#include <bitset>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace ws {

struct CompileError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

using ByteSet = std::bitset<256>;

// ------------------------------------------------------------------ syntax tree
struct ReNode {
  enum Type : uint8_t { BYTES, CAT, ALT, REP, LOOK, EMPTY, CAPTURE } type;
  ByteSet bytes;              // BYTES
  std::vector<int> kids;      // CAT / ALT / REP(1) / CAPTURE(1)
  int lo = 0, hi = -1;        // REP bounds, hi = -1 unbounded
  bool greedy = true;         // REP
  int look = 0;               // LOOK kind
};

struct ReTree {
  std::vector<ReNode> nodes;
  int root = -1;
};

ReTree parse_regex(const std::string& src);  // throws CompileError

// Analyses the reference performs on the HIR.
bool tree_literal(const ReTree& t, std::vector<uint8_t>* out);   // compiler.rs:353-373
bool tree_pathological(const ReTree& t);                         // compiler.rs:381-405
bool tree_nullable(const ReTree& t);
bool tree_has_look(const ReTree& t);
int64_t tree_max_len(const ReTree& t);  // -1 when unbounded

// ------------------------------------------------------------------------- NFA
struct NfaState {
  enum Kind : uint8_t { CONSUME, SPLIT, EPS, MATCH, ASSERT } kind;
  int a = -1, b = -1;  // successors (SPLIT: a has priority over b)
  int set = -1;        // CONSUME: index into Nfa::sets
  int pattern = -1;    // MATCH: local pattern index
  int look = 0;        // ASSERT: look-around kind (LOOK_* below); passes to a when it holds
};

// Look-around kinds (multi_line(true), ASCII word characters).
enum { LOOK_LINE_START = 1, LOOK_LINE_END, LOOK_TEXT_START, LOOK_TEXT_END, LOOK_WORD, LOOK_NOT_WORD };

// Context of a position for the assertions: the byte before it (CTX_BEGIN at
// the start of the input or batch item) and the byte at it (CTX_BEGIN standing
// for the end of the input or item): a line feed, an ASCII word byte
// [0-9A-Za-z_], or any other byte.
enum { CTX_BEGIN = 0, CTX_NL = 1, CTX_WORD = 2, CTX_OTHER = 3 };
inline int byte_context(uint8_t c) {
  if (c == '\n') return CTX_NL;
  const bool w = (c >= '0' && c <= '9') || (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || c == '_';
  return w ? CTX_WORD : CTX_OTHER;
}
// Whether an assertion holds between a position's left and right contexts.
bool look_holds(int look, int left, int right);

struct Nfa {
  std::vector<NfaState> states;
  std::vector<ByteSet> sets;
  std::vector<int> starts;  // one start per pattern
};

// Builds the NFA of several patterns; `reverse` builds the NFA of the reversed
// language (used for start discovery after an unanchored forward walk).
Nfa build_nfa(const std::vector<const ReTree*>& trees, bool reverse);

// Byte classes: bytes that no set in the NFA distinguishes share a class.
struct ByteClasses {
  uint8_t map[256];
  int count = 0;
  std::vector<uint8_t> representative;  // one byte per class
};
ByteClasses compute_classes(const std::vector<const Nfa*>& nfas);

// ------------------------------------------------------------------------- DFA
// Transition words use the reference's packing (core/src/dfa/mod.rs:19-22):
// bits 0..29 next state index, bit 31 = next state is a match state,
// bit 30 = next state is dead.  State 0 is the dead state.
constexpr uint32_t DFA_FLAG_MATCH = 0x80000000u;
constexpr uint32_t DFA_FLAG_DEAD = 0x40000000u;
constexpr uint32_t DFA_MASK_STATE = 0x3FFFFFFFu;

struct Dfa {
  int n_states = 0;
  int n_classes = 0;
  std::vector<uint32_t> trans;          // n_states * n_classes
  std::vector<uint8_t> is_match;        // per state
  std::vector<uint32_t> match_ptr;      // n_states + 1 offsets into match_list
  std::vector<uint32_t> match_list;     // local pattern indices
  uint32_t start_anchored = 0;
  uint32_t start_unanchored = 0;        // forward DFAs only
  bool too_big = false;
  uint32_t ctx_start[4] = {0, 0, 0, 0};  // context DFAs: start state per left context
};

// MatchKind::All DFA over a group of patterns.  With `with_unanchored`, the
// unanchored start (an implicit (?s-u:.)*? prefix) and every state reachable
// from it are included, next to the anchored start.
Dfa build_all_dfa(const Nfa& nfa, const ByteClasses& cls, bool with_unanchored, int max_states);

// Leftmost-first anchored DFA of one pattern (priority-ordered subsets; a match
// drops every lower-priority thread), the automaton a backtracking engine's
// first match corresponds to.  Walking it from s and remembering the last match
// position gives the end find_iter reports for a match starting at s.
Dfa build_leftmost_first_dfa(const Nfa& nfa, const ByteClasses& cls, int max_states);

// Context DFAs of patterns with look-around assertions.  A state is the set of
// NFA threads before their epsilon closure plus the left context of the
// current position; the closure is taken on the next byte, whose context
// decides the look-ahead half of every assertion.  So the transition on the
// byte at position p reports the matches that END AT p (one byte late), and
// the end of the input or item needs the end step: the closure under the
// right context CTX_BEGIN.  Anchored only; ctx_start[k] is the start state for
// left context k.  The byte classes must separate the contexts
// (compute_classes does when the NFA has assertions).
//   build_context_all_dfa: MatchKind::All over a group of patterns.  The
//     patterns matching at p are listed per (state, right context):
//     match_ptr has 4 * n_states + 1 entries, list (s, k) at 4 * s + k; the
//     match flag of a transition says its list is not empty.
//   build_context_lf_dfa: leftmost-first over one pattern (a match drops
//     every lower-priority thread); is_match[s] says the end step matches.
Dfa build_context_all_dfa(const Nfa& nfa, const ByteClasses& cls, int max_states);
Dfa build_context_lf_dfa(const Nfa& nfa, const ByteClasses& cls, int max_states);

// Reorders states so that `order` (old ids, dead state first) becomes 0..n-1.
void renumber_dfa(Dfa& d, const std::vector<uint32_t>& order);

}  // namespace ws
