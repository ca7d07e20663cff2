// Device forms of alpacc's grammar tables, derived once per grammar on the host.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/alpacc_b200.h"

namespace alpacc {

constexpr int kMaxLanes = 32;     // distinct live states a chunk may start with
constexpr int kMaxMachine = 255;  // states of the minimised lexer automaton (u8)

// The sequential lexer of backends/c/lexer.c run over encoded endomorphism
// states is a Moore machine: state = encoded state_t, input = byte,
// delta(s, b) = COMPOSE[idx(s)][idx(TO_STATE[b])], outputs terminal(s),
// produce(s) and ACCEPT[idx(s)]. This is that machine restricted to the states
// reachable from IDENTITY and minimised, with bytes grouped into classes that
// act identically. Running it reproduces lex_string exactly.
struct LexerMachine {
  int M = 0;                  // states
  int C = 0;                  // byte classes
  int m0 = 0;                 // state for IDENTITY (before the first byte)
  int dead = -1;              // absorbing non-accepting state, or -1
  int max_lanes = 0;          // largest number of distinct live targets of a class
  int reachable = 0;          // endomorphism states reachable from IDENTITY
  std::vector<uint8_t> cls;   // [256] byte -> class
  std::vector<uint8_t> trans; // [M*C] next state
  std::vector<uint8_t> term;  // [M] terminal of the state
  std::vector<uint8_t> flags; // [M] bit0 produce, bit1 accept, bit2 kept (terminal != ignore)
  std::vector<uint8_t> img;       // [C*kMaxLanes] distinct live targets of each class
  std::vector<uint8_t> img_cnt;   // [C]
  std::vector<uint8_t> lane_of;   // [C*M] slot of trans[s][c] in img[c] or 0xff (dead)
  // [C*C] (machines of at most 64 states): bit s set when some live state
  // reaches live state s on a byte of class c0 followed by one of class c1
  std::vector<unsigned long long> img2;
};

// The lexer kernel's shared-memory form of the machine: rows of CP >= C
// 32-bit entries (CP a power of two), entry(s, c) stored at
// s * CP + (c ^ (s & swz)) = F(next) | code << 24, where F(x) = (x << shift) |
// ((x & swz) << 2) is the byte offset of x's row (so F(s) ^ (c * 4) is the
// byte offset of entry (s, c)), and code is what happens before the byte:
// 0xFF no token boundary, 0xFE the token ending there is ignored, else its
// terminal id.
//
// The window machine: the subset automaton of the machine's live states,
// started from the set of all of them, in the same row format (rows of CP
// entries, F and swizzle as above): entry(p, c) = F(next set) | info << 24,
// info = the next set's one state when it has exactly one, the dead state
// when it is empty, 0xFF when it has two or more. Walking it over the bytes
// before a chunk gives the set of states the chunk can start in. Built when
// it has at most kMaxWindowSets sets and its rows fit kWindowBytes; else
// ps_tab is empty.
constexpr int kMaxWindowSets = 1024;
constexpr size_t kWindowBytes = 48 * 1024;

struct LexerTable {
  std::vector<uint32_t> tab;   // [M * CP]
  std::vector<uint16_t> cls4;  // [256] class * 4
  int shift = 2;               // log2(CP) + 2
  int swz = 0;                 // min(CP, 32) - 1
  int wide_cls = 0;            // class * 4 does not fit a byte (C > 64)
  std::vector<uint32_t> ps_tab;             // [P * CP] window machine, or empty
  std::vector<unsigned long long> ps_mask;  // [P * 4] member states of each set (bit s of word s / 64)
  uint32_t ps_full = 0;                     // F of the set of all live states
  int ps_sets = 0;                          // P
};

int build_lexer_table(const LexerMachine &lm, LexerTable *out, std::string *why);

// LLP pair table, in one of two forms. Dense (key spaces up to 2^26): an
// array indexed by the key's terminals in base NT (NT = END + 1), entry =
// record index or 0xffffffff when the reference's lookup_key
// (backends/c/parser.c:17-45) would fail for that key. Hashed (larger key
// spaces, or forced): the reference's own open-addressing table, probed on
// the device exactly as lookup_key probes it - FNV-1a over the key's
// terminals, linear probing up to MAX_ITERS slots, the first slot holding the
// key decides - with the key's terminals packed 8 bits each into a u64 and per
// slot a record index, kEmptySlot (not a valid slot: probing goes on) or
// kMissingKey (the key is there but a span is negative: lookup fails).
constexpr uint32_t kEmptySlot = 0xffffffffu, kMissingKey = 0xfffffffeu;
constexpr uint64_t kDenseLimit = 1ull << 26;

struct PairTable {
  int nt = 0;                     // terminal ids 0..nt-1
  int q = 0, k = 0;
  uint64_t dense_size = 0;
  std::vector<uint32_t> dense;    // [nt^(q+k)], empty in the hashed form
  bool hashed = false;
  uint64_t max_iters = 0;
  std::vector<unsigned long long> ht_key;  // [HASH_TABLE_SIZE] packed key terminals
  std::vector<uint32_t> ht_rec;            // [HASH_TABLE_SIZE] record index, kEmptySlot or kMissingKey
  // record r: STACKS[rec_ss[r] .. +rec_nb[r]) and PRODUCTIONS[rec_ps[r] .. +rec_np[r])
  std::vector<uint32_t> rec_ss, rec_ps;
  std::vector<uint8_t> rec_nb, rec_np;
  std::vector<uint32_t> stacks;   // bracket: bit31 = left, low bits = unpacked symbol
  std::vector<uint32_t> prods;    // production ids
  std::vector<int32_t> arity;     // per production
  std::vector<uint8_t> is_term;   // per production: terminal production flag
  int max_br = 0, max_pr = 0;
};

struct HostGrammar {
  alpacc_tables t;    // widths and scalars (pointers not retained)
  LexerMachine lex;
  PairTable pairs;
  uint64_t len_max = 0;
  int ignore = -1;
  int parts = 0;      // ALPACC_PARTS_*
};

// Validates the tables and builds the device forms. Returns ALPACC_OK or an
// error code with a message in *why.
int build_host_grammar(const alpacc_tables *t, HostGrammar *out, std::string *why);

}  // namespace alpacc
