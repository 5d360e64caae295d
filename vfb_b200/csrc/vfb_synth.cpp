// vfb_synth.cpp -- native twin of vfb_b200/synth.py's planted_instance().
//
// Rejection-samples traces labelled by a uniformly drawn planted formula with
// exactly the random stream of the Python generator (xoshiro256** state passed
// in and out), so both produce identical instances for the same seed; the
// Python module uses this when the library is present because the per-bit
// draws are slow in Python.  Formula numbering: generateMatrix and
// numberToFormula of ltl_nocache.cu:169-224, 248-287; labelling semantics:
// evaluateRPN, ltl_nocache.cu:95-150.
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/vfb.h"

namespace {

typedef unsigned __int128 u128;

struct Rng {
  uint64_t s[4];
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {
    const uint64_t result = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return result;
  }
  // uniform in [0, n), n >= 1, as Rng.below (bit-length rejection)
  u128 below(u128 n) {
    int bits = 1;
    for (u128 m = n - 1; m >> bits; ) ++bits;
    if (n - 1 == 0) bits = 1;
    const int words = (bits + 63) / 64;
    for (;;) {
      u128 v = 0;
      for (int w = 0; w < words; ++w) v = (v << 64) | next();
      v >>= (words * 64 - bits);
      if (v < n) return v;
    }
  }
  double random() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
  uint64_t bernoulli_word(int nbits, double p) {
    uint64_t w = 0;
    for (int t = 0; t < nbits; ++t)
      if (random() < p) w |= 1ULL << t;
    return w;
  }
};

int bit_length(u128 x) {
  int b = 0;
  while (x) { ++b; x >>= 1; }
  return b;
}

void counts(int A, int K, std::vector<u128>& c) {   // c[size*8 + op], op 7 = total
  c.assign((size_t)(K < 2 ? 3 : K + 1) * 8, 0);
  c[1 * 8 + 7] = A;
  c[2 * 8 + 0] = c[2 * 8 + 3] = c[2 * 8 + 4] = c[2 * 8 + 5] = A;
  c[2 * 8 + 7] = 4 * (u128)A;
  for (int i = 3; i <= K; ++i) {
    const u128 un = c[(i - 1) * 8 + 7];
    u128 com = 0, ncom = 0;
    for (int j = 1; j <= (i - 1) / 2; ++j) com += c[j * 8 + 7] * c[(i - j - 1) * 8 + 7];
    for (int j = 1; j <= i - 2; ++j) ncom += c[j * 8 + 7] * c[(i - j - 1) * 8 + 7];
    c[i * 8 + 0] = c[i * 8 + 3] = c[i * 8 + 4] = c[i * 8 + 5] = un;
    c[i * 8 + 1] = c[i * 8 + 2] = com;
    c[i * 8 + 6] = ncom;
    c[i * 8 + 7] = 4 * un + 2 * com + ncom;
  }
}

const char kOps[] = "~&|XFGU";

void decode(u128 n, int size, const std::vector<u128>& c, std::vector<int>& out) {
  if (size == 1) {
    out.push_back((int)n);
    return;
  }
  int op = 0;
  while (n >= c[size * 8 + op]) n -= c[size * 8 + op++];
  const int sub = size - 1;
  if (op == 0 || op == 3 || op == 4 || op == 5) {
    decode(n, sub, c, out);
  } else {
    int left = 1;
    while (n >= c[left * 8 + 7] * c[(sub - left) * 8 + 7]) {
      n -= c[left * 8 + 7] * c[(sub - left) * 8 + 7];
      ++left;
    }
    const u128 nr = c[(sub - left) * 8 + 7];
    decode(n / nr, left, c, out);
    decode(n % nr, sub - left, c, out);
  }
  out.push_back(-(1 + op));
}

uint64_t mask(int L) { return L >= 64 ? ~0ULL : ((1ULL << L) - 1); }
uint64_t suffix_or(uint64_t w) {
  for (int s = 1; s <= 32; s <<= 1) w |= w >> s;
  return w;
}

uint64_t eval_word(const std::vector<int>& rpn, const uint64_t* words, int L) {
  uint64_t st[64];
  int sp = 0;
  for (int tk : rpn) {
    if (tk >= 0) { st[sp++] = words[tk]; continue; }
    const char op = kOps[-tk - 1];
    if (op == '~') st[sp - 1] = ~st[sp - 1] & mask(L);
    else if (op == 'X') st[sp - 1] >>= 1;
    else if (op == 'F') st[sp - 1] = suffix_or(st[sp - 1]);
    else if (op == 'G') st[sp - 1] &= ~suffix_or(~st[sp - 1] & mask(L));
    else {
      uint64_t r = st[--sp], l = st[sp - 1];
      if (op == '&') r &= l;
      else if (op == '|') r |= l;
      else {
        for (int s = 1; s <= 16; s <<= 1) {
          r |= l & (r >> s);
          l &= l >> s;
        }
        r |= l & (r >> 32);
      }
      st[sp - 1] = r;
    }
  }
  return st[0];
}

}  // namespace

extern "C" int vfb_synth_planted(uint64_t* rng_state, int num_vars, int planted_size, int n_pos, int n_neg,
                                 int len_lo, int len_hi, double p, int max_draws_per_trace, uint64_t* words_out,
                                 int* lengths_out, int16_t* rpn_out, int* rpn_len) {
  if (num_vars < 1 || num_vars > VFB_MAX_VARS || planted_size < 1 || planted_size > VFB_MAX_SIZE || n_pos < 0 ||
      n_neg < 0 || len_lo < 1 || len_hi > 64 || len_lo > len_hi)
    return -1;
  Rng rng;
  std::memcpy(rng.s, rng_state, sizeof(rng.s));
  std::vector<u128> c;
  counts(num_vars, planted_size, c);
  const int T = n_pos + n_neg;
  std::vector<uint64_t> w(num_vars);
  std::vector<int> rpn;
  for (;;) {
    rpn.clear();
    decode(rng.below(c[planted_size * 8 + 7]), planted_size, c, rpn);
    int np = 0, nn = 0;
    long long budget = (long long)max_draws_per_trace * T;
    while ((np < n_pos || nn < n_neg) && budget > 0) {
      --budget;
      const int L = (len_lo == len_hi) ? len_lo : len_lo + (int)rng.below((u128)(len_hi - len_lo + 1));
      for (int v = 0; v < num_vars; ++v) w[v] = rng.bernoulli_word(L, p);
      const bool holds = eval_word(rpn, w.data(), L) & 1ULL;
      int slot = -1;
      if (holds && np < n_pos) slot = np++;
      else if (!holds && nn < n_neg) slot = n_pos + nn++;
      if (slot >= 0) {
        lengths_out[slot] = L;
        for (int v = 0; v < num_vars; ++v) words_out[(size_t)slot * num_vars + v] = w[v];
      }
    }
    if (np == n_pos && nn == n_neg) break;
  }
  for (size_t i = 0; i < rpn.size(); ++i) rpn_out[i] = (int16_t)rpn[i];
  *rpn_len = (int)rpn.size();
  std::memcpy(rng_state, rng.s, sizeof(rng.s));
  (void)bit_length;
  return 0;
}
