// vfb_device.cuh -- device-side data layout and per-word primitives.
//
// Characteristic set (CS): one uint64 word per trace, bit t = "formula holds
// at step t of that trace" (LTL_BS.cu:146, 183-238).  Rows of the level cache
// are stored row-major with a padded pitch of TP = T rounded up to an even
// number of words, so every row starts on a 16-byte boundary (128-bit loads,
// bulk copies).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace vfb {

constexpr int kMaxTraces = 128;
constexpr int kMaxSize = 32;          // formula size limit (ltl_nocache.cu:11)
constexpr int kMaxSplits = 16;        // floor((32-1)/2)
// P1 operand groups of a level: up to 4 unary (one per operand level) and the
// binary level pairs; with unit costs, 1 + floor((k-1)/2)
constexpr int kGroups = 64;
constexpr int kTS = 128;              // stream rows per P1 tile (= threads per CTA)
// Staged rows per P1 tile (maximum).  The shared memory of a tile holds kTS
// stream rows and kTQ staged rows; 16 rather than 32 lets three CTAs share an
// SM at 64 words per row instead of two (k_p1 of the large instance 40 ->
// 34 ms), and 32 staged rows gained under 1% where the autotuner chose them.
constexpr int kTQ = 16;
constexpr int kTQDefault = 16;        // staged rows per P1 tile unless the tune table says otherwise
constexpr int kP1TileTarget = 4096;   // shrink the staged height until a level has this many tiles
// P1 launch shape per level band (tuned by the host): band b holds the levels
// of 4^b to 4^(b+1)-1 candidates, the last band every larger level
constexpr int kTuneBands = 16;
constexpr int kMaxProbes = 4096;      // bounded linear probing
// first buffers of at most this many table + bitmap bytes are initialised by
// one k_fill launch for every new instance of the call instead of by two
// memsets each (larger ones keep their memsets)
constexpr uint64_t kInitFillMax = 64ull << 20;
constexpr uint64_t kEmpty = ~0ULL;
constexpr int kPayShift = 58;         // payload = level << 58 | candidate index
constexpr uint64_t kIdxMask = (1ULL << kPayShift) - 1;

enum Op : int { OP_NOT = 0, OP_AND, OP_OR, OP_X, OP_F, OP_G, OP_U, OP_ATOM = 7 };

enum Status : int {
  ST_IDLE = 0,
  ST_RUNNING = 1,
  ST_FOUND = 2,
  ST_NOT_FOUND = 3,
  ST_NEED_MEM = 4,     // a buffer is too small: host grows it and re-runs the level
  ST_ERROR = 5,
  ST_LIMIT = 6,        // an on-the-fly level held no solution: the search cannot go on
  ST_WAIT = 7,         // batch: memory for the next level is held by other instances; the
                       // host retries the growth later (kernels leave the instance alone)
};

enum NeedBits : int {
  NEED_BITMAP = 1, NEED_TABLE = 2, NEED_LIST = 4, NEED_ROWS = 8, NEED_LIMIT = 16,
  NEED_PROMOTE = 32,   // level too large for the cluster solver: continue on the whole GPU
  NEED_ROWS_EST = 64,  // with NEED_ROWS: the rows were asked for by the plan's projection (the
                       // level's owners are not known yet), not by the owner count
};

enum KeyMode : int { KEY_CONCAT = 0, KEY_SAMPLED = 1, KEY_HASH = 3 };

struct __align__(32) Slot {
  unsigned long long h, l, pay, aux;
};
struct __align__(16) Key128 {
  unsigned long long h, l;
};

// Tuning band of a level of `cands` candidates: floor(log4(cands)), clamped.
__host__ __device__ inline int tune_band(unsigned long long cands) {
  int b = 0;
  while (b < kTuneBands - 1 && (cands >> (2 * b + 2)) != 0) ++b;
  return b;
}

// Per-instance device state.  Kernels read everything they need from here,
// so one captured launch sequence serves every level and every batch.
struct InstDev {
  // ---- problem (written once by the host)
  int T, TP, A, npos, max_size, key_mode, stride1, lensum;
  uint8_t len[kMaxTraces];
  uint8_t off[kMaxTraces];     // bit offset of the trace's key field (<=126)
  uint8_t width[kMaxTraces];   // key field width (0 when past bit 126)
  // P1 launch shape by level band (tune_band); 0 everywhere = the built-in
  // choice: staged rows at most tune_rows (a power of two, 0: kTQDefault), at least
  // 2^tune_tiles tiles while the staged height can shrink (0: kP1TileTarget),
  // tune_blocks CTAs (0: every resident CTA)
  uint8_t tune_rows[kTuneBands], tune_tiles[kTuneBands];
  uint16_t tune_blocks[kTuneBands];
  uint64_t posmask[2];         // bit i: trace i is positive
  uint8_t cost[8];             // operator costs c1..c8 of LTL_BS (p ~ & | X F G U); 0 means 1.
                               // Level k holds the formulas of cost k (unit costs: size k)
  int neg_type;                // 2: ~ applies to propositions only (LTL_BS NegType)
  int weighted;                // some cost above 1 or neg_type 2 (else the size order's fast paths)
  int on_the_fly;              // the level's rows did not fit: its candidates are only tested as
                               // solutions, nothing is stored (LTL_BS onTheFly, LTL_BS.cu:331-349)
  // ---- buffers (host-owned allocations; pointers may change between levels)
  uint64_t* rows;              // [row_cap][TP]
  uint64_t* origin;            // [row_cap] candidate index within the row's level
  uint64_t row_cap;
  Slot* table;
  uint64_t table_mask;         // capacity - 1 (power of two)
  uint32_t* bitmap;            // owner bits, one per candidate of the level being built
  uint64_t bitmap_words;
  uint64_t* wins;              // owners of new keys, ascending candidate index
  uint64_t tent_cap;           // capacity of wins
  // ---- search state
  int status, level, need, pad0;
  uint64_t need_amount[4];     // requested bitmap words / slots / list entries / rows
  uint64_t lstart[kMaxSize + 2];
  uint64_t lcount[kMaxSize + 2];
  uint64_t lcands[kMaxSize + 2];
  uint64_t keys;               // keys in the table
  uint64_t cands;              // candidates of the level being built
  uint64_t base_not, base_x, base_f, base_g;
  uint64_t base_and[kMaxSize + 1], base_or[kMaxSize + 1];   // indexed by the left operand's level
  uint64_t base_u[kMaxSize];
  // P1 tile groups.  Unit costs: groups 0..m-1 = the size splits (i, k-1-i),
  // i = 1..m, then group m = the unary operators over level k-1
  uint64_t grp_prefix[kGroups + 1];
  uint32_t grp_qtiles[kGroups];
  // group g: kind 0 = unary over level la (mask bits ~ X F G), kind 1 = binary
  // over levels la <= lb (mask bits &, |, la U lb, lb U la)
  uint8_t grp_kind[kGroups], grp_mask[kGroups], grp_la[kGroups], grp_lb[kGroups];
  // first candidate index of each operator of a group: unary ~ X F G at
  // operand row 0, binary & | laUlb lbUla at operand rows (0, 0)
  uint64_t grp_base[kGroups][4];
  int p1_masked;   // a P1 tile of this attempt skipped operators past best_cand
  int no_mask;     // this level is re-run without skipping (set by the table scan)
  int mask_off;    // never skip (contexts that cannot re-run a level)
  int rows_deferred;  // the projected rows of this level did not fit the budget: the level
                      // runs without them and the owner count after the table scan decides
  int ngroups;
  int tq;                      // staged rows per P1 tile at this level (1..kTQ)
  int p1_blocks;               // P1 CTAs this level asks for (0: every resident CTA)
  unsigned long long promote_above;  // candidates per level above which the instance
                                     // leaves the cluster solver (~0: never)
  // per-level counters
  unsigned long long n_new, n_wins, probe_fail;
  unsigned long long best_cand;  // min candidate index whose CS satisfies the sample (P1)
  unsigned long long best_sol;   // min candidate index of a solution owning its key
  int sol_known;                 // best_sol settled before the rows were emitted
  // At a level with a solution candidate the table scan counts the owners
  // below it (n_below) instead of marking every owner's bit; counted_below:
  // the count stands (the candidate owns its key), lcount = n_below + 1
  unsigned long long n_below;
  int counted_below;
  int fill;                      // 1: the table and the bitmap are still to be initialised (k_fill)
  int atoms_staged;              // 1: the proposition rows wait in the batch's staging buffer at
  uint64_t atom_off;             // word atom_off; k_init copies them into the level cache
  unsigned long long n_newlist;  // slots of keys first inserted by this level's P1 (listed in wins)
  int attempt, attempt_level;    // attempts at the current level (> 1: a retry after growth)
  int planned, p1_tail;          // level the current plan (bases, tiling) was made for (0: none);
                                 // 1 when this step's k_p1 finishes the level's tiles
  unsigned long long p1_done;    // tiles of the level processed by earlier steps
  unsigned long long p1_step;    // tiles this step processes
  unsigned long long p1_quota;   // candidates per step (0: the whole level in one step)
  unsigned long long plan_tiles, plan_words, plan_tchunks;   // P1 tiles, bitmap words, table-scan
                                                             // chunks of the current plan
  // figures of the last level built (for the host's profile): candidates,
  // owners, hash-set slots the owner scan visited, solution settled early
  unsigned long long built_cands, built_wins, built_scanned;
  int built_sol_known;
  int emit_item;                 // owners per k_emit work item at this level (set by the table scan)
  uint32_t scan_slots;           // table-scan chunk of this level's plan (slots; a power of two)
  int no_list;                   // the level has a solution from the start (unary hits): P1 does not
                                 // list its new slots and the table scan reads the whole table
  // First rows of each stored level whose ~ / X / F / G candidates satisfy
  // the sample (step 0 of every trace equal to its label), stored as
  // 0xFFFFFFFF - row (0: none, so a zeroed record has none); written when
  // the level's rows are (k_init, k_emit), read by the plan of the levels
  // that apply those operators to it
  uint32_t uhit[kMaxSize + 2][4];
  // ---- result
  int res_size, rpn_len;
  int16_t rpn[kMaxSize];
  uint64_t sol_index;
};

// ------------------------------------------------------------- word operators
__device__ __forceinline__ uint64_t len_mask(int L) {
  return L >= 64 ? ~0ULL : ((1ULL << L) - 1ULL);
}

// F: bit t set iff some bit >= t is set (suffix OR), i.e. every bit at or
// below the most significant set bit.  Same function as the shift-doubling of
// LTL_BS.cu:208-213, computed from the leading-zero count.
__device__ __forceinline__ uint64_t w_fin(uint64_t w) {
  const uint64_t m = ~0ULL >> (__clzll((long long)w) & 63);
  return w ? m : 0ULL;
}

__device__ __forceinline__ uint64_t w_glob(uint64_t w, uint64_t lm) {
  return w & ~w_fin(~w & lm);
}

// l U r on one word: U_t = r_t | (l_t & U_{t+1}).  Reversing the bit order
// turns the recurrence into a carry chain (generate = r, propagate = l), which
// one 64-bit addition resolves; the carry out of bit 63 supplies the top bit.
// Equal to the 6-step doubling of LTL_BS.cu:222-233 on every input.
__device__ __forceinline__ uint64_t w_until(uint64_t l, uint64_t r) {
  const uint64_t lr = __brevll(l), rr = __brevll(r);
  const uint64_t a = lr | rr;
  const uint64_t s = a + rr;
  const uint64_t c = s ^ a ^ rr;
  const uint64_t cout = (s < a) ? 1ULL : 0ULL;
  return __brevll((c >> 1) | (cout << 63));
}

__device__ __forceinline__ uint64_t splitmix_fin(uint64_t x) {
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}

// ------------------------------------------------------------------ key state
// Streaming accumulation of the 126-bit key of LTL_BS.cu:30-110 over the words
// of one CS (word i of trace i, in trace order).
struct KeyAcc {
  uint64_t a0, a1;  // KEY_CONCAT/KEY_SAMPLED: bits 0..127; KEY_HASH: l, h
};

__device__ __forceinline__ void key_init(KeyAcc& k) { k.a0 = k.a1 = 0; }

__device__ __forceinline__ uint64_t compress_stride(uint64_t w, int stride, int L) {
  uint64_t f = 0;
  int j = 0;
  for (int k = 0; k < L; k += stride, ++j) f |= ((w >> k) & 1ULL) << j;
  return f;
}

template <int MODE>
__device__ __forceinline__ void key_word(KeyAcc& k, uint64_t w, int i, int half, int off, int width,
                                         int stride, int L) {
  if (MODE == KEY_HASH) {
    const uint64_t x = splitmix_fin(w);
    if (i < half) k.a1 ^= x; else k.a0 ^= x;   // a1 = h, a0 = l
  } else {
    uint64_t f = (MODE == KEY_SAMPLED) ? compress_stride(w, stride, L) : w;
    f &= (width >= 64) ? ~0ULL : ((1ULL << width) - 1ULL);
    if (width == 0) return;
    if (off < 64) {
      k.a0 |= f << off;
      if (off > 0 && off + width > 64) k.a1 |= f >> (64 - off);
    } else {
      k.a1 |= f << (off - 64);
    }
  }
}

template <int MODE>
__device__ __forceinline__ void key_final(const KeyAcc& k, uint64_t& h, uint64_t& l) {
  if (MODE == KEY_HASH) {
    h = k.a1;
    l = k.a0;
  } else {
    const uint64_t lo = k.a0, hi = k.a1 & ((1ULL << 62) - 1ULL);   // 126 bits
    l = lo & ((1ULL << 63) - 1ULL);
    h = ((lo >> 63) | (hi << 1)) & ((1ULL << 63) - 1ULL);
  }
  // WarpCore rejects its empty (~0) and tombstone (~0-1) keys with slot code 0
  // (hash_set.cuh:201-205): both values name the same pair component.
  if (h == ~0ULL) h = ~0ULL - 1;
  if (l == ~0ULL) l = ~0ULL - 1;
}

__device__ __forceinline__ uint64_t slot_hash(uint64_t h, uint64_t l) {
  return splitmix_fin(h ^ (l * 0x9E3779B97F4A7C15ULL) ^ 0x5ad0dedULL);
}

// Operator cost (op index into ~ & | X F G U) and the propositions' cost
// (their level); 0 in the record means 1.
__host__ __device__ __forceinline__ int op_cost(const InstDev& I, int op) {
  return I.cost[1 + op] ? I.cost[1 + op] : 1;
}
__host__ __device__ __forceinline__ int atom_level(const InstDev& I) { return I.cost[0] ? I.cost[0] : 1; }
// Operand level of ~ at level k, or -1 when ~ has no candidates there.
__host__ __device__ __forceinline__ int not_level(const InstDev& I, int k) {
  const int L = k - op_cost(I, OP_NOT), c1 = atom_level(I);
  return (L < c1 || (I.neg_type == 2 && L != c1)) ? -1 : L;
}

__device__ __forceinline__ bool is_pos(const InstDev& I, int i) {
  return (I.posmask[i >> 6] >> (i & 63)) & 1ULL;
}

}  // namespace vfb
