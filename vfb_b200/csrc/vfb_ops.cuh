// vfb_ops.cuh -- device building blocks shared by the level-step kernels
// and the persistent and cluster solvers (vfb_kernels.cu): hash-set
// insert/find, candidate decoding, key computation, P1 tile processing,
// scans, formula reconstruction.
#pragma once
#include "vfb_kernels.cuh"

namespace vfb {

// ------------------------------------------------------------------ helpers
__device__ __forceinline__ Key128 ld_key(const Slot* s) {
  const ulonglong2 v = __ldcg(reinterpret_cast<const ulonglong2*>(s));
  return Key128{v.x, v.y};
}

__device__ __forceinline__ unsigned long long pay_of(int k, uint64_t g) {
  return ((unsigned long long)k << kPayShift) | (unsigned long long)g;
}

// Lower the key's payload to pay.  Returns 1 when pay is the key's minimum
// after the update (the candidate may own the key), 0 otherwise.  A payload
// equal to pay means the same candidate claimed it in an earlier attempt of
// this level, which still counts as owning.
__device__ __forceinline__ int claim(Slot* s, unsigned long long pay) {
  const unsigned long long cur = __ldcg(&s->pay);
  if (cur < pay) return 0;
  if (cur == pay) return 1;
  const unsigned long long old = atomicMin(&s->pay, pay);
  return old >= pay ? 1 : 0;
}

// Insert-or-find (h,l) starting at slot idx whose key half-words were already
// loaded into cur.  Returns 1/0 as claim(), -1 when the probe limit is hit.
__device__ inline int insert_min(Slot* tab, uint64_t mask, uint64_t& idx, Key128 cur, uint64_t h, uint64_t l,
                          unsigned long long pay, int& isnew) {
  for (int p = 0; p < kMaxProbes; ++p) {
    if (p > 0) cur = ld_key(tab + idx);
    if (cur.h == h && cur.l == l) return claim(tab + idx, pay);
    // A real key never has a half equal to ~0 (normalised away), so a ~0 half
    // is either an empty slot or a key being published: resolve with the CAS.
    if (cur.h == kEmpty || cur.l == kEmpty) {
      const Key128 old = atomicCAS(reinterpret_cast<Key128*>(tab + idx), Key128{kEmpty, kEmpty},
                                   Key128{h, l});
      if (old.h == kEmpty && old.l == kEmpty) {
        // this thread published the key: its payload is still the empty word,
        // so the minimum needs no read first (and its result is not awaited)
        isnew = 1;
        atomicMin(&tab[idx].pay, pay);
        return 1;
      }
      if (old.h == h && old.l == l) return claim(tab + idx, pay);
    }
    idx = (idx + 1) & mask;
  }
  return -1;
}

// Payload of (h,l), or ~0 if the key is absent.
__device__ inline unsigned long long find_pay(const Slot* tab, uint64_t mask, uint64_t h, uint64_t l) {
  uint64_t idx = slot_hash(h, l) & mask;
  for (int p = 0; p < kMaxProbes; ++p) {
    const Key128 cur = ld_key(tab + idx);
    if (cur.h == h && cur.l == l) return __ldcg(&tab[idx].pay);
    if (cur.h == kEmpty && cur.l == kEmpty) return ~0ULL;
    idx = (idx + 1) & mask;
  }
  return ~0ULL;
}

// Largest b with prefix[b] <= x (prefix non-decreasing, prefix[0] = 0 <= x < prefix[n]).
__device__ __forceinline__ int find_owner(const unsigned long long* prefix, int n, unsigned long long x) {
  int lo = 0, hi = n;  // prefix[lo] <= x < prefix[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (prefix[mid] <= x) lo = mid; else hi = mid;
  }
  return lo;
}

template <typename V>
__device__ __forceinline__ V warp_sum(V v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide exclusive scan of one value per thread (blockDim multiple of 32).
__device__ inline unsigned long long block_excl_scan(unsigned long long v, unsigned long long* s_warp,
                                              unsigned long long& total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  unsigned long long x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[wid] = x;
  __syncthreads();
  if (wid == 0) {
    unsigned long long w = lane < nw ? s_warp[lane] : 0ULL;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < nw) s_warp[lane] = w;
  }
  __syncthreads();
  total = s_warp[nw - 1];
  const unsigned long long before = wid > 0 ? s_warp[wid - 1] : 0ULL;
  __syncthreads();
  return before + x - v;
}

// Three exclusive block scans at once (one pass of barriers): v[c] -> the
// sum of v[c] over the threads before this one; total[c] = the block's sum.
__device__ inline void block_excl_scan3(const unsigned long long (&v)[3], unsigned long long (*s_warp)[3],
                                        unsigned long long (&excl)[3], unsigned long long (&total)[3]) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  unsigned long long x[3] = {v[0], v[1], v[2]};
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, x[c], o);
      if (lane >= o) x[c] += y;
    }
  }
  if (lane == 31) {
#pragma unroll
    for (int c = 0; c < 3; ++c) s_warp[wid][c] = x[c];
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      unsigned long long w = lane < nw ? s_warp[lane][c] : 0ULL;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      if (lane < nw) s_warp[lane][c] = w;
    }
  }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    total[c] = s_warp[nw - 1][c];
    excl[c] = (wid > 0 ? s_warp[wid - 1][c] : 0ULL) + x[c] - v[c];
  }
  __syncthreads();
}

__device__ __forceinline__ uint64_t apply_w(int op, uint64_t l, uint64_t r, int L) {
  switch (op) {
    case OP_NOT: return ~l & len_mask(L);
    case OP_AND: return l & r;
    case OP_OR: return l | r;
    case OP_X: return l >> 1;
    case OP_F: return w_fin(l);
    case OP_G: return w_glob(l, len_mask(L));
    default: return w_until(l, r);
  }
}

struct Cand {
  int op, la, lb;
  uint64_t a, b;
};

// q = g / n, r = g % n.  Below 2^52 the quotient comes from one correctly
// rounded double division (off by at most one, corrected from the remainder),
// which is much shorter than the 64-bit integer division sequence.
__device__ __forceinline__ void divmod64(uint64_t g, uint64_t n, uint64_t& q, uint64_t& r) {
  if (g < (1ULL << 52) && n < (1ULL << 52)) {
    uint64_t qq = (uint64_t)((double)g / (double)n);
    long long rr = (long long)(g - qq * n);
    if (rr < 0) { --qq; rr += (long long)n; }
    else if ((uint64_t)rr >= n) { ++qq; rr -= (long long)n; }
    q = qq;
    r = (uint64_t)rr;
  } else {
    q = g / n;
    r = g % n;
  }
}

// Canonical candidate index g of level k -> operator and operands (levels and
// indices within them).  Block order ~ & | X F G U; a unary operator of cost
// c reads level k - c; & and | over splits (i, k - c - i) with i <= k - c - i,
// U over every split; left index major (ltl_nocache.cu:169-224 with unit
// costs, LTL_BS.cu:1226-1488 with the operator costs).
__device__ inline Cand decode(const InstDev& I, int k, uint64_t g) {
  const uint64_t* n = I.lcount;
  Cand c;
  c.lb = 0;
  c.b = 0;
  if (!I.weighted) {
    // unit costs: the size order
    const uint64_t un = n[k - 1];
    if (g < un) { c.op = OP_NOT; c.la = k - 1; c.a = g; return c; }
    g -= un;
    for (int pass = 0; pass < 2; ++pass) {
      for (int i = 1; 2 * i <= k - 1; ++i) {
        const int j = k - 1 - i;
        const uint64_t cnt = n[i] * n[j];
        if (g < cnt) {
          c.op = pass ? OP_OR : OP_AND;
          c.la = i; c.lb = j;
          divmod64(g, n[j], c.a, c.b);
          return c;
        }
        g -= cnt;
      }
    }
    for (int op = OP_X; op <= OP_G; ++op) {
      if (g < un) { c.op = op; c.la = k - 1; c.a = g; return c; }
      g -= un;
    }
    for (int i = 1; i <= k - 2; ++i) {
      const int j = k - 1 - i;
      const uint64_t cnt = n[i] * n[j];
      if (g < cnt) {
        c.op = OP_U; c.la = i; c.lb = j;
        divmod64(g, n[j], c.a, c.b);
        return c;
      }
      g -= cnt;
    }
    c.op = -1;
    c.la = 1;
    c.a = 0;
    return c;
  }
  const int c1 = atom_level(I);
  const int Ln = not_level(I, k);
  if (Ln >= 0) {
    if (g < n[Ln]) { c.op = OP_NOT; c.la = Ln; c.a = g; return c; }
    g -= n[Ln];
  }
  for (int pass = 0; pass < 2; ++pass) {
    const int w = op_cost(I, pass ? OP_OR : OP_AND);
    for (int i = c1; 2 * i <= k - w; ++i) {
      const int j = k - w - i;
      const uint64_t cnt = n[i] * n[j];
      if (g < cnt) {
        c.op = pass ? OP_OR : OP_AND;
        c.la = i; c.lb = j;
        divmod64(g, n[j], c.a, c.b);
        return c;
      }
      g -= cnt;
    }
  }
  for (int op = OP_X; op <= OP_G; ++op) {
    const int L = k - op_cost(I, op);
    if (L < c1) continue;
    if (g < n[L]) { c.op = op; c.la = L; c.a = g; return c; }
    g -= n[L];
  }
  const int w = op_cost(I, OP_U);
  for (int i = c1; k - w - i >= c1; ++i) {
    const int j = k - w - i;
    const uint64_t cnt = n[i] * n[j];
    if (g < cnt) {
      c.op = OP_U; c.la = i; c.lb = j;
      divmod64(g, n[j], c.a, c.b);
      return c;
    }
    g -= cnt;
  }
  c.op = -1;
  c.la = 1;
  c.a = 0;
  return c;
}

// decode() for a candidate of the level being planned or built (k =
// I.level) with unit costs: the block is found by comparing g with the block
// bases the plan recorded (base_not, base_and / base_or by split, base_x,
// base_f, base_g, base_u by split), then one division splits a pair index.
// Same numbering as decode(); weighted levels take decode().
__device__ inline Cand decode_level(const InstDev& I, int k, uint64_t g) {
  if (I.weighted) return decode(I, k, g);
  const uint64_t* n = I.lcount;
  Cand c;
  c.lb = 0;
  c.b = 0;
  const int ns = (k - 1) / 2;   // & and | splits: left sizes 1..ns
  if (g < I.base_x) {
    if (ns == 0 || g < I.base_and[1]) {
      c.op = OP_NOT; c.la = k - 1; c.a = g - I.base_not;
      return c;
    }
    const bool orb = g >= I.base_or[1];
    const uint64_t* base = orb ? I.base_or : I.base_and;
    int i = 1;
    while (i < ns && g >= base[i + 1]) ++i;
    c.op = orb ? OP_OR : OP_AND;
    c.la = i;
    c.lb = k - 1 - i;
    divmod64(g - base[i], n[k - 1 - i], c.a, c.b);
    return c;
  }
  c.la = k - 1;
  if (g < I.base_f) { c.op = OP_X; c.a = g - I.base_x; return c; }
  if (g < I.base_g) { c.op = OP_F; c.a = g - I.base_f; return c; }
  if (k < 3 || g < I.base_u[1]) {
    if (g - I.base_g < n[k - 1]) { c.op = OP_G; c.a = g - I.base_g; return c; }
    c.op = -1; c.la = 1; c.a = 0;
    return c;
  }
  int i = 1;
  while (i < k - 2 && g >= I.base_u[i + 1]) ++i;
  c.op = OP_U;
  c.la = i;
  c.lb = k - 1 - i;
  divmod64(g - I.base_u[i], n[k - 1 - i], c.a, c.b);
  if (c.a >= n[i]) { c.op = -1; c.la = 1; c.a = 0; c.lb = 0; c.b = 0; }
  return c;
}

__device__ __forceinline__ const uint64_t* row_ptr(const InstDev& I, int lvl, uint64_t idx) {
  return I.rows + (I.lstart[lvl] + idx) * (uint64_t)I.TP;
}

template <int MODE>
__device__ inline void cand_key(const InstDev& I, const Cand& c, uint64_t& h, uint64_t& l) {
  const uint64_t* ra = row_ptr(I, c.la, c.a);
  const uint64_t* rb = (c.op == OP_AND || c.op == OP_OR || c.op == OP_U) ? row_ptr(I, c.lb, c.b) : ra;
  KeyAcc k;
  key_init(k);
  const int T = I.T, half = T / 2;
  for (int t = 0; t < T; ++t) {
    const uint64_t w = apply_w(c.op, ra[t], rb[t], I.len[t]);
    key_word<MODE>(k, w, t, half, I.off[t], I.width[t], I.stride1, I.len[t]);
  }
  key_final<MODE>(k, h, l);
}

__device__ inline void row_key(const InstDev& I, const uint64_t* row, uint64_t& h, uint64_t& l) {
  KeyAcc k;
  key_init(k);
  const int T = I.T, half = T / 2;
  switch (I.key_mode) {
    case KEY_HASH:
      for (int t = 0; t < T; ++t) key_word<KEY_HASH>(k, row[t], t, half, 0, 0, 0, 0);
      key_final<KEY_HASH>(k, h, l);
      break;
    case KEY_SAMPLED:
      for (int t = 0; t < T; ++t)
        key_word<KEY_SAMPLED>(k, row[t], t, half, I.off[t], I.width[t], I.stride1, I.len[t]);
      key_final<KEY_SAMPLED>(k, h, l);
      break;
    default:
      for (int t = 0; t < T; ++t)
        key_word<KEY_CONCAT>(k, row[t], t, half, I.off[t], I.width[t], 0, I.len[t]);
      key_final<KEY_CONCAT>(k, h, l);
  }
}

// ======================================================================= P1
// Shared per-tile parameters.
struct TileSh {
  unsigned long long tile;
  int inst, grp, k, T, TP, half, stride, mode, skip;
  int kind, mask;   // operand group: 0 unary / 1 binary; the operators it evaluates
  int otf;          // on-the-fly level: solution test only, nothing inserted
  int nolist;       // new slots are not listed (the table scan reads the whole table)
  uint64_t s0, q0, nS, nQ, ni, nj;
  int si, qi;   // levels of the stream / staged operand
  int qleft;    // staged operand is the left operand of & | and of U(i->j)
  int i, j, tq;
  uint64_t pos[2];   // bit t: trace t is positive
  uint8_t len[kMaxTraces], off[kMaxTraces], wid[kMaxTraces];
};

// Copy nrows consecutive rows (pitch TP words) into shared memory with pitch
// sp, one 8-byte asynchronous copy per word (cp.async: no registers held, every
// copy of the tile in flight at once); stage_wait() completes them.  Rows
// with an odd pitch are only 8-byte aligned, hence 8-byte copies.
__device__ __forceinline__ void stage_rows(uint64_t* dst, int sp, const uint64_t* src, int nrows, int TP) {
  const int n = nrows * TP;
  const int dr = blockDim.x / TP, dc = blockDim.x - dr * TP;
  int r = threadIdx.x / TP, c = threadIdx.x - r * TP;
  for (int w = threadIdx.x; w < n; w += blockDim.x) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(dst + r * sp + c);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(src + w) : "memory");
    r += dr;
    c += dc;
    if (c >= TP) { c -= TP; ++r; }
  }
}

__device__ __forceinline__ void stage_wait() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

struct P1Count {
  unsigned long long fresh, fail, sol;   // keys inserted, probe failures, min solution candidate
};

// Insert N keys of one thread: all home-slot loads are issued first, then the
// keys are resolved one by one.  bad[j] == 0 marks a candidate whose step-0
// bits match every trace's label (a solution candidate).
template <int N>
__device__ __forceinline__ void insert_group(InstDev& I, unsigned live, int k, const uint64_t* h,
                                             const uint64_t* l, const uint64_t* g, const uint32_t* bad,
                                             P1Count& cnt, unsigned valid, bool list) {
  Slot* tab = I.table;
  const uint64_t mask = I.table_mask;
  uint64_t idx[N];
  Key128 cur[N];
#pragma unroll
  for (int j = 0; j < N; ++j) idx[j] = slot_hash(h[j], l[j]) & mask;
#pragma unroll
  for (int j = 0; j < N; ++j) cur[j] = ld_key(tab + idx[j]);
  uint64_t fresh[N];
  int nf = 0;
#pragma unroll
  for (int j = 0; j < N; ++j) {
    if (!((valid >> j) & 1u)) continue;
    int isnew = 0;
    const int r = insert_min(tab, mask, idx[j], cur[j], h[j], l[j], pay_of(k, g[j]), isnew);
    if (r < 0) ++cnt.fail;
    if (isnew) fresh[nf++] = idx[j];
    if (!bad[j] && g[j] < cnt.sol) cnt.sol = g[j];
  }
  cnt.fresh += nf;
  if (!list) return;   // (warp-uniform)
  // list the slots of the keys this warp inserted: one atomic per warp, the
  // per-lane offsets from three ballots of the lane's count (0..4)
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  const unsigned b0 = __ballot_sync(live, nf & 1), b1 = __ballot_sync(live, nf & 2),
                 b2 = __ballot_sync(live, nf & 4);
  const unsigned pre = __popc(b0 & lt) + 2 * __popc(b1 & lt) + 4 * __popc(b2 & lt);
  const unsigned tot = __popc(b0) + 2 * __popc(b1) + 4 * __popc(b2);
  const int leader = __ffs(live) - 1;
  unsigned long long base = 0;
  if (lane == leader && tot) base = atomicAdd(&I.n_newlist, (unsigned long long)tot);
  base = __shfl_sync(live, base, leader);
  for (int r = 0; r < nf; ++r) {
    const unsigned long long pos = base + pre + r;
    if (pos < I.tent_cap) I.wins[pos] = fresh[r];
  }
}

__device__ __forceinline__ uint64_t pos_bit(const TileSh& P, int t) {
  return (P.pos[t >> 6] >> (t & 63)) & 1ULL;
}

// Compile-time half of a trace index: HASH keys fold traces t < T/2 into h,
// the others into l (LTL_BS.cu:30-110), so the P1 loops run the two halves
// as separate loops and pick the accumulator statically.
template <bool HI>
struct Half {
  static constexpr bool hi = HI;
  static constexpr bool fixed = true;
};
// The half decided at run time (rotated word order of the bulk-staged tiles).
struct HalfRt {
  bool hi;
  static constexpr bool fixed = false;
};

template <int MODE, bool HI>
__device__ __forceinline__ void key_word_h(KeyAcc& k, uint64_t w, int t, int off, int width, int stride, int L) {
  if (MODE == KEY_HASH) {
    const uint64_t x = splitmix_fin(w);
    if (HI) k.a1 ^= x; else k.a0 ^= x;
  } else {
    key_word<MODE>(k, w, t, 0, off, width, stride, L);
  }
}

template <int MODE, typename H>
__device__ __forceinline__ void key_word_any(KeyAcc& k, uint64_t w, int t, H half, int off, int width, int stride,
                                             int L) {
  if constexpr (H::fixed) {
    key_word_h<MODE, H::hi>(k, w, t, off, width, stride, L);
  } else if (MODE == KEY_HASH) {
    const uint64_t x = splitmix_fin(w), m = half.hi ? ~0ULL : 0ULL;
    k.a1 ^= x & m;
    k.a0 ^= x & ~m;
  } else {
    key_word<MODE>(k, w, t, 0, off, width, stride, L);
  }
}

// The trace words of a tile row in the order a thread visits them.  Copied
// rows (odd pitch): 0..T-1, the words below T/2 first (the hash folds the two
// halves into different words, chosen at compile time).  Bulk-staged rows
// (pitch TP, even): lane l starts at word l mod T and wraps, so the 16 lanes
// of a shared-memory wavefront read 16 different banks; the half is then
// decided per word.
template <bool BULK, typename F>
__device__ __forceinline__ void p1_words(const TileSh& P, F&& body) {
  if (!BULK) {
    for (int t = 0; t < P.half; ++t) body(t, Half<true>{});
    for (int t = P.half; t < P.T; ++t) body(t, Half<false>{});
  } else {
    int t = (threadIdx.x & 31) % P.T;
    for (int i = 0; i < P.T; ++i) {
      body(t, HalfRt{t < P.half});
      if (++t == P.T) t = 0;
    }
  }
}

// Solution test accumulators: only bit 0 (step 0) of a word is compared
// with the trace's label, so 32 bits carry the whole test.
__device__ __forceinline__ uint32_t lo32(uint64_t w) { return (uint32_t)w; }

// Step 0 of ~w, X w, F w and G w on one trace word (length mask lm) against
// the trace's label: bit o set (o = ~ X F G) where it differs.  The same
// bits as the P1 tests of ~w & lm, w >> 1, w_fin(w) and w_glob(w, lm); a row
// whose bits stay clear over every trace makes that operator's candidate on
// it a solution.
__device__ __forceinline__ unsigned unary_miss(uint64_t w, uint64_t lm, unsigned lab) {
  const unsigned n0 = (unsigned)(~w & lm) & 1u;
  const unsigned x0 = (unsigned)(w >> 1) & 1u;
  const unsigned f0 = w != 0 ? 1u : 0u;
  const unsigned g0 = ((w & 1ULL) != 0 && (~w & lm) == 0) ? 1u : 0u;
  return (n0 ^ lab) | ((x0 ^ lab) << 1) | ((f0 ^ lab) << 2) | ((g0 ^ lab) << 3);
}

// The step-0 tests of k_emit on one word of a row, trace lengths being at
// least 1 (so ~w passes exactly where w fails, and G w at step 0 is the word
// covering the whole trace): bit 0 = the row's own test missed, bits 1-4 =
// X, F, G, ~ missed.  OR-ed over the words they are the row's miss bits.
__device__ __forceinline__ unsigned emit_miss(uint64_t w, uint64_t lm, unsigned lab) {
  const unsigned x = ((unsigned)w ^ (lab ? 3u : 0u)) & 3u;
  const unsigned nz = w != 0 ? 1u : 0u;
  const unsigned fu = (~w & lm) == 0 ? 1u : 0u;
  return x | ((nz ^ lab) << 2) | ((fu ^ lab) << 3) | ((~x & 1u) << 4);
}

// Records row `row` of level k as the first one found so far whose ~ X F G
// candidates pass the sample, for the operators whose miss bits are clear.
__device__ __forceinline__ void record_unary(InstDev& I, int k, uint64_t row, unsigned miss) {
  if ((miss & 0xFu) == 0xFu || row >= 0xFFFFFFFFull) return;
  const unsigned v = (unsigned)(0xFFFFFFFFull - row);
#pragma unroll
  for (int o = 0; o < 4; ++o)
    if (!((miss >> o) & 1u)) atomicMax(&I.uhit[k][o], v);
}

// BULK: rows staged by one bulk copy at the even pitch TP (rotated word
// order), else by 8-byte copies at the odd pitch TP + 1.
// NU: the operators computed, ~ alone (1: every other one lies past the
// level's first solution) or ~ X F G (4; the inserted ones are P.mask).
template <int MODE, bool BULK, int NU>
__device__ inline void p1_unary(InstDev& I, const TileSh& P, const uint64_t* sS, int sp, P1Count& cnt) {
  const uint64_t a = P.s0 + threadIdx.x;
  const unsigned live = __ballot_sync(0xffffffffu, a < P.nS);
  if (a >= P.nS) return;
  const uint64_t* srow = sS + threadIdx.x * sp;
  KeyAcc k0, k1, k2, k3;
  key_init(k0);
  if (NU == 4) { key_init(k1); key_init(k2); key_init(k3); }
  uint32_t bad[4] = {0, 0, 0, 0};
  auto body = [&](int t, auto half) {
    const uint64_t w = srow[t];
    const int L = P.len[t], off = P.off[t], wd = P.wid[t];
    const uint64_t lm = len_mask(L);
    const uint32_t pb = (uint32_t)pos_bit(P, t);
    const uint64_t w0 = ~w & lm;
    bad[0] |= lo32(w0) ^ pb;
    key_word_any<MODE>(k0, w0, t, half, off, wd, P.stride, L);
    if (NU == 4) {
      const uint64_t w1 = w >> 1, w2 = w_fin(w), w3 = w_glob(w, lm);
      bad[1] |= lo32(w1) ^ pb;
      bad[2] |= lo32(w2) ^ pb;
      bad[3] |= lo32(w3) ^ pb;
      key_word_any<MODE>(k1, w1, t, half, off, wd, P.stride, L);
      key_word_any<MODE>(k2, w2, t, half, off, wd, P.stride, L);
      key_word_any<MODE>(k3, w3, t, half, off, wd, P.stride, L);
    }
  };
  p1_words<BULK>(P, body);
  uint64_t h[4], l[4], g[4];
  key_final<MODE>(k0, h[0], l[0]);
  g[0] = I.base_not + a;
  if (NU == 4) {
    key_final<MODE>(k1, h[1], l[1]);
    key_final<MODE>(k2, h[2], l[2]);
    key_final<MODE>(k3, h[3], l[3]);
    g[1] = I.base_x + a;
    g[2] = I.base_f + a;
    g[3] = I.base_g + a;
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) bad[j] &= 1u;
  insert_group<NU>(I, live, P.k, h, l, g, bad, cnt, (unsigned)P.mask, !P.nolist);
}

// KEYS: the operators computed, a prefix of (&, |, laUlb, lbUla) as bits
// 3, 7, 15; the inserted ones are P.mask within it.
template <int MODE, int KEYS, bool BULK>
__device__ inline void p1_binary(InstDev& I, const TileSh& P, const uint64_t* sS, int sp, const uint64_t* sQ,
                          P1Count& cnt) {
  constexpr bool kO = (KEYS & 2) != 0, kU = (KEYS & 4) != 0, kV = (KEYS & 8) != 0;
  constexpr int N = 1 + (kO ? 1 : 0) + (kU ? 1 : 0) + (kV ? 1 : 0);
  const uint64_t s = P.s0 + threadIdx.x;
  const unsigned live = __ballot_sync(0xffffffffu, s < P.nS);
  if (s >= P.nS) return;
  const uint64_t* srow = sS + threadIdx.x * sp;
  const int nq = (int)((P.nQ - P.q0) < (uint64_t)P.tq ? (P.nQ - P.q0) : (uint64_t)P.tq);
  for (int q = 0; q < nq; ++q) {
    const uint64_t* qrow = sQ + q * P.TP;
    KeyAcc kA, kOr, kUn, kVn;
    key_init(kA);
    if (kO) key_init(kOr);
    if (kU) key_init(kUn);
    if (kV) key_init(kVn);
    uint32_t bad[4] = {0, 0, 0, 0};
    auto body = [&](int t, auto half) {
      const uint64_t qw = qrow[t], sw = srow[t];
      const uint64_t la = P.qleft ? qw : sw, lb = P.qleft ? sw : qw;
      const int L = P.len[t], off = P.off[t], wd = P.wid[t];
      const uint32_t pb = (uint32_t)pos_bit(P, t);
      const uint64_t wa = la & lb;
      bad[0] |= lo32(wa) ^ pb;
      key_word_any<MODE>(kA, wa, t, half, off, wd, P.stride, L);
      if (kO) {
        const uint64_t wo = la | lb;
        bad[1] |= lo32(wo) ^ pb;
        key_word_any<MODE>(kOr, wo, t, half, off, wd, P.stride, L);
      }
      if (kU) {
        const uint64_t wu = w_until(la, lb);
        bad[2] |= lo32(wu) ^ pb;
        key_word_any<MODE>(kUn, wu, t, half, off, wd, P.stride, L);
      }
      if (kV) {
        const uint64_t wv = w_until(lb, la);
        bad[3] |= lo32(wv) ^ pb;
        key_word_any<MODE>(kVn, wv, t, half, off, wd, P.stride, L);
      }
    };
    p1_words<BULK>(P, body);
    const uint64_t a = P.qleft ? P.q0 + q : s;     // index in level i
    const uint64_t b = P.qleft ? s : P.q0 + q;     // index in level j
    const uint64_t ab = a * P.nj + b;
    uint64_t h[4], l[4], g[4];
    key_final<MODE>(kA, h[0], l[0]);
    g[0] = I.base_and[P.i] + ab;
    if (kO) { key_final<MODE>(kOr, h[1], l[1]); g[1] = I.base_or[P.i] + ab; }
    if (kU) { key_final<MODE>(kUn, h[2], l[2]); g[2] = I.base_u[P.i] + ab; }
    if (kV) { key_final<MODE>(kVn, h[3], l[3]); g[3] = I.base_u[P.j] + b * P.ni + a; }
#pragma unroll
    for (int j = 0; j < 4; ++j) bad[j] &= 1u;
    insert_group<N>(I, live, P.k, h, l, g, bad, cnt, (unsigned)P.mask & (unsigned)KEYS, !P.nolist);
  }
}

template <int MODE, bool BULK>
__device__ inline void p1_binary_keys(int keys, InstDev& I, const TileSh& P, const uint64_t* sS, int sp,
                                      const uint64_t* sQ, P1Count& cnt) {
  switch (keys) {
    case 15: p1_binary<MODE, 15, BULK>(I, P, sS, sp, sQ, cnt); break;
    case 7: p1_binary<MODE, 7, BULK>(I, P, sS, sp, sQ, cnt); break;
    // & alone is computed with | (one variant less: a smaller kernel image
    // measured faster on small levels)
    default: p1_binary<MODE, 3, BULK>(I, P, sS, sp, sQ, cnt);
  }
}

// On-the-fly level (nothing stored): the tile's candidates get the solution
// test alone, step 0 of every trace against its label; no key, no insert.
template <bool BULK>
__device__ inline void p1_solutions(InstDev& I, const TileSh& P, const uint64_t* sS, int sp, const uint64_t* sQ,
                                    P1Count& cnt) {
  const uint64_t s = P.s0 + threadIdx.x;
  if (s >= P.nS) return;
  const uint64_t* srow = sS + threadIdx.x * sp;
  if (P.kind == 0) {
    uint32_t bad[4] = {0, 0, 0, 0};
    p1_words<BULK>(P, [&](int t, auto) {
      const uint64_t w = srow[t], lm = len_mask(P.len[t]);
      const uint32_t pb = (uint32_t)pos_bit(P, t);
      bad[0] |= lo32(~w & lm) ^ pb;
      bad[1] |= lo32(w >> 1) ^ pb;
      bad[2] |= lo32(w_fin(w)) ^ pb;
      bad[3] |= lo32(w_glob(w, lm)) ^ pb;
    });
    const uint64_t g[4] = {I.base_not + s, I.base_x + s, I.base_f + s, I.base_g + s};
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (((P.mask >> j) & 1) && !(bad[j] & 1u) && g[j] < cnt.sol) cnt.sol = g[j];
    return;
  }
  const int nq = (int)((P.nQ - P.q0) < (uint64_t)P.tq ? (P.nQ - P.q0) : (uint64_t)P.tq);
  for (int q = 0; q < nq; ++q) {
    const uint64_t* qrow = sQ + q * P.TP;
    uint32_t bad[4] = {0, 0, 0, 0};
    p1_words<BULK>(P, [&](int t, auto) {
      const uint64_t qw = qrow[t], sw = srow[t];
      const uint64_t la = P.qleft ? qw : sw, lb = P.qleft ? sw : qw;
      const uint32_t pb = (uint32_t)pos_bit(P, t);
      bad[0] |= lo32(la & lb) ^ pb;
      bad[1] |= lo32(la | lb) ^ pb;
      bad[2] |= lo32(w_until(la, lb)) ^ pb;
      bad[3] |= lo32(w_until(lb, la)) ^ pb;
    });
    const uint64_t a = P.qleft ? P.q0 + q : s, b = P.qleft ? s : P.q0 + q;
    const uint64_t ab = a * P.nj + b;
    const uint64_t g[4] = {I.base_and[P.i] + ab, I.base_or[P.i] + ab, I.base_u[P.i] + ab, I.base_u[P.j] + b * P.ni + a};
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (((P.mask >> j) & 1) && !(bad[j] & 1u) && g[j] < cnt.sol) cnt.sol = g[j];
  }
}

// Warp per candidate, lane per trace word: the two operand rows are read
// coalesced, every lane folds its words into a partial key, and the partial
// keys are combined with XOR shuffles (hash mode XOR-folds by definition; the
// bit fields of the other modes are disjoint, so XOR equals OR).
template <int MODE>
__device__ __forceinline__ void warp_key(const InstDev& I, const Cand& c, int lane, uint64_t& h, uint64_t& l) {
  const uint64_t* ra = row_ptr(I, c.la, c.a);
  const uint64_t* rb = (c.op == OP_AND || c.op == OP_OR || c.op == OP_U) ? row_ptr(I, c.lb, c.b) : ra;
  KeyAcc k;
  key_init(k);
  const int T = I.T, half = T / 2;
  for (int t = lane; t < T; t += 32) {
    const uint64_t w = apply_w(c.op, __ldcg(ra + t), __ldcg(rb + t), I.len[t]);
    key_word<MODE>(k, w, t, half, I.off[t], I.width[t], I.stride1, I.len[t]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    k.a0 ^= __shfl_xor_sync(0xffffffffu, k.a0, o);
    k.a1 ^= __shfl_xor_sync(0xffffffffu, k.a1, o);
  }
  key_final<MODE>(k, h, l);
}

// RPN of the node (level lvl, candidate g) into I.rpn (postfix).
// RPN of candidate g of level lvl, rebuilt through the operands' canonical
// indices (origin); returns its length (0 if it does not fit cap).
__device__ inline int reconstruct_to(const InstDev& I, int lvl, uint64_t g, int16_t* rpn, int cap) {
  struct Fr { int lvl; uint64_t g; int state; };
  Fr st[2 * kMaxSize + 2];
  int sp = 0, out = 0;
  st[0] = {lvl, g, 0};
  while (sp >= 0) {
    if (out >= cap) return 0;
    Fr& f = st[sp];
    if (f.lvl <= atom_level(I)) {
      rpn[out++] = (int16_t)f.g;
      --sp;
      continue;
    }
    const Cand c = decode(I, f.lvl, f.g);
    if (c.op < 0) return 0;
    const bool bin = (c.op == OP_AND || c.op == OP_OR || c.op == OP_U);
    if (f.state == 0) {
      f.state = 1;
      st[++sp] = {c.la, I.origin[I.lstart[c.la] + c.a], 0};
    } else if (f.state == 1 && bin) {
      f.state = 2;
      st[++sp] = {c.lb, I.origin[I.lstart[c.lb] + c.b], 0};
    } else {
      rpn[out++] = (int16_t)(-(1 + c.op));
      --sp;
    }
  }
  return out;
}

__device__ inline void reconstruct(InstDev& I, int lvl, uint64_t g) {
  I.rpn_len = reconstruct_to(I, lvl, g, I.rpn, kMaxSize);
}

}  // namespace vfb
