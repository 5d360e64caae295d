// vfb_kernels.cu -- sm_100a kernels of one level step of the cached search.
//
// One level k is built by this launch sequence (every kernel reads its work
// from device memory, so the same sequence serves every level and any number
// of instances):
//
//   k_plan        per instance: candidate-block bases of level k, P1 tiling,
//                 buffer checks                         (LTL_BS.cu:1226-1488)
//   k_p1          every candidate: operator words -> 126-bit key -> insert
//                 into the instance's hash set with atomicMin on the
//                 candidate's canonical index; candidates that may own their
//                 key set a bit in the tentative bitmap
//                 (applyOperator LTL_BS.cu:183-238, makeRlxUnqChkCSs 30-110,
//                  processUniqueCS 251-269)
//   k_chunk_*     order-preserving compaction of the bitmap into the
//                 ascending list of tentative candidates (count/scan/emit)
//   k_verify      a tentative candidate owns its key iff the key's final
//                 payload is its own index -> winner bitmap
//   k_chunk_*     compaction of winners (ascending candidate index)
//   k_emit_rows   winner rows appended to the level cache in canonical order;
//                 solution test (insertInCache LTL_BS.cu:299-329)
//   k_finish      level bookkeeping, formula reconstruction (LTL_BS.cu:561-705)
//
// The reference's thrust::remove/copy_n compaction (storeUniqueLTLs
// LTL_BS.cu:489-530) is replaced by the bitmap compaction; its racy
// atomicCAS winners (LTL_BS.cu:319, hash_set.cuh:232) by min-index ownership.
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
__device__ int insert_min(Slot* tab, uint64_t mask, uint64_t idx, Key128 cur, uint64_t h, uint64_t l,
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
        isnew = 1;
        return claim(tab + idx, pay);
      }
      if (old.h == h && old.l == l) return claim(tab + idx, pay);
    }
    idx = (idx + 1) & mask;
  }
  return -1;
}

// Payload of (h,l), or ~0 if the key is absent.
__device__ unsigned long long find_pay(const Slot* tab, uint64_t mask, uint64_t h, uint64_t l) {
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
__device__ unsigned long long block_excl_scan(unsigned long long v, unsigned long long* s_warp,
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

// Canonical candidate index g of level k -> operator and operands (levels and
// indices within them).  Block order ~ & | X F G U; & and | over left sizes
// 1..floor((k-1)/2), U over 1..k-2; left index major (ltl_nocache.cu:169-224).
__device__ Cand decode(const InstDev& I, int k, uint64_t g) {
  const uint64_t* n = I.lcount;
  Cand c;
  c.lb = 0;
  c.b = 0;
  const uint64_t un = n[k - 1];
  if (g < un) { c.op = OP_NOT; c.la = k - 1; c.a = g; return c; }
  g -= un;
  for (int pass = 0; pass < 2; ++pass) {
    for (int i = 1; 2 * i <= k - 1; ++i) {
      const int j = k - 1 - i;
      const uint64_t cnt = n[i] * n[j];
      if (g < cnt) {
        c.op = pass ? OP_OR : OP_AND;
        c.la = i; c.lb = j; c.a = g / n[j]; c.b = g % n[j];
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
      c.op = OP_U; c.la = i; c.lb = j; c.a = g / n[j]; c.b = g % n[j];
      return c;
    }
    g -= cnt;
  }
  c.op = -1;
  c.la = 1;
  c.a = 0;
  return c;
}

__device__ __forceinline__ const uint64_t* row_ptr(const InstDev& I, int lvl, uint64_t idx) {
  return I.rows + (I.lstart[lvl] + idx) * (uint64_t)I.TP;
}

template <int MODE>
__device__ void cand_key(const InstDev& I, const Cand& c, uint64_t& h, uint64_t& l) {
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

__device__ void row_key(const InstDev& I, const uint64_t* row, uint64_t& h, uint64_t& l) {
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

// ===================================================================== plan
__global__ void k_plan(BatchDev* Bp) {
  const BatchDev B = *Bp;
  for (int b = threadIdx.x; b < B.ninst; b += blockDim.x) {
    InstDev& I = B.inst[b];
    unsigned long long tiles = 0, chunks = 0;
    if (I.status == ST_RUNNING) {
      const int k = I.level;
      const uint64_t* n = I.lcount;
      I.lstart[k] = I.lstart[k - 1] + n[k - 1];
      uint64_t g = 0;
      I.base_not = g;
      g += n[k - 1];
      for (int i = 1; 2 * i <= k - 1; ++i) { I.base_and[i] = g; g += n[i] * n[k - 1 - i]; }
      for (int i = 1; 2 * i <= k - 1; ++i) { I.base_or[i] = g; g += n[i] * n[k - 1 - i]; }
      I.base_x = g; g += n[k - 1];
      I.base_f = g; g += n[k - 1];
      I.base_g = g; g += n[k - 1];
      for (int i = 1; i <= k - 2; ++i) { I.base_u[i] = g; g += n[i] * n[k - 1 - i]; }
      I.cands = g;
      // P1 tiling: kTS stream rows x tq staged rows per tile; small levels get
      // shorter tiles so that they still spread over every SM
      uint64_t t = 0;
      int tq = kTQ;
      for (;;) {
        t = (n[k - 1] + kTS - 1) / kTS;
        I.grp_prefix[0] = 0;
        I.grp_prefix[1] = t;
        for (int i = 1; i < kGroups; ++i) {
          if (2 * i <= k - 1) {
            const int j = k - 1 - i;
            const bool qleft = (i == j) || (n[i] <= n[j]);
            const uint64_t nS = qleft ? n[j] : n[i], nQ = qleft ? n[i] : n[j];
            const uint64_t qt = (nQ + tq - 1) / tq, st = (nS + kTS - 1) / kTS;
            I.grp_qtiles[i] = (uint32_t)qt;
            t += st * qt;
          }
          I.grp_prefix[i + 1] = t;
        }
        if (t >= (uint64_t)kP1TileTarget || tq == 1) break;
        tq >>= 1;
      }
      I.tq = tq;
      const uint64_t words = (g + 31) / 32;
      const uint64_t cap = I.table_mask + 1;
      // new keys of this level: at most all candidates; expect ~8x growth
      const uint64_t grow = 8 * n[k - 1] + 4096;
      const uint64_t est = g < grow ? g : grow;
      int need = 0;
      if (g >= (1ULL << kPayShift)) need |= NEED_LIMIT;
      if (words > I.bitmap_words) { need |= NEED_BITMAP; I.need_amount[0] = words; }
      if (2 * (I.keys + est) > cap) { need |= NEED_TABLE; I.need_amount[1] = 4 * (I.keys + est); }
      if (I.lstart[k] + est > I.row_cap) { need |= NEED_ROWS; I.need_amount[3] = I.lstart[k] + est; }
      if (est > I.tent_cap) { need |= NEED_TENT; I.need_amount[2] = est; }
      if (need) {
        I.status = ST_NEED_MEM;
        I.need = need;
      } else {
        tiles = t;
        chunks = (words + kChunkWords - 1) / kChunkWords;
        I.n_tent = I.n_new = I.n_wins = I.probe_fail = 0;
        I.best_sol = ~0ULL;
      }
    }
    B.p1_prefix[b + 1] = tiles;
    B.chunk_prefix0[b + 1] = chunks;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    B.p1_prefix[0] = 0;
    B.chunk_prefix0[0] = 0;
    for (int b = 0; b < B.ninst; ++b) {
      B.p1_prefix[b + 1] += B.p1_prefix[b];
      B.chunk_prefix0[b + 1] += B.chunk_prefix0[b];
    }
    for (int i = 0; i < 4; ++i) B.tickets[i] = 0;
  }
}

// ======================================================================= P1
// Shared per-tile parameters.
struct TileSh {
  unsigned long long tile;
  int inst, grp, k, T, TP, half, stride, mode, skip;
  uint64_t s0, q0, nS, nQ, ni, nj;
  int si, qi;   // levels of the stream / staged operand
  int qleft;    // staged operand is the left operand of & | and of U(i->j)
  int i, j, tq;
  uint8_t len[kMaxTraces], off[kMaxTraces], wid[kMaxTraces];
};

// Copy nrows consecutive rows (pitch TP words, 16-byte aligned) into shared
// memory with pitch sp, as 128-bit coalesced loads.
__device__ __forceinline__ void stage_rows(uint64_t* dst, int sp, const uint64_t* src, int nrows, int TP) {
  const int n2 = nrows * TP / 2;
  const ulonglong2* s2 = reinterpret_cast<const ulonglong2*>(src);
  for (int u = threadIdx.x; u < n2; u += blockDim.x) {
    const ulonglong2 v = __ldg(s2 + u);
    const int w = 2 * u, r = w / TP, c = w - r * TP;
    dst[r * sp + c] = v.x;
    dst[r * sp + c + 1] = v.y;
  }
}

struct P1Count {
  unsigned long long tent, fresh, fail;
};

template <int N>
__device__ __forceinline__ void insert_group(InstDev& I, Slot* tab, uint64_t mask, int k, const uint64_t* h,
                                             const uint64_t* l, const uint64_t* g, P1Count& cnt) {
  uint64_t idx[N];
  Key128 cur[N];
#pragma unroll
  for (int j = 0; j < N; ++j) idx[j] = slot_hash(h[j], l[j]) & mask;
#pragma unroll
  for (int j = 0; j < N; ++j) cur[j] = ld_key(tab + idx[j]);
#pragma unroll
  for (int j = 0; j < N; ++j) {
    int isnew = 0;
    const int r = insert_min(tab, mask, idx[j], cur[j], h[j], l[j], pay_of(k, g[j]), isnew);
    if (r > 0) {
      atomicOr(I.bitmap + (g[j] >> 5), 1u << (g[j] & 31));
      ++cnt.tent;
    } else if (r < 0) {
      ++cnt.fail;
    }
    cnt.fresh += isnew;
  }
}

template <int MODE>
__device__ void p1_unary(InstDev& I, const TileSh& P, const uint64_t* sS, int sp, P1Count& cnt) {
  const uint64_t a = P.s0 + threadIdx.x;
  if (a >= P.nS) return;
  const uint64_t* srow = sS + threadIdx.x * sp;
  KeyAcc k0, k1, k2, k3;
  key_init(k0); key_init(k1); key_init(k2); key_init(k3);
  for (int t = 0; t < P.T; ++t) {
    const uint64_t w = srow[t];
    const int L = P.len[t], off = P.off[t], wd = P.wid[t];
    const uint64_t lm = len_mask(L);
    key_word<MODE>(k0, ~w & lm, t, P.half, off, wd, P.stride, L);
    key_word<MODE>(k1, w >> 1, t, P.half, off, wd, P.stride, L);
    key_word<MODE>(k2, w_fin(w), t, P.half, off, wd, P.stride, L);
    key_word<MODE>(k3, w_glob(w, lm), t, P.half, off, wd, P.stride, L);
  }
  uint64_t h[4], l[4], g[4];
  key_final<MODE>(k0, h[0], l[0]);
  key_final<MODE>(k1, h[1], l[1]);
  key_final<MODE>(k2, h[2], l[2]);
  key_final<MODE>(k3, h[3], l[3]);
  g[0] = I.base_not + a;
  g[1] = I.base_x + a;
  g[2] = I.base_f + a;
  g[3] = I.base_g + a;
  insert_group<4>(I, I.table, I.table_mask, P.k, h, l, g, cnt);
}

template <int MODE, bool FOUR>
__device__ void p1_binary(InstDev& I, const TileSh& P, const uint64_t* sS, int sp, const uint64_t* sQ,
                          P1Count& cnt) {
  const uint64_t s = P.s0 + threadIdx.x;
  if (s >= P.nS) return;
  const uint64_t* srow = sS + threadIdx.x * sp;
  const int nq = (int)((P.nQ - P.q0) < (uint64_t)P.tq ? (P.nQ - P.q0) : (uint64_t)P.tq);
  for (int q = 0; q < nq; ++q) {
    const uint64_t* qrow = sQ + q * P.TP;
    KeyAcc kA, kO, kU, kV;
    key_init(kA); key_init(kO); key_init(kU); key_init(kV);
    for (int t = 0; t < P.T; ++t) {
      const uint64_t qw = qrow[t], sw = srow[t];
      const uint64_t la = P.qleft ? qw : sw, lb = P.qleft ? sw : qw;
      const int L = P.len[t], off = P.off[t], wd = P.wid[t];
      key_word<MODE>(kA, la & lb, t, P.half, off, wd, P.stride, L);
      key_word<MODE>(kO, la | lb, t, P.half, off, wd, P.stride, L);
      key_word<MODE>(kU, w_until(la, lb), t, P.half, off, wd, P.stride, L);
      if (FOUR) key_word<MODE>(kV, w_until(lb, la), t, P.half, off, wd, P.stride, L);
    }
    const uint64_t a = P.qleft ? P.q0 + q : s;     // index in level i
    const uint64_t b = P.qleft ? s : P.q0 + q;     // index in level j
    uint64_t h[4], l[4], g[4];
    key_final<MODE>(kA, h[0], l[0]);
    key_final<MODE>(kO, h[1], l[1]);
    key_final<MODE>(kU, h[2], l[2]);
    const uint64_t ab = a * P.nj + b;
    g[0] = I.base_and[P.i] + ab;
    g[1] = I.base_or[P.i] + ab;
    g[2] = I.base_u[P.i] + ab;
    if (FOUR) {
      key_final<MODE>(kV, h[3], l[3]);
      g[3] = I.base_u[P.j] + b * P.ni + a;
      insert_group<4>(I, I.table, I.table_mask, P.k, h, l, g, cnt);
    } else {
      insert_group<3>(I, I.table, I.table_mask, P.k, h, l, g, cnt);
    }
  }
}

__global__ void __launch_bounds__(kTS) k_p1(BatchDev* Bp) {
  extern __shared__ __align__(16) uint64_t smem[];
  __shared__ TileSh P;
  __shared__ unsigned long long s_red[3][kTS / 32];
  const BatchDev B = *Bp;
  const unsigned long long total = B.p1_prefix[B.ninst];
  while (true) {
    if (threadIdx.x == 0) {
      const unsigned long long tile = atomicAdd(B.tickets, 1ULL);
      P.tile = tile;
      if (tile < total) {
        const int b = find_owner(B.p1_prefix, B.ninst, tile);
        InstDev& I = B.inst[b];
        const uint64_t local = tile - B.p1_prefix[b];
        int grp = 0;
        while (grp + 1 < kGroups && I.grp_prefix[grp + 1] <= local) ++grp;
        const int k = I.level;
        P.inst = b;
        P.grp = grp;
        P.k = k;
        P.T = I.T;
        P.TP = I.TP;
        P.half = I.T / 2;
        P.stride = I.stride1;
        P.mode = I.key_mode;
        P.tq = I.tq;
        // give up early once the table is known to be too small for this level
        const unsigned long long cap = I.table_mask + 1;
        P.skip = (*(volatile unsigned long long*)&I.probe_fail != 0) ||
                 (4 * (I.keys + *(volatile unsigned long long*)&I.n_new) > 3 * cap);
        const uint64_t within = local - I.grp_prefix[grp];
        if (grp == 0) {
          P.si = k - 1;
          P.nS = I.lcount[k - 1];
          P.s0 = within * kTS;
        } else {
          const int i = grp, j = k - 1 - i;
          const uint64_t ni = I.lcount[i], nj = I.lcount[j];
          const int qleft = (i == j) || (ni <= nj);
          P.i = i;
          P.j = j;
          P.ni = ni;
          P.nj = nj;
          P.qleft = qleft;
          P.si = qleft ? j : i;
          P.qi = qleft ? i : j;
          P.nS = qleft ? nj : ni;
          P.nQ = qleft ? ni : nj;
          const uint64_t qt = I.grp_qtiles[grp];
          P.s0 = (within / qt) * kTS;
          P.q0 = (within % qt) * I.tq;
        }
      }
    }
    __syncthreads();
    if (P.tile >= total) break;
    InstDev& I = B.inst[P.inst];
    for (int t = threadIdx.x; t < P.T; t += blockDim.x) {
      P.len[t] = I.len[t];
      P.off[t] = I.off[t];
      P.wid[t] = I.width[t];
    }
    const int sp = P.TP + 1;                      // odd pitch: conflict-free row reads
    uint64_t* sS = smem;
    uint64_t* sQ = smem + kTS * sp;
    P1Count cnt{0, 0, 0};
    if (!P.skip) {
      const int ns = (int)((P.nS - P.s0) < (uint64_t)kTS ? (P.nS - P.s0) : (uint64_t)kTS);
      stage_rows(sS, sp, row_ptr(I, P.si, P.s0), ns, P.TP);
      if (P.grp > 0) {
        const int nq = (int)((P.nQ - P.q0) < (uint64_t)P.tq ? (P.nQ - P.q0) : (uint64_t)P.tq);
        stage_rows(sQ, P.TP, row_ptr(I, P.qi, P.q0), nq, P.TP);
      }
    }
    __syncthreads();
    if (!P.skip) {
      const bool four = P.grp > 0 && P.i != P.j;
      switch (P.mode) {
        case KEY_HASH:
          if (P.grp == 0) p1_unary<KEY_HASH>(I, P, sS, sp, cnt);
          else if (four) p1_binary<KEY_HASH, true>(I, P, sS, sp, sQ, cnt);
          else p1_binary<KEY_HASH, false>(I, P, sS, sp, sQ, cnt);
          break;
        case KEY_SAMPLED:
          if (P.grp == 0) p1_unary<KEY_SAMPLED>(I, P, sS, sp, cnt);
          else if (four) p1_binary<KEY_SAMPLED, true>(I, P, sS, sp, sQ, cnt);
          else p1_binary<KEY_SAMPLED, false>(I, P, sS, sp, sQ, cnt);
          break;
        default:
          if (P.grp == 0) p1_unary<KEY_CONCAT>(I, P, sS, sp, cnt);
          else if (four) p1_binary<KEY_CONCAT, true>(I, P, sS, sp, sQ, cnt);
          else p1_binary<KEY_CONCAT, false>(I, P, sS, sp, sQ, cnt);
      }
    }
    // per-tile counter flush: warp sums, then one atomic per counter
    cnt.tent = warp_sum(cnt.tent);
    cnt.fresh = warp_sum(cnt.fresh);
    cnt.fail = warp_sum(cnt.fail);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
      s_red[0][wid] = cnt.tent;
      s_red[1][wid] = cnt.fresh;
      s_red[2][wid] = cnt.fail;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned long long a = 0, f = 0, x = 0;
      for (int w = 0; w < kTS / 32; ++w) { a += s_red[0][w]; f += s_red[1][w]; x += s_red[2][w]; }
      if (a) atomicAdd(&I.n_tent, a);
      if (f) atomicAdd(&I.n_new, f);
      if (P.skip) x += 1;
      if (x) atomicAdd(&I.probe_fail, x);
    }
    __syncthreads();
  }
}

// ========================================================== bitmap compaction
// phase 0: candidate bitmap (bits = candidate index) -> I.tent
// phase 1: winner bitmap (bits = tentative index)     -> I.wins (values I.tent[bit])
__device__ __forceinline__ uint64_t phase_bits(const InstDev& I, int phase) {
  return phase ? I.n_tent : I.cands;
}

__global__ void k_chunk_count(BatchDev* Bp, int phase) {
  __shared__ unsigned long long s_w[32];
  const BatchDev B = *Bp;
  const unsigned long long* prefix = phase ? B.chunk_prefix1 : B.chunk_prefix0;
  const unsigned long long total = prefix[B.ninst];
  for (unsigned long long c = blockIdx.x; c < total; c += gridDim.x) {
    const int b = find_owner(prefix, B.ninst, c);
    const InstDev& I = B.inst[b];
    const uint64_t words = (phase_bits(I, phase) + 31) / 32;
    const uint64_t w0 = (c - prefix[b]) * kChunkWords;
    const uint64_t w1 = (w0 + kChunkWords < words) ? w0 + kChunkWords : words;
    unsigned long long s = 0;
    for (uint64_t w = w0 + threadIdx.x; w < w1; w += blockDim.x) s += __popc(I.bitmap[w]);
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned long long t = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_w[w];
      B.chunk_cnt[c] = (unsigned int)t;
    }
    __syncthreads();
  }
}

// One CTA per instance: scan its chunk counts, check capacities.  The last CTA
// to finish (ticket) builds the cross-instance prefixes of the next kernels.
__global__ void k_chunk_scan(BatchDev* Bp, int phase) {
  __shared__ unsigned long long s_w[32];
  __shared__ int s_last;
  const BatchDev B = *Bp;
  const unsigned long long* prefix = phase ? B.chunk_prefix1 : B.chunk_prefix0;
  for (int b = blockIdx.x; b < B.ninst; b += gridDim.x) {
    InstDev& I = B.inst[b];
    if (I.status != ST_RUNNING) continue;
    const unsigned long long c0 = prefix[b], nc = prefix[b + 1] - c0;
    unsigned long long running = 0;
    for (unsigned long long base = 0; base < nc; base += blockDim.x) {
      const unsigned long long i = base + threadIdx.x;
      const unsigned long long v = i < nc ? B.chunk_cnt[c0 + i] : 0ULL;
      unsigned long long tot;
      const unsigned long long ex = block_excl_scan(v, s_w, tot);
      if (i < nc) B.chunk_base[c0 + i] = running + ex;
      running += tot;
    }
    if (threadIdx.x == 0) {
      int need = 0;
      if (phase == 0) {
        I.keys += I.n_new;
        const unsigned long long cap = I.table_mask + 1;
        if (I.probe_fail != 0 || 4 * I.keys > 3 * cap) {
          need |= NEED_TABLE;
          I.need_amount[1] = 4 * I.keys + 4096;
        }
        I.n_tent = running;
        if (running > I.tent_cap) { need |= NEED_TENT; I.need_amount[2] = running; }
      } else {
        I.n_wins = running;
        const uint64_t rows = I.lstart[I.level] + running;
        if (rows > I.row_cap) { need |= NEED_ROWS; I.need_amount[3] = rows; }
      }
      if (need) {
        I.status = ST_NEED_MEM;
        I.need = need;
      }
    }
    __syncthreads();
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned long long t = atomicAdd(B.tickets + 1 + phase, 1ULL);
    s_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (s_last && threadIdx.x == 0) {
    __threadfence();
    if (phase == 0) {
      B.tent_prefix[0] = 0;
      B.chunk_prefix1[0] = 0;
      for (int b = 0; b < B.ninst; ++b) {
        const InstDev& I = B.inst[b];
        const bool run = *(volatile const int*)&I.status == ST_RUNNING;
        const unsigned long long nt = run ? *(volatile const unsigned long long*)&I.n_tent : 0ULL;
        B.tent_prefix[b + 1] = B.tent_prefix[b] + nt;
        B.chunk_prefix1[b + 1] = B.chunk_prefix1[b] + ((nt + 31) / 32 + kChunkWords - 1) / kChunkWords;
      }
    } else {
      B.win_prefix[0] = 0;
      for (int b = 0; b < B.ninst; ++b) {
        const InstDev& I = B.inst[b];
        const bool run = *(volatile const int*)&I.status == ST_RUNNING;
        B.win_prefix[b + 1] = B.win_prefix[b] + (run ? *(volatile const unsigned long long*)&I.n_wins : 0ULL);
      }
    }
  }
}

// Emit set bits of each chunk in order; always clears the chunk's words.
// The chunk is loaded coalesced into shared memory (padded rows of 16 words),
// then every thread scans its 16 consecutive words.
__global__ void __launch_bounds__(kChunkThreads) k_chunk_emit(BatchDev* Bp, int phase) {
  __shared__ unsigned long long s_w[32];
  constexpr int kPer = kChunkWords / kChunkThreads;   // 16 words per thread
  __shared__ uint32_t s_bits[kChunkThreads * (kPer + 1)];
  const BatchDev B = *Bp;
  const unsigned long long* prefix = phase ? B.chunk_prefix1 : B.chunk_prefix0;
  const unsigned long long total = prefix[B.ninst];
  for (unsigned long long c = blockIdx.x; c < total; c += gridDim.x) {
    const int b = find_owner(prefix, B.ninst, c);
    InstDev& I = B.inst[b];
    const uint64_t words = (phase_bits(I, phase) + 31) / 32;
    const uint64_t cbeg = (c - prefix[b]) * kChunkWords;
    for (int u = threadIdx.x; u < kChunkWords; u += blockDim.x) {
      const uint64_t w = cbeg + u;
      const uint32_t v = (w < words) ? I.bitmap[w] : 0u;
      s_bits[(u / kPer) * (kPer + 1) + (u % kPer)] = v;
      if (v) I.bitmap[w] = 0u;
    }
    __syncthreads();
    const uint32_t* mine = s_bits + threadIdx.x * (kPer + 1);
    unsigned long long cnt = 0;
#pragma unroll
    for (int u = 0; u < kPer; ++u) cnt += __popc(mine[u]);
    unsigned long long tot;
    unsigned long long pos = block_excl_scan(cnt, s_w, tot) + B.chunk_base[c];
    if (I.status == ST_RUNNING && cnt) {
      uint64_t* out = phase ? I.wins : I.tent;
      const uint64_t wbeg = cbeg + (uint64_t)threadIdx.x * kPer;
      for (int u = 0; u < kPer; ++u) {
        uint32_t bits = mine[u];
        while (bits) {
          const int p = __ffs(bits) - 1;
          bits &= bits - 1;
          const uint64_t idx = (wbeg + u) * 32 + p;
          out[pos++] = phase ? I.tent[idx] : idx;
        }
      }
    }
    __syncthreads();
  }
}

// ================================================================== verify
__global__ void k_verify(BatchDev* Bp) {
  const BatchDev B = *Bp;
  const unsigned long long total = B.tent_prefix[B.ninst];
  for (unsigned long long e = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (unsigned long long)gridDim.x * blockDim.x) {
    const int b = find_owner(B.tent_prefix, B.ninst, e);
    InstDev& I = B.inst[b];
    const uint64_t i = e - B.tent_prefix[b];
    const int k = I.level;
    const uint64_t g = I.tent[i];
    const Cand c = decode(I, k, g);
    uint64_t h, l;
    switch (I.key_mode) {
      case KEY_HASH: cand_key<KEY_HASH>(I, c, h, l); break;
      case KEY_SAMPLED: cand_key<KEY_SAMPLED>(I, c, h, l); break;
      default: cand_key<KEY_CONCAT>(I, c, h, l);
    }
    if (find_pay(I.table, I.table_mask, h, l) == pay_of(k, g))
      atomicOr(I.bitmap + (i >> 5), 1u << (i & 31));
  }
}

// ================================================================ emit rows
__global__ void k_emit_rows(BatchDev* Bp) {
  const BatchDev B = *Bp;
  const unsigned long long total = B.win_prefix[B.ninst];
  for (unsigned long long e = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (unsigned long long)gridDim.x * blockDim.x) {
    const int b = find_owner(B.win_prefix, B.ninst, e);
    InstDev& I = B.inst[b];
    const uint64_t w = e - B.win_prefix[b];
    const int k = I.level;
    const uint64_t g = I.wins[w];
    const Cand c = decode(I, k, g);
    const uint64_t* ra = row_ptr(I, c.la, c.a);
    const uint64_t* rb = (c.op == OP_AND || c.op == OP_OR || c.op == OP_U) ? row_ptr(I, c.lb, c.b) : ra;
    const uint64_t r = I.lstart[k] + w;
    uint64_t* dst = I.rows + r * (uint64_t)I.TP;
    uint64_t bad = 0;
    const int T = I.T;
    for (int t = 0; t < I.TP; t += 2) {
      const uint64_t w0 = apply_w(c.op, ra[t], rb[t], I.len[t]);
      const uint64_t w1 = (t + 1 < T) ? apply_w(c.op, ra[t + 1], rb[t + 1], I.len[t + 1]) : 0ULL;
      bad |= (w0 ^ (is_pos(I, t) ? 1ULL : 0ULL)) & 1ULL;
      if (t + 1 < T) bad |= (w1 ^ (is_pos(I, t + 1) ? 1ULL : 0ULL)) & 1ULL;
      *reinterpret_cast<ulonglong2*>(dst + t) = make_ulonglong2(w0, w1);
    }
    I.origin[r] = g;
    if (!bad) atomicMin(&I.best_sol, (unsigned long long)g);
  }
}

// ================================================================== finish
// RPN of the node (level lvl, candidate g) into I.rpn (postfix).
__device__ void reconstruct(InstDev& I, int lvl, uint64_t g) {
  struct Fr { int lvl; uint64_t g; int state; };
  Fr st[2 * kMaxSize + 2];
  int sp = 0, out = 0;
  st[0] = {lvl, g, 0};
  while (sp >= 0 && out < kMaxSize) {
    Fr& f = st[sp];
    if (f.lvl <= 1) {
      I.rpn[out++] = (int16_t)f.g;
      --sp;
      continue;
    }
    const Cand c = decode(I, f.lvl, f.g);
    if (c.op < 0) { out = 0; break; }
    const bool bin = (c.op == OP_AND || c.op == OP_OR || c.op == OP_U);
    if (f.state == 0) {
      f.state = 1;
      st[++sp] = {c.la, I.origin[I.lstart[c.la] + c.a], 0};
    } else if (f.state == 1 && bin) {
      f.state = 2;
      st[++sp] = {c.lb, I.origin[I.lstart[c.lb] + c.b], 0};
    } else {
      I.rpn[out++] = (int16_t)(-(1 + c.op));
      --sp;
    }
  }
  I.rpn_len = out;
}

__global__ void k_finish(BatchDev* Bp) {
  const BatchDev B = *Bp;
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < B.ninst; b += gridDim.x * blockDim.x) {
    InstDev& I = B.inst[b];
    if (I.status == ST_RUNNING) {
      const int k = I.level;
      if (I.best_sol != ~0ULL) {
        const uint64_t g = I.best_sol;
        uint64_t lo = 0, hi = I.n_wins;   // first index with wins[idx] >= g
        while (lo < hi) {
          const uint64_t mid = (lo + hi) >> 1;
          if (I.wins[mid] < g) lo = mid + 1; else hi = mid;
        }
        I.lcount[k] = lo + 1;
        I.lcands[k] = g + 1;
        I.sol_index = g;
        I.res_size = k;
        I.status = ST_FOUND;
        reconstruct(I, k, g);
      } else {
        I.lcount[k] = I.n_wins;
        I.lcands[k] = I.cands;
        I.res_size = k;
        if (k >= I.max_size) I.status = ST_NOT_FOUND;
        else I.level = k + 1;
      }
    }
    B.status_out[b] = make_int2(I.status, I.need);
  }
}

__global__ void k_loop_ctl(BatchDev* Bp, cudaGraphConditionalHandle handle, unsigned int max_iter) {
  __shared__ int s_run, s_need;
  const BatchDev B = *Bp;
  if (threadIdx.x == 0) { s_run = 0; s_need = 0; }
  __syncthreads();
  int run = 0, need = 0;
  for (int b = threadIdx.x; b < B.ninst; b += blockDim.x) {
    const int st = B.status_out[b].x;
    run |= (st == ST_RUNNING);
    need |= (st == ST_NEED_MEM);
  }
  if (run) atomicOr(&s_run, 1);
  if (need) atomicOr(&s_need, 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned long long it = ++(*B.loop_iter);
    const bool more = s_run && !s_need && it < max_iter;
    cudaGraphSetConditional(handle, more ? 1u : 0u);
  }
}

// ==================================================================== init
// Level 1: every proposition is a row (duplicates included); its key enters
// the set; propositions are tested as size-1 solutions in order
// (LTL_BS.cu:1127-1163, hashSetsInitialisation 136-160).
__global__ void k_init(BatchDev* Bp) {
  __shared__ unsigned long long s_first;
  __shared__ unsigned long long s_new;
  const BatchDev B = *Bp;
  for (int b = blockIdx.x; b < B.ninst; b += gridDim.x) {
    InstDev& I = B.inst[b];
    if (I.status != ST_RUNNING || I.level != 1) continue;
    if (threadIdx.x == 0) { s_first = ~0ULL; s_new = 0; }
    __syncthreads();
    for (int v = threadIdx.x; v < I.A; v += blockDim.x) {
      const uint64_t* row = I.rows + (uint64_t)v * I.TP;
      uint64_t h, l;
      row_key(I, row, h, l);
      int isnew = 0;
      const uint64_t idx = slot_hash(h, l) & I.table_mask;
      const int r = insert_min(I.table, I.table_mask, idx, ld_key(I.table + idx), h, l, pay_of(1, v), isnew);
      if (r < 0) atomicAdd(&I.probe_fail, 1ULL);
      if (isnew) atomicAdd(&s_new, 1ULL);
      I.origin[v] = v;
      bool sol = true;
      for (int t = 0; t < I.T; ++t) sol = sol && (((row[t] & 1ULL) != 0) == is_pos(I, t));
      if (sol) atomicMin(&s_first, (unsigned long long)v);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      I.keys = s_new;
      I.lstart[0] = 0;
      I.lcount[0] = 0;
      I.lstart[1] = 0;
      I.lcount[1] = I.A;
      I.lcands[1] = I.A;
      I.res_size = 1;
      if (I.probe_fail) {
        I.status = ST_ERROR;
      } else if (s_first != ~0ULL) {
        I.lcount[1] = s_first + 1;
        I.lcands[1] = s_first + 1;
        I.sol_index = s_first;
        I.rpn[0] = (int16_t)s_first;
        I.rpn_len = 1;
        I.status = ST_FOUND;
      } else if (I.max_size <= 1) {
        I.status = ST_NOT_FOUND;
      } else {
        I.level = 2;
      }
      B.status_out[b] = make_int2(I.status, I.need);
    }
    __syncthreads();
  }
}

// ================================================================== rehash
__global__ void k_rehash(const Slot* old_tab, unsigned long long old_cap, Slot* new_tab,
                         unsigned long long new_mask, unsigned long long* fail) {
  for (unsigned long long s = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; s < old_cap;
       s += (unsigned long long)gridDim.x * blockDim.x) {
    const Slot o = old_tab[s];
    if (o.h == kEmpty && o.l == kEmpty) continue;
    uint64_t idx = slot_hash(o.h, o.l) & new_mask;
    bool done = false;
    for (int p = 0; p < kMaxProbes && !done; ++p) {
      const Key128 old = atomicCAS(reinterpret_cast<Key128*>(new_tab + idx), Key128{kEmpty, kEmpty},
                                   Key128{o.h, o.l});
      if (old.h == kEmpty && old.l == kEmpty) {
        new_tab[idx].pay = o.pay;
        done = true;
      } else {
        idx = (idx + 1) & new_mask;
      }
    }
    if (!done) atomicAdd(fail, 1ULL);
  }
}

}  // namespace vfb
