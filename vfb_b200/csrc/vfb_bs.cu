// vfb_bs.cu -- the BS stage: boolean combinations of the cached formulas over
// their step-0 vectors, after a search that found nothing up to max_size.
//
// LTL_BS (BS LTL_BS.cu:870-1067) projects every cached characteristic set to
// one word, bit i = the formula holds at step 0 of trace i (transfer
// LTL_BS.cu:808-822), and enumerates ~ & | over those words by cost until a
// word equals the positive traces' bits (BSInsertInCache LTL_BS.cu:279-288).
// Here the same search runs in canonical order with min-index ownership, as
// the LTL levels do: the base entries of size c are the projections of the
// level-c rows first seen in row order; a size c > max_size holds ~ over size
// c-1, then & and | over the size splits i <= (c-1)/2, left index major.  A
// word is a 64-bit key (two 32-bit halves, so never the table's empty word)
// in the same 32-byte slot table as the LTL keys; payload = level << 58 |
// index, level 0 for base entries (index = cache row).
#include "vfb_ops.cuh"

namespace vfb {

__device__ __forceinline__ uint64_t bs_project(const BsDev& D, uint64_t row) {
  const uint64_t* w = D.rows + row * (uint64_t)D.TP;
  uint64_t v = 0;
  for (int t = 0; t < D.T; ++t) v |= (__ldcg(w + t) & 1ULL) << t;
  return v;
}

__device__ __forceinline__ uint64_t bs_value(const BsDev& D, const BsCand& c) {
  const uint64_t a = __ldcg(D.vals + c.a);
  if (c.op == OP_NOT) return ~a & D.full;
  const uint64_t b = __ldcg(D.vals + c.b);
  return c.op == OP_AND ? (a & b) : (a | b);
}

__device__ __forceinline__ void bs_insert(const BsDev& D, uint64_t v, unsigned long long pay) {
  const uint64_t h = v & 0xffffffffULL, l = v >> 32;
  uint64_t idx = slot_hash(h, l) & D.mask;
  int isnew = 0;
  if (insert_min(D.tab, D.mask, idx, ld_key(D.tab + idx), h, l, pay, isnew) < 0) atomicAdd(D.fail, 1ULL);
}

// Base: every cache row's word enters the table with its row as payload.
__global__ void k_bs_base(BsDev D, unsigned long long nrows) {
  for (unsigned long long r = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; r < nrows;
       r += (unsigned long long)gridDim.x * blockDim.x)
    bs_insert(D, bs_project(D, r), (unsigned long long)r);
}

// BS size c: every candidate's word; the first solving candidate is kept
// apart (the target word is new: no base entry can hold it, or the search
// would have found a solution).
__global__ void k_bs_level(BsDev D, int c, unsigned long long cands) {
  for (unsigned long long g = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; g < cands;
       g += (unsigned long long)gridDim.x * blockDim.x) {
    const BsCand cd = bs_decode(D.st, D.cn, c, g);
    if (cd.op < 0) continue;
    const uint64_t v = bs_value(D, cd);
    if (v == D.target) atomicMin(D.best, g);
    else bs_insert(D, v, ((unsigned long long)c << kPayShift) | g);
  }
}

// Owner bits: a slot whose payload carries level c (0: base) marks its index
// when the index is below limit.
__global__ void k_bs_mark(BsDev D, int c, unsigned long long cap, unsigned long long limit) {
  for (unsigned long long s = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; s < cap;
       s += (unsigned long long)gridDim.x * blockDim.x) {
    const Key128 k = ld_key(D.tab + s);
    if (k.h == kEmpty && k.l == kEmpty) continue;
    const unsigned long long pay = __ldcg(&D.tab[s].pay);
    if ((pay >> kPayShift) != (unsigned long long)c) continue;
    const uint64_t g = pay & kIdxMask;
    if (g < limit) atomicOr(D.bitmap + (g >> 5), 1u << (g & 31));
  }
}

// Owners per chunk of kBsChunkWords bitmap words.
__global__ void k_bs_count(BsDev D, unsigned long long nwords) {
  __shared__ unsigned long long s_w[32];
  const unsigned long long w0 = (unsigned long long)blockIdx.x * kBsChunkWords;
  unsigned long long cnt = 0;
  for (int u = threadIdx.x; u < kBsChunkWords; u += blockDim.x)
    if (w0 + u < nwords) cnt += __popc(D.bitmap[w0 + u]);
  unsigned long long tot;
  block_excl_scan(cnt, s_w, tot);
  if (threadIdx.x == 0) D.counts[blockIdx.x] = tot;
}

// Owners of each chunk appended in order from entry out0 + offs[chunk]: their
// words and their indices (cache row for base entries, candidate index else);
// the chunk's bitmap words are cleared.
__global__ void k_bs_emit(BsDev D, int c, unsigned long long nwords, unsigned long long out0) {
  __shared__ unsigned long long s_w[32];
  constexpr int kPer = kBsChunkWords / 256;
  const unsigned long long w0 = (unsigned long long)blockIdx.x * kBsChunkWords + (unsigned long long)threadIdx.x * kPer;
  uint32_t bits[kPer];
  unsigned long long cnt = 0;
#pragma unroll
  for (int u = 0; u < kPer; ++u) {
    bits[u] = (w0 + u < nwords) ? D.bitmap[w0 + u] : 0u;
    cnt += __popc(bits[u]);
  }
  unsigned long long tot;
  unsigned long long pos = out0 + D.offs[blockIdx.x] + block_excl_scan(cnt, s_w, tot);
#pragma unroll
  for (int u = 0; u < kPer; ++u) {
    uint32_t b = bits[u];
    if (b) D.bitmap[w0 + u] = 0u;
    while (b) {
      const int bit = __ffs(b) - 1;
      b &= b - 1;
      const uint64_t g = (w0 + u) * 32 + bit;
      uint64_t v;
      if (c == 0) {
        v = bs_project(D, g);
      } else {
        v = bs_value(D, bs_decode(D.st, D.cn, c, g));
      }
      D.vals[pos] = v;
      D.org[pos] = g;
      ++pos;
    }
  }
}

// First entry index at or after each of n row boundaries (entries ascending by
// row): the base sizes' start entries.
__global__ void k_bs_bounds(BsDev D, unsigned long long nent, const unsigned long long* rows_at, int n,
                            unsigned long long* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned long long x = rows_at[i];
  unsigned long long lo = 0, hi = nent;
  while (lo < hi) {
    const unsigned long long mid = (lo + hi) >> 1;
    if (__ldcg(D.org + mid) < x) lo = mid + 1; else hi = mid;
  }
  out[i] = lo;
}

// RPN of each of n cache rows (one thread; rows of any level), kMaxSize tokens
// apart; len[i] = 0 when a row does not reconstruct.
__global__ void k_bs_leaves(const InstDev* Ip, const unsigned long long* rows, int n, int16_t* rpn, int* len) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const InstDev& I = *Ip;
  for (int i = 0; i < n; ++i) {
    const uint64_t r = rows[i];
    int lvl = 1;
    while (lvl < I.res_size && I.lstart[lvl + 1] <= r) ++lvl;
    len[i] = reconstruct_to(I, lvl, __ldcg(I.origin + r), rpn + (size_t)i * kMaxSize, kMaxSize);
  }
}

}  // namespace vfb
