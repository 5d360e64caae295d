// vfb_exhaustive.cu -- cache-free search in formula-number order.
//
// The reference's ltl_nocache (ltl_nocache.cu:319-446) evaluates every
// formula of a size, numbered by numberToFormula (ltl_nocache.cu:169-224) over
// the count matrix of generateMatrix (ltl_nocache.cu:248-287), and keeps any
// solution of the first operator block that has one (a race inside the block).
// This kernel evaluates a range of formula numbers of one size, each thread
// decoding its number into RPN and testing it trace by trace (most formulas
// fail on the first traces), and lowers the smallest solving number with
// atomicMin, so the host gets the first solution of the numbering order.  No
// cache and no hash set: memory is the instance and one word.
#include "vfb_ops.cuh"

namespace vfb {

// Decode formula number n of size k into RPN tokens (>= 0: proposition,
// < 0: -(1 + operator index in ~ & | X F G U)).  A subtree of size s occupies
// s consecutive positions with its operator last.  cnt[s][op] = formulas of
// size s whose root is op, cnt[s][7] = all of size s.
__device__ __forceinline__ void exh_decode(uint64_t n, int k, const uint64_t (*cnt)[8], int16_t* rpn) {
  struct Pend {
    uint64_t n;
    int size, pos;
  };
  Pend st[kMaxSize];
  int sp = 0;
  st[0] = Pend{n, k, 0};
  while (sp >= 0) {
    Pend e = st[sp--];
    if (e.size == 1) {
      rpn[e.pos] = (int16_t)e.n;
      continue;
    }
    int op = 0;
    while (op < OP_U && e.n >= cnt[e.size][op]) e.n -= cnt[e.size][op++];
    rpn[e.pos + e.size - 1] = (int16_t)(-(1 + op));
    const int sub = e.size - 1;
    if (op == OP_NOT || op == OP_X || op == OP_F || op == OP_G) {
      st[++sp] = Pend{e.n, sub, e.pos};
    } else {
      int left = 1;
      while (left < sub - 1 && e.n >= cnt[left][7] * cnt[sub - left][7]) {
        e.n -= cnt[left][7] * cnt[sub - left][7];
        ++left;
      }
      uint64_t q, r;
      divmod64(e.n, cnt[sub - left][7], q, r);
      st[++sp] = Pend{q, left, e.pos};
      st[++sp] = Pend{r, sub - left, e.pos + left};
    }
  }
}

// 1 iff the RPN formula holds at step 0 of every positive trace and of no
// negative trace (semantics of evaluateRPN, ltl_nocache.cu:78-161).
__device__ __forceinline__ bool exh_solves(const ExhDev& P, const int16_t* rpn, int k) {
  for (int t = 0; t < P.T; ++t) {
    uint64_t stk[kMaxSize];
    int sp = 0;
    const int L = P.len[t];
    const uint64_t* w = P.words + (size_t)t * P.A;
    for (int i = 0; i < k; ++i) {
      const int tok = rpn[i];
      if (tok >= 0) {
        stk[sp++] = __ldg(w + tok);
      } else {
        const int op = -tok - 1;
        if (op == OP_AND || op == OP_OR || op == OP_U) {
          const uint64_t r = stk[--sp];
          stk[sp - 1] = apply_w(op, stk[sp - 1], r, L);
        } else {
          stk[sp - 1] = apply_w(op, stk[sp - 1], 0, L);
        }
      }
    }
    const uint64_t want = (P.posmask[t >> 6] >> (t & 63)) & 1ULL;
    if ((stk[0] & 1ULL) != want) return false;
  }
  return true;
}

__global__ void __launch_bounds__(256) k_exhaustive(const ExhDev* __restrict__ Pp, int k, unsigned long long lo,
                                                    unsigned long long hi, unsigned long long* best) {
  __shared__ uint64_t s_cnt[kMaxSize + 1][8];
  const ExhDev& P = *Pp;
  for (int i = threadIdx.x; i < (k + 1) * 8; i += blockDim.x) s_cnt[i / 8][i % 8] = P.cnt[i / 8][i % 8];
  __syncthreads();
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  unsigned long long seen = *(volatile unsigned long long*)best;
  int16_t rpn[kMaxSize];
  unsigned it = 0;
  for (unsigned long long n = lo + (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; n < hi; n += stride) {
    // a smaller solving number already found: nothing left to gain here
    if ((++it & 31u) == 0) seen = *(volatile unsigned long long*)best;
    if (n >= seen) break;
    exh_decode(n, k, s_cnt, rpn);
    if (exh_solves(P, rpn, k)) atomicMin(best, n);
  }
}

}  // namespace vfb
