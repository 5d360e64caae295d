// vfb_kernels.cu -- sm_100a kernels of one level step of the cached search.
//
// Every kernel reads its work from device memory, so the same launch
// sequence serves every level and any number of instances.  The graph solver
// builds level k with
//
//   k_p1          every candidate: operator words -> 126-bit key -> insert
//                 into the instance's hash set with atomicMin on the
//                 candidate's canonical index; the smallest candidate index
//                 whose CS satisfies the sample is recorded
//                 (applyOperator LTL_BS.cu:183-238, makeRlxUnqChkCSs 30-110,
//                  processUniqueCS 251-269)
//   k_table_scan  a slot whose final payload carries level k holds a key first
//                 seen at this level; its payload's index is the key's owner
//                 (the minimum candidate index): set the owner's bit.  Also
//                 settles whether the recorded solution candidate owns its key
//   k_compact     ordered compaction of the owner bitmap into the ascending
//                 owner list and the owners' rows appended to the level cache
//                 in canonical order, solution test (insertInCache
//                 LTL_BS.cu:299-329); rows skipped when the solution is settled
//   k_advance     level bookkeeping, formula reconstruction (LTL_BS.cu:561-705),
//                 then the next level's candidate-block bases, P1 tiling and
//                 buffer checks (LTL_BS.cu:1226-1488)
//
// The persistent, cluster and allocation-free solvers run the same phases
// as k_plan, k_p1, k_table_scan, k_chunk_count/scan/emit, k_emit_rows,
// k_finish.
//
// The reference's thrust::remove/copy_n compaction (storeUniqueLTLs
// LTL_BS.cu:489-530) is replaced by the bitmap compaction; its racy
// atomicCAS winners (LTL_BS.cu:319, hash_set.cuh:232) by min-index ownership.
#include <cooperative_groups.h>

#include "vfb_ops.cuh"

namespace vfb {

// Programmatic dependent launch inside the level step: wait until the
// preceding kernel has completed and its writes are visible, then let the
// next kernel be scheduled while this one runs (its CTAs then wait here
// themselves).  Both are no-ops for a launch without the attribute.
__device__ __forceinline__ void step_entry() {
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

// ===================================================================== plan
// Plan level k = I.level of a RUNNING instance: candidate-block bases, P1
// tiling, buffer checks.  Records the plan (planned = k, plan_*) or asks the
// host for memory (NEED_MEM, planned = 0).
__device__ void plan_one(InstDev& I) {
  // Everything the plan reads is loaded first: the plan runs on one thread,
  // and a load issued after a store to the record waits for that store.
  const int k = I.level, weighted = I.weighted, on_the_fly = I.on_the_fly;
  const int c1 = atom_level(I), Ln = not_level(I, k);
  const int wA = op_cost(I, OP_AND), wO = op_cost(I, OP_OR), wX = op_cost(I, OP_X), wF = op_cost(I, OP_F),
            wG = op_cost(I, OP_G), wU = op_cost(I, OP_U);
  uint64_t n[kMaxSize + 1];
  for (int i = 0; i <= k; ++i) n[i] = I.lcount[i];
  const uint64_t lstart_prev = I.lstart[k - 1];
  const uint64_t keys = I.keys, table_cap = I.table_mask + 1, bitmap_words = I.bitmap_words,
                 row_cap = I.row_cap, tent_cap = I.tent_cap, promote_above = I.promote_above;
  const int attempt = I.attempt, attempt_level = I.attempt_level, rows_deferred = I.rows_deferred;
  const int no_mask = (attempt_level == k) ? I.no_mask : 0, mask_off = I.mask_off;
  // the first operand rows whose ~ X F G candidates satisfy the sample
  // (recorded when those rows were written)
  const int ulev[4] = {Ln, k - wX, k - wF, k - wG};
  uint32_t uh[4];
#pragma unroll
  for (int o = 0; o < 4; ++o) uh[o] = ulev[o] >= c1 ? I.uhit[ulev[o]][o] : 0u;
  const uint64_t lstart_k = lstart_prev + n[k - 1];
  I.lstart[k] = lstart_k;
  // candidate blocks in canonical order: ~ & | X F G U; a unary operator of
  // cost c reads level k - c, & | over splits (i, k - c - i) with i <= k - c - i,
  // U over every split (LTL_BS.cu:1226-1488; unit costs: the size order)
  uint64_t g = 0;
  uint64_t bA[kMaxSize + 1], bO[kMaxSize + 1], bU[kMaxSize + 1];   // block bases by left level
  I.base_not = g;
  if (Ln >= 0) g += n[Ln];
  for (int pass = 0; pass < 2; ++pass) {
    const int w = pass ? wO : wA;
    for (int i = c1; 2 * i <= k - w; ++i) {
      const int j = k - w - i;
      (pass ? bO : bA)[i] = g;
      (pass ? I.base_or : I.base_and)[i] = g;
      g += n[i] * n[j];
    }
  }
  uint64_t bx[3];
  {
    const int ws[3] = {wX, wF, wG};
#pragma unroll
    for (int o = 0; o < 3; ++o) {
      const int L = k - ws[o];
      bx[o] = g;
      if (L >= c1) g += n[L];
    }
    I.base_x = bx[0];
    I.base_f = bx[1];
    I.base_g = bx[2];
  }
  for (int i = c1; k - wU - i >= c1; ++i) {
    bU[i] = g;
    I.base_u[i] = g;
    g += n[i] * n[k - wU - i];
  }
  I.cands = g;
  // operand groups: the unary operators by operand level (bits ~ X F G), the
  // binary ones by level pair la <= lb (bits &, |, la U lb, lb U la); with
  // unit costs one unary group and one group per split, as the reference's
  // launches fuse them.  The tiles of every staged height 2^0..2^5 are summed
  // on the way.
  int ng = 0;
  uint64_t tl[6] = {0, 0, 0, 0, 0, 0};
  auto add_tiles = [&](int kind, int la, int lb) {
    if (kind == 0) {
      const uint64_t st = (n[la] + kTS - 1) / kTS;
#pragma unroll
      for (int u = 0; u < 6; ++u) tl[u] += st;
    } else {
      const bool qleft = (la == lb) || (n[la] <= n[lb]);
      const uint64_t nS = qleft ? n[lb] : n[la], nQ = qleft ? n[la] : n[lb];
      const uint64_t st = (nS + kTS - 1) / kTS;
#pragma unroll
      for (int u = 0; u < 6; ++u) tl[u] += st * ((nQ + (1ULL << u) - 1) >> u);
    }
  };
  // unit costs: one group per size split, then one unary group over level
  // k-1.  The unary group comes last so that a solution among the & | blocks,
  // which precede X F G in the candidate order, is known before its tiles
  // start: they then compute ~ alone.
  const int msplit = (k - 1) / 2;
  auto u_kind = [&](int q) { return q < msplit ? 1 : 0; };
  auto u_la = [&](int q) { return q < msplit ? q + 1 : k - 1; };
  auto u_lb = [&](int q) { return q < msplit ? k - 2 - q : 0; };
  auto u_mask = [&](int q) { return q < msplit ? (2 * (q + 1) == k - 1 ? 7 : 15) : 0xF; };
  if (!weighted) {
    for (ng = 0; ng <= msplit; ++ng) {
      I.grp_kind[ng] = (uint8_t)u_kind(ng);
      I.grp_la[ng] = (uint8_t)u_la(ng);
      I.grp_lb[ng] = (uint8_t)u_lb(ng);
      I.grp_mask[ng] = (uint8_t)u_mask(ng);
      add_tiles(u_kind(ng), u_la(ng), u_lb(ng));
    }
  } else {
    // weighted: a level (pair) may serve several operators, so the groups
    // are collected first, then their tiles summed
    auto unary = [&](int L, int bit) {
      if (L < c1) return;
      for (int q = 0; q < ng; ++q)
        if (I.grp_kind[q] == 0 && I.grp_la[q] == L) { I.grp_mask[q] |= (uint8_t)(1 << bit); return; }
      if (ng >= kGroups) return;
      I.grp_kind[ng] = 0; I.grp_la[ng] = (uint8_t)L; I.grp_lb[ng] = 0; I.grp_mask[ng] = (uint8_t)(1 << bit);
      ++ng;
    };
    auto binary = [&](int la, int lb, int bits) {
      for (int q = 0; q < ng; ++q)
        if (I.grp_kind[q] == 1 && I.grp_la[q] == la && I.grp_lb[q] == lb) { I.grp_mask[q] |= (uint8_t)bits; return; }
      if (ng >= kGroups) return;
      I.grp_kind[ng] = 1; I.grp_la[ng] = (uint8_t)la; I.grp_lb[ng] = (uint8_t)lb; I.grp_mask[ng] = (uint8_t)bits;
      ++ng;
    };
    unary(Ln, 0);
    unary(k - wX, 1);
    unary(k - wF, 2);
    unary(k - wG, 3);
    const int s3 = k - wA, s4 = k - wO, s8 = k - wU;
    const int sums[3] = {s3, s4, s8};
    for (int q = 0; q < 3; ++q) {
      const int sm = sums[q];
      if (q == 1 && sm == s3) continue;
      if (q == 2 && (sm == s3 || sm == s4)) continue;
      for (int i = c1; 2 * i <= sm; ++i) {
        const int j = sm - i;
        int bits = 0;
        if (sm == s3) bits |= 1;
        if (sm == s4) bits |= 2;
        if (sm == s8) bits |= (i == j) ? 4 : (4 | 8);
        binary(i, j, bits);
      }
    }
    for (int q = 0; q < ng; ++q) add_tiles(I.grp_kind[q], I.grp_la[q], I.grp_lb[q]);
  }
  I.ngroups = ng;
  // operator bases of every group (what a P1 tile needs to tell whether an
  // operator's candidates can still come before the best solution found)
  for (int q = 0; q < ng; ++q) {
    const int kind = weighted ? I.grp_kind[q] : u_kind(q);
    const int mask = weighted ? I.grp_mask[q] : u_mask(q);
    const int la = weighted ? I.grp_la[q] : u_la(q);
    const int lb = weighted ? I.grp_lb[q] : u_lb(q);
    uint64_t b4[4];
    if (kind == 0) {
      b4[0] = 0;   // ~ is the first block
      b4[1] = bx[0];
      b4[2] = bx[1];
      b4[3] = bx[2];
    } else {
      b4[0] = (mask & 1) ? bA[la] : 0;
      b4[1] = (mask & 2) ? bO[la] : 0;
      b4[2] = (mask & 4) ? bU[la] : 0;
      b4[3] = (mask & 8) ? bU[lb] : 0;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) I.grp_base[q][u] = b4[u];
  }
  // P1 tiling: kTS stream rows x tq staged rows per tile.  The staged height
  // is the largest power of two within the band's bound whose tile count
  // reaches the band's target (small levels get shorter tiles so that they
  // still spread over every SM and end in a short last wave), else 1.  The
  // level's band of the tune table also sets the CTAs to launch.
  const int band = tune_band(g);
  const int rows_cap = I.tune_rows[band] ? (I.tune_rows[band] < kTQ ? I.tune_rows[band] : kTQ) : kTQDefault;
  const uint64_t target = I.tune_tiles[band] ? 1ULL << I.tune_tiles[band] : (uint64_t)kP1TileTarget;
  I.p1_blocks = I.tune_blocks[band];
  int lg = 0;
  uint64_t t = tl[0];
#pragma unroll
  for (int u = 1; u < 6; ++u)
    if ((1 << u) <= rows_cap && tl[u] >= target) { lg = u; t = tl[u]; }
  I.tq = 1 << lg;
  // group boundaries in tiles (ph_p1 reads the first ngroups of them)
  {
    uint64_t acc = 0;
    I.grp_prefix[0] = 0;
    for (int q = 0; q < ng; ++q) {
      const int kind = weighted ? I.grp_kind[q] : u_kind(q);
      const int la = weighted ? I.grp_la[q] : u_la(q);
      const int lb = weighted ? I.grp_lb[q] : u_lb(q);
      if (kind == 0) {
        acc += (n[la] + kTS - 1) / kTS;
      } else {
        const bool qleft = (la == lb) || (n[la] <= n[lb]);
        const uint64_t nS = qleft ? n[lb] : n[la], nQ = qleft ? n[la] : n[lb];
        const uint64_t qt = (nQ + (1ULL << lg) - 1) >> lg, st = (nS + kTS - 1) / kTS;
        I.grp_qtiles[q] = (uint32_t)qt;
        acc += st * qt;
      }
      I.grp_prefix[q + 1] = acc;
    }
  }
  const uint64_t words = on_the_fly ? 0 : (g + 31) / 32;
  // new keys of this level: at most all candidates; expect ~8x growth
  const uint64_t grow = 8 * n[k - 1] + 4096;
  const uint64_t est = g < grow ? g : grow;
  int need = 0;
  if (g >= (1ULL << kPayShift)) need |= NEED_LIMIT;
  if (!on_the_fly) {   // an on-the-fly level stores nothing
    if (g > promote_above) need |= NEED_PROMOTE;
    if (words > bitmap_words) { need |= NEED_BITMAP; I.need_amount[0] = words; }
    // (twice the projected keys, rounded up to a power of two: at most half
    // full if the projection holds; 4x measured 6% slower on large
    // instances, from filling and rehashing twice the bytes)
    if (2 * (keys + est) > table_cap) { need |= NEED_TABLE; I.need_amount[1] = 2 * (keys + est); }
    // (a projection the host cannot hold is deferred: the table scan asks for
    // the rows the level's owners need, none when it settles the solution)
    if (!rows_deferred && lstart_k + est > row_cap) {
      need |= NEED_ROWS | NEED_ROWS_EST;
      I.need_amount[3] = lstart_k + est;
    }
    if (est > tent_cap) { need |= NEED_LIST; I.need_amount[2] = est; }
  }
  if (need) {
    I.status = ST_NEED_MEM;
    I.need = need;
    I.planned = 0;
  } else {
    I.plan_tiles = t;
    I.plan_words = words;
    // scan chunks of kScanSlots, larger on large tables (down to 8192 chunks,
    // chunks of at most 4 kScanSlots): fewer per-chunk reductions and atomics
    uint64_t ss = (uint64_t)kScanSlots;
    while (ss < 4 * (uint64_t)kScanSlots && table_cap / (2 * ss) >= 8192) ss *= 2;
    I.scan_slots = (uint32_t)ss;
    I.plan_tchunks = on_the_fly ? 0 : (table_cap + ss - 1) / ss;
    I.planned = k;
    I.p1_done = 0;
    I.p1_step = t;
    I.p1_tail = 1;
    I.n_new = I.n_wins = I.probe_fail = I.n_newlist = 0;
    // A unary candidate recorded as satisfying the sample bounds the level's
    // first solution from the start, as if a P1 tile had found it: operators
    // past it are skipped everywhere (not in a full re-run, nor where the
    // level cannot be re-run)
    uint64_t first = ~0ULL;
    if (!no_mask && !mask_off) {
      const uint64_t ub[4] = {0, bx[0], bx[1], bx[2]};
#pragma unroll
      for (int o = 0; o < 4; ++o) {
        const uint64_t row = 0xFFFFFFFFull - uh[o];
        if (uh[o] && row < n[ulev[o]] && ub[o] + row < first) first = ub[o] + row;
      }
    }
    I.best_cand = first;
    // a level with a solution from the start and millions of candidates before
    // it: P1 skips listing its new slots (one atomic per warp and candidate
    // group) and the table scan reads the whole table instead
    I.no_list = (first != ~0ULL && first >= (1ULL << 22)) ? 1 : 0;
    I.best_sol = ~0ULL;
    I.n_below = 0;
    I.counted_below = 0;
#pragma unroll
    for (int o = 0; o < 4; ++o) I.uhit[k][o] = 0u;   // (this level's rows are written after it)
    I.sol_known = 0;
    I.p1_masked = 0;
    if (attempt_level != k) I.no_mask = 0;   // a new level may skip again
    I.attempt = (attempt_level == k) ? attempt + 1 : 1;
    I.attempt_level = k;
  }
}

__device__ void ph_plan(const BatchDev& B, unsigned bid, unsigned nb) {
  for (int b = bid * blockDim.x + threadIdx.x; b < B.ninst; b += nb * blockDim.x) {
    InstDev& I = B.inst[b];
    unsigned long long tiles = 0, chunks = 0, tchunks = 0;
    if (I.status == ST_RUNNING) {
      plan_one(I);
      if (I.status == ST_RUNNING) {
        tiles = I.plan_tiles;
        chunks = (I.plan_words + kChunkWords - 1) / kChunkWords;
        tchunks = I.plan_tchunks;
      }
    }
    B.p1_prefix[b + 1] = tiles;
    B.chunk_prefix[b + 1] = chunks;
    B.tscan_prefix[b + 1] = tchunks;
  }
}

// One thread: cross-instance prefixes of P1 tiles and bitmap chunks; resets
// the work tickets of the step.
__device__ void ph_plan_prefix(const BatchDev& B) {
  B.p1_prefix[0] = 0;
  B.chunk_prefix[0] = 0;
  B.tscan_prefix[0] = 0;
  for (int b = 0; b < B.ninst; ++b) {
    B.p1_prefix[b + 1] += B.p1_prefix[b];
    B.chunk_prefix[b + 1] += B.chunk_prefix[b];
    B.tscan_prefix[b + 1] += B.tscan_prefix[b];
  }
  for (int i = 0; i < kTickets; ++i) B.tickets[i] = 0;
}

__global__ void __launch_bounds__(1024) k_plan(BatchDev* Bp) {
  const BatchDev B = *Bp;
  ph_plan(B, 0, 1);
  __syncthreads();
  if (threadIdx.x == 0) ph_plan_prefix(B);
}

// ======================================================================= P1
// Bulk staging (BULK): a tile's stream rows and staged rows are each one
// contiguous block of the level cache, copied into shared memory by one
// cp.async.bulk apiece (issued by thread 0, completion counted by an
// mbarrier in bytes).  The wait is bounded: a copy that has not landed after
// about a second stops the instance with an error instead of hanging.
constexpr long long kBulkWaitCycles = 2000000000LL;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void bulk_copy(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
               ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar)) : "memory");
}

// true when the barrier's phase `parity` completed within the bound
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity) {
  const long long t0 = clock64();
  for (;;) {
    uint32_t done = 0;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                 " selp.u32 %0, 1, 0, p;\n}\n" : "=r"(done) : "r"(smem_addr(bar)), "r"(parity) : "memory");
    if (done) return true;
    if (clock64() - t0 > kBulkWaitCycles) return false;
  }
}

template <bool BULK>
__device__ void ph_p1(const BatchDev& B) {
  extern __shared__ __align__(16) uint64_t smem[];
  __shared__ TileSh P;
  __shared__ unsigned long long s_red[3][kTS / 32];
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ int s_stop;
  uint32_t phase = 0;
  if (BULK) {
    if (threadIdx.x == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(&s_bar)) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
      s_stop = 0;
    }
    __syncthreads();
  }
  const unsigned long long total = B.p1_prefix[B.ninst];
  while (true) {
    if (threadIdx.x < 32) {
      // tile set-up by warp 0: the group boundaries are read one per lane and
      // the remaining fields with their loads issued before any shared store,
      // so the chain is a few memory round trips long
      const int lane = threadIdx.x;
      unsigned long long tile = 0;
      if (lane == 0) tile = atomicAdd(B.tickets, 1ULL);
      tile = __shfl_sync(0xffffffffu, tile, 0);
      if (lane == 0) P.tile = tile;
      if (tile < total) {
        const int b = find_owner(B.p1_prefix, B.ninst, tile);
        const InstDev* Ip = B.inst + b;
        const uint64_t local = tile - B.p1_prefix[b] + __ldcg(&Ip->p1_done);
        // lane l holds group boundaries 2l+1 and 2l+2; the group is the number
        // of boundaries at or below the tile
        const int e1 = 2 * lane + 1, e2 = 2 * lane + 2;
        // (boundaries past the level's groups are stale: read as never reached)
        const int ngr = __ldcg(&Ip->ngroups);
        uint64_t gp1 = e1 < kGroups ? __ldcg(&Ip->grp_prefix[e1]) : ~0ULL;
        uint64_t gp2 = e2 < kGroups ? __ldcg(&Ip->grp_prefix[e2]) : ~0ULL;
        if (e1 >= ngr) gp1 = ~0ULL;
        if (e2 >= ngr) gp2 = ~0ULL;
        const int grp = __popc(__ballot_sync(0xffffffffu, gp1 <= local)) +
                        __popc(__ballot_sync(0xffffffffu, gp2 <= local));
        const int src = grp >= 1 ? (grp - 1) >> 1 : 0;
        const uint64_t s1 = __shfl_sync(0xffffffffu, gp1, src), s2 = __shfl_sync(0xffffffffu, gp2, src);
        const uint64_t gstart = grp == 0 ? 0 : ((grp & 1) ? s1 : s2);
        if (lane == 0) {
          const int k = __ldcg(&Ip->level), T = __ldcg(&Ip->T), TP = __ldcg(&Ip->TP);
          const int stride = __ldcg(&Ip->stride1), mode = __ldcg(&Ip->key_mode), tq = __ldcg(&Ip->tq);
          const uint64_t pos0 = __ldcg(&Ip->posmask[0]), pos1 = __ldcg(&Ip->posmask[1]);
          const unsigned long long cap = __ldcg(&Ip->table_mask) + 1, keys = __ldcg(&Ip->keys);
          const unsigned long long fails = __ldcg(&Ip->probe_fail), fresh = __ldcg(&Ip->n_new);
          const int kind = __ldcg(&Ip->grp_kind[grp]), gmask = __ldcg(&Ip->grp_mask[grp]);
          const int i = __ldcg(&Ip->grp_la[grp]), j = __ldcg(&Ip->grp_lb[grp]);
          const uint64_t ni = __ldcg(&Ip->lcount[i]), nj = kind ? __ldcg(&Ip->lcount[j]) : 0;
          const uint64_t qt = kind ? __ldcg(&Ip->grp_qtiles[grp]) : 1;
          const unsigned long long best = __ldcg(&Ip->best_cand);
          const int may_skip = !__ldcg(&Ip->no_mask) && !__ldcg(&Ip->mask_off);
          uint64_t gb[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) gb[u] = __ldcg(&Ip->grp_base[grp][u]);
          const uint64_t within = local - gstart;
          P.inst = b;
          P.grp = grp;
          P.k = k;
          P.T = T;
          P.TP = TP;
          P.half = T / 2;
          P.stride = stride;
          P.mode = mode;
          P.tq = tq;
          P.pos[0] = pos0;
          P.pos[1] = pos1;
          // give up early once the table is known to be too small for this level
          P.otf = __ldcg(&Ip->on_the_fly);
          P.nolist = __ldcg(&Ip->no_list);
          P.skip = !P.otf && ((fails != 0) || (4 * (keys + fresh) > 3 * cap));
          P.kind = kind;
          // operators whose first candidate in this tile comes after the best
          // solution candidate found so far cannot change the result (every
          // candidate before it is still evaluated): they are skipped
          unsigned keep = 0xF;
          if (kind == 0) {
            P.si = i;
            P.nS = ni;
            P.s0 = within * kTS;
            if (may_skip && best != ~0ULL) {
              keep = 0;
#pragma unroll
              for (int u = 0; u < 4; ++u) keep |= (gb[u] + P.s0 <= best ? 1u : 0u) << u;
            }
          } else {
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
            uint64_t sq, qr;
            divmod64(within, qt, sq, qr);
            P.s0 = sq * kTS;
            P.q0 = qr * tq;
            if (may_skip && best != ~0ULL) {
              const uint64_t amin = qleft ? P.q0 : P.s0, bmin = qleft ? P.s0 : P.q0;
              const uint64_t ab = amin * nj + bmin;
              keep = (gb[0] + ab <= best ? 1u : 0u) | (gb[1] + ab <= best ? 2u : 0u) |
                     (gb[2] + ab <= best ? 4u : 0u) | (gb[3] + bmin * ni + amin <= best ? 8u : 0u);
            }
          }
          P.mask = gmask & keep;
          if (P.mask != gmask) *(volatile int*)&const_cast<InstDev*>(Ip)->p1_masked = 1;
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
    // odd pitch for 8-byte copies (conflict-free row reads); the bulk copy
    // keeps the rows' own pitch and rotates the word order instead
    const int sp = BULK ? P.TP : P.TP + 1;
    uint64_t* sS = smem;
    uint64_t* sQ = smem + kTS * sp;
    P1Count cnt{0, 0, ~0ULL};
    // a tile whose every operator is skipped has nothing to do
    bool idle = P.skip || (!P.otf && P.mask == 0);
    if (!idle) {
      const int ns = (int)((P.nS - P.s0) < (uint64_t)kTS ? (P.nS - P.s0) : (uint64_t)kTS);
      const int nq = P.kind == 1 ? (int)((P.nQ - P.q0) < (uint64_t)P.tq ? (P.nQ - P.q0) : (uint64_t)P.tq) : 0;
      if (BULK) {
        if (threadIdx.x == 0) {
          // the previous tile's reads (generic proxy) come before these writes
          asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
          const uint32_t bs = (uint32_t)ns * P.TP * 8, bq = (uint32_t)nq * P.TP * 8;
          asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n"
                       ::"r"(smem_addr(&s_bar)), "r"(bs + bq) : "memory");
          bulk_copy(sS, row_ptr(I, P.si, P.s0), bs, &s_bar);
          if (nq) bulk_copy(sQ, row_ptr(I, P.qi, P.q0), bq, &s_bar);
        }
        if (!bar_wait(&s_bar, phase)) {
          *(volatile int*)&I.status = ST_ERROR;
          s_stop = 1;
        }
        phase ^= 1u;
      } else {
        stage_rows(sS, sp, row_ptr(I, P.si, P.s0), ns, P.TP);
        if (nq) stage_rows(sQ, P.TP, row_ptr(I, P.qi, P.q0), nq, P.TP);
        stage_wait();
      }
    }
    __syncthreads();
    if (BULK && s_stop) break;
    if (!idle && P.otf) {
      p1_solutions<BULK>(I, P, sS, sp, sQ, cnt);
    } else if (!idle) {
      // binary tiles compute the operators up to the last one kept (& | laUlb lbUla)
      const int keys = (P.mask & 8) ? 15 : (P.mask & 4) ? 7 : 3;
      switch (P.mode) {
        case KEY_HASH:
          if (P.kind == 0 && P.mask == 1) p1_unary<KEY_HASH, BULK, 1>(I, P, sS, sp, cnt);
          else if (P.kind == 0) p1_unary<KEY_HASH, BULK, 4>(I, P, sS, sp, cnt);
          else p1_binary_keys<KEY_HASH, BULK>(keys, I, P, sS, sp, sQ, cnt);
          break;
        case KEY_SAMPLED:
          if (P.kind == 0 && P.mask == 1) p1_unary<KEY_SAMPLED, BULK, 1>(I, P, sS, sp, cnt);
          else if (P.kind == 0) p1_unary<KEY_SAMPLED, BULK, 4>(I, P, sS, sp, cnt);
          else p1_binary_keys<KEY_SAMPLED, BULK>(keys, I, P, sS, sp, sQ, cnt);
          break;
        default:
          if (P.kind == 0 && P.mask == 1) p1_unary<KEY_CONCAT, BULK, 1>(I, P, sS, sp, cnt);
          else if (P.kind == 0) p1_unary<KEY_CONCAT, BULK, 4>(I, P, sS, sp, cnt);
          else p1_binary_keys<KEY_CONCAT, BULK>(keys, I, P, sS, sp, sQ, cnt);
      }
    }
    // per-tile counter flush: warp reductions, then one atomic per counter
    cnt.fresh = warp_sum(cnt.fresh);
    cnt.fail = warp_sum(cnt.fail);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long y = __shfl_down_sync(0xffffffffu, cnt.sol, o);
      cnt.sol = y < cnt.sol ? y : cnt.sol;
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
      s_red[0][wid] = cnt.sol;
      s_red[1][wid] = cnt.fresh;
      s_red[2][wid] = cnt.fail;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned long long m = ~0ULL, f = 0, x = 0;
      for (int w = 0; w < kTS / 32; ++w) {
        m = s_red[0][w] < m ? s_red[0][w] : m;
        f += s_red[1][w];
        x += s_red[2][w];
      }
      if (m != ~0ULL) atomicMin(&I.best_cand, m);
      if (f) atomicAdd(&I.n_new, f);
      if (P.skip) x += 1;
      if (x) atomicAdd(&I.probe_fail, x);
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kTS) k_p1(BatchDev* Bp) {
  step_entry();
  const BatchDev B = *Bp;
  if (blockIdx.x >= B.p1_prefix[B.ninst]) return;   // more CTAs than tiles: no ticket needed
  const unsigned long long cap = B.tickets[kTicketP1Blocks];
  if (cap && blockIdx.x >= cap) return;               // the tuned CTA count of this step
  ph_p1<false>(B);
}

// k_p1 with bulk-copied tiles (VFB_P1_STAGING=bulk; measured against the
// 8-byte copies of k_p1, see the design notes)
__global__ void __launch_bounds__(kTS) k_p1_bulk(BatchDev* Bp) {
  step_entry();
  const BatchDev B = *Bp;
  if (blockIdx.x >= B.p1_prefix[B.ninst]) return;
  const unsigned long long cap = B.tickets[kTicketP1Blocks];
  if (cap && blockIdx.x >= cap) return;
  ph_p1<true>(B);
}

// ============================================================== table scan
// Owners of the keys first seen at level k: every slot whose payload carries
// level k.  One chunk of scan_slots slots per CTA iteration; an empty slot's
// payload (~0) carries no level <= 32.  One warp per instance also settles
// whether the recorded solution candidate owns its key.
// The table scan's counting mode at a level that has a solution candidate
// after P1 (the fields read are not written during the scan, except no_mask
// by a failed ownership check, which rebuilds the level anyway).
__device__ __forceinline__ bool below_mode(const InstDev& I) {
  return I.best_cand != ~0ULL && !I.on_the_fly && !I.no_mask && !I.mask_off;
}

__device__ void ph_table_scan(const BatchDev& B, unsigned bid, unsigned nb) {
  __shared__ unsigned long long s_w[32], s_b[32];
  const unsigned long long total = B.tscan_prefix[B.ninst];
  for (unsigned long long c = bid; c < total; c += nb) {
    const int b = find_owner(B.tscan_prefix, B.ninst, c);
    InstDev& I = B.inst[b];
    const unsigned long long k = (unsigned long long)I.level;
    // first attempt at this level with every new slot listed: visit the list;
    // otherwise (a retried level) scan the whole table
    const bool listed = I.attempt == 1 && !I.no_list && I.n_newlist <= I.tent_cap;
    const uint64_t ss = I.scan_slots;
    const uint64_t s0 = (c - B.tscan_prefix[b]) * ss;
    const uint64_t cap = listed ? I.n_newlist : I.table_mask + 1;
    const uint64_t s1 = (s0 + ss < cap) ? s0 + ss : cap;
    // a level with a solution candidate (where it may skip operators) counts
    // the owners below the candidate instead of marking owner bits: if the
    // candidate owns its key (nearly always, and always with exact keys)
    // that count is all the level needs; if not, the level is built again in
    // full (the ownership check below)
    const unsigned long long bc = I.best_cand;
    const bool below = below_mode(I);
    unsigned long long cnt = 0, nbelow = 0;
    // kScanBatch entries per thread at a time: their list reads, then their
    // payload reads, are in flight together
    for (uint64_t e0 = s0 + threadIdx.x; e0 < s1; e0 += (uint64_t)kScanBatch * blockDim.x) {
      uint64_t sl[kScanBatch];
      unsigned long long pay[kScanBatch];
#pragma unroll
      for (int u = 0; u < kScanBatch; ++u) {
        const uint64_t e = e0 + (uint64_t)u * blockDim.x;
        sl[u] = e < s1 ? (listed ? __ldcg(I.wins + e) : e) : ~0ULL;
      }
#pragma unroll
      for (int u = 0; u < kScanBatch; ++u) pay[u] = sl[u] != ~0ULL ? __ldcg(&I.table[sl[u]].pay) : ~0ULL;
#pragma unroll
      for (int u = 0; u < kScanBatch; ++u) {
        if ((pay[u] >> kPayShift) == k) {
          const uint64_t g = pay[u] & kIdxMask;
          if (below) nbelow += g < bc ? 1 : 0;
          else atomicOr(I.bitmap + (g >> 5), 1u << (g & 31));
          ++cnt;
        }
      }
    }
    cnt = warp_sum(cnt);
    nbelow = warp_sum(nbelow);
    if ((threadIdx.x & 31) == 0) {
      s_w[threadIdx.x >> 5] = cnt;
      s_b[threadIdx.x >> 5] = nbelow;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned long long t = 0, tb = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
        t += s_w[w];
        tb += s_b[w];
      }
      if (t) atomicAdd(&I.n_wins, t);
      if (tb) atomicAdd(&I.n_below, tb);
    }
    __syncthreads();
  }
  // solution candidate ownership (warp per instance)
  const int lane = threadIdx.x & 31;
  const unsigned long long gw = ((unsigned long long)bid * blockDim.x + threadIdx.x) >> 5;
  const unsigned long long nw = ((unsigned long long)nb * blockDim.x) >> 5;
  for (unsigned long long b = gw; b < (unsigned long long)B.ninst; b += nw) {
    InstDev& I = B.inst[b];
    if (I.status != ST_RUNNING || I.best_cand == ~0ULL || !I.p1_tail || I.on_the_fly) continue;
    const int k = I.level;
    const uint64_t g = I.best_cand;
    const Cand cd = decode(I, k, g);
    if (cd.op < 0) continue;
    uint64_t h, l;
    switch (I.key_mode) {
      case KEY_HASH: warp_key<KEY_HASH>(I, cd, lane, h, l); break;
      case KEY_SAMPLED: warp_key<KEY_SAMPLED>(I, cd, lane, h, l); break;
      default: warp_key<KEY_CONCAT>(I, cd, lane, h, l);
    }
    if (lane == 0) {
      const bool counting = below_mode(I);
      if (find_pay(I.table, I.table_mask, h, l) == pay_of(k, g)) {
        I.best_sol = g;
        I.sol_known = 1;
        I.counted_below = counting ? 1 : 0;
      } else if (I.p1_masked || counting) {
        // an earlier candidate of the level shares the first solution's key
        // (a relaxed-key collision) while operators past it were skipped or
        // the owners were only counted: the level is built again in full (the
        // host re-plans it, nothing to grow)
        I.no_mask = 1;
        I.need = 0;
        I.planned = 0;
        I.status = ST_NEED_MEM;
      }
    }
  }
}

__global__ void k_table_scan(BatchDev* Bp) {
  const BatchDev B = *Bp;
  ph_table_scan(B, blockIdx.x, gridDim.x);
}

// Graph solver: k_table_scan, then the last CTA to finish checks every
// instance's buffers against its owner count (a shortfall asks the host for
// memory before anything of the level is written) and builds the prefix of
// row-emission items (kEmitItem owners each) over the instances.
__global__ void k_table_scan_check(BatchDev* Bp) {
  __shared__ int s_last;
  __shared__ unsigned long long s_w[32], s_carry;
  step_entry();
  const BatchDev B = *Bp;
  // CTAs beyond the level's scan chunks (but at least one, and enough warps
  // for the per-instance settle) leave at once and take no ticket
  const unsigned long long chunks = B.tscan_prefix[B.ninst];
  const unsigned long long want = (unsigned long long)(B.ninst + (blockDim.x >> 5) - 1) / (blockDim.x >> 5);
  unsigned long long part = chunks > want ? chunks : want;
  if (part > gridDim.x) part = gridDim.x;
  if (part == 0) part = 1;
  if (blockIdx.x >= part) return;
  ph_table_scan(B, blockIdx.x, (unsigned)part);
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    s_last = atomicAdd(B.tickets + 1, 1ULL) == part - 1;
    s_carry = 0;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  for (int base = 0; base < B.ninst; base += blockDim.x) {
    const int b = base + threadIdx.x;
    unsigned long long groups = 0;
    if (b < B.ninst) {
      InstDev& I = B.inst[b];
      if (*(volatile int*)&I.status == ST_RUNNING) {
        const unsigned long long nw = *(volatile unsigned long long*)&I.n_wins;
        const unsigned long long fails = *(volatile unsigned long long*)&I.probe_fail;
        const int sk = *(volatile int*)&I.sol_known;
        const unsigned long long cap = I.table_mask + 1;
        const int k = I.level;
        int need = 0;
        if (fails != 0 || 4 * (I.keys + nw) > 3 * cap) { need |= NEED_TABLE; I.need_amount[1] = 4 * (I.keys + nw) + 4096; }
        if (nw > I.tent_cap) { need |= NEED_LIST; I.need_amount[2] = nw; }
        if (!sk && I.lstart[k] + nw > I.row_cap) { need |= NEED_ROWS; I.need_amount[3] = I.lstart[k] + nw; }
        if (need) {
          I.need = need;
          I.planned = 0;
          I.status = ST_NEED_MEM;
        } else if (!sk) {
          const int item = nw >= kEmitItemFrom ? kEmitItem : kEmitGroup;
          I.emit_item = item;
          groups = (nw + item - 1) / item;
        }
      }
    }
    unsigned long long tot;
    const unsigned long long ex = block_excl_scan(groups, s_w, tot);
    if (b < B.ninst) B.win_prefix[b + 1] = s_carry + ex + groups;
    __syncthreads();
    if (threadIdx.x == 0) s_carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) B.win_prefix[0] = 0;
}

// ========================================================== bitmap compaction
// Owner bitmap (bit g = candidate g owns a new key) -> ascending list I.wins.
__device__ void ph_chunk_count(const BatchDev& B, unsigned bid, unsigned nb) {
  __shared__ unsigned long long s_w[32];
  const unsigned long long* prefix = B.chunk_prefix;
  const unsigned long long total = prefix[B.ninst];
  for (unsigned long long c = bid; c < total; c += nb) {
    const int b = find_owner(prefix, B.ninst, c);
    const InstDev& I = B.inst[b];
    const uint64_t words = (I.cands + 31) / 32;
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

__global__ void k_chunk_count(BatchDev* Bp) {
  const BatchDev B = *Bp;
  ph_chunk_count(B, blockIdx.x, gridDim.x);
}

// One CTA per instance: buffer checks for the level's new keys, scan of its
// chunk counts.  The last CTA to finish (ticket) builds the owners' prefix
// over instances.
__device__ void ph_chunk_scan(const BatchDev& B, unsigned bid, unsigned nb) {
  __shared__ unsigned long long s_w[32];
  __shared__ int s_last;
  const unsigned long long* prefix = B.chunk_prefix;
  for (int b = bid; b < B.ninst; b += nb) {
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
      const unsigned long long cap = I.table_mask + 1;
      if (I.probe_fail != 0 || 4 * (I.keys + I.n_wins) > 3 * cap) {
        need |= NEED_TABLE;
        I.need_amount[1] = 4 * (I.keys + I.n_wins) + 4096;
      }
      if (running > I.tent_cap) { need |= NEED_LIST; I.need_amount[2] = running; }
      const uint64_t rows = I.lstart[I.level] + running;
      if (!I.sol_known && rows > I.row_cap) { need |= NEED_ROWS; I.need_amount[3] = rows; }
      I.n_wins = running;
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
    const unsigned long long t = atomicAdd(B.tickets + 1, 1ULL);
    s_last = (t == nb - 1);
  }
  __syncthreads();
  if (s_last && threadIdx.x == 0) {
    __threadfence();
    B.win_prefix[0] = 0;
    for (int b = 0; b < B.ninst; ++b) {
      const InstDev& I = B.inst[b];
      const bool run = *(volatile const int*)&I.status == ST_RUNNING &&
                       *(volatile const int*)&I.sol_known == 0;
      B.win_prefix[b + 1] = B.win_prefix[b] + (run ? *(volatile const unsigned long long*)&I.n_wins : 0ULL);
    }
  }
}

__global__ void k_chunk_scan(BatchDev* Bp) {
  const BatchDev B = *Bp;
  ph_chunk_scan(B, blockIdx.x, gridDim.x);
}

// Emit set bits of each chunk in order; always clears the chunk's words.
// The chunk is loaded coalesced into shared memory (padded rows), then every
// thread scans its consecutive words.
__device__ void ph_chunk_emit(const BatchDev& B, unsigned bid, unsigned nb) {
  __shared__ unsigned long long s_w[32];
  const int kPer = kChunkWords / blockDim.x;   // consecutive words per thread
  __shared__ uint32_t s_bits[kChunkWords + 256];
  const unsigned long long* prefix = B.chunk_prefix;
  const unsigned long long total = prefix[B.ninst];
  for (unsigned long long c = bid; c < total; c += nb) {
    const int b = find_owner(prefix, B.ninst, c);
    InstDev& I = B.inst[b];
    const uint64_t words = (I.cands + 31) / 32;
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
    for (int u = 0; u < kPer; ++u) cnt += __popc(mine[u]);
    unsigned long long tot;
    unsigned long long pos = block_excl_scan(cnt, s_w, tot) + B.chunk_base[c];
    if (I.status == ST_RUNNING && cnt) {
      uint64_t* out = I.wins;
      const uint64_t wbeg = cbeg + (uint64_t)threadIdx.x * kPer;
      for (int u = 0; u < kPer; ++u) {
        const uint32_t bits = mine[u];
        if (!bits) continue;
        const uint64_t base = (wbeg + u) * 32;
#pragma unroll
        for (int p = 0; p < 32; ++p)
          if ((bits >> p) & 1u) out[pos++] = base + p;
      }
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kChunkThreads) k_chunk_emit(BatchDev* Bp) {
  const BatchDev B = *Bp;
  ph_chunk_emit(B, blockIdx.x, gridDim.x);
}

// ================================================================ emit rows
// Warp per winner, lane per trace word (coalesced row reads and writes).
__device__ void ph_emit_rows(const BatchDev& B, unsigned bid, unsigned nb) {
  const unsigned long long total = B.win_prefix[B.ninst];
  const int lane = threadIdx.x & 31;
  const unsigned long long nwarps = ((unsigned long long)nb * blockDim.x) >> 5;
  for (unsigned long long e = ((unsigned long long)bid * blockDim.x + threadIdx.x) >> 5; e < total;
       e += nwarps) {
    const int b = find_owner(B.win_prefix, B.ninst, e);
    InstDev& I = B.inst[b];
    const uint64_t w = e - B.win_prefix[b];
    const int k = I.level;
    const uint64_t g = I.wins[w];
    const Cand c = decode(I, k, g);
    if (c.op < 0) continue;   // (instances whose solution is settled have no winners listed)
    const uint64_t* ra = row_ptr(I, c.la, c.a);
    const uint64_t* rb = (c.op == OP_AND || c.op == OP_OR || c.op == OP_U) ? row_ptr(I, c.lb, c.b) : ra;
    const uint64_t r = I.lstart[k] + w;
    uint64_t* dst = I.rows + r * (uint64_t)I.TP;
    const int T = I.T;
    unsigned miss = 0u;   // emit_miss OR-ed over the words (the row's own and ~ X F G step-0 tests)
    for (int t = lane; t < I.TP; t += 32) {
      uint64_t word = 0;
      if (t < T) {
        word = apply_w(c.op, __ldcg(ra + t), __ldcg(rb + t), I.len[t]);
        miss |= emit_miss(word, len_mask(I.len[t]), is_pos(I, t) ? 1u : 0u);
      }
      dst[t] = word;
    }
    const unsigned m = __reduce_or_sync(0xffffffffu, miss);
    if (lane == 0) {
      I.origin[r] = g;
      if (!(m & 1u)) atomicMin(&I.best_sol, (unsigned long long)g);
      record_unary(I, k, w, ((m >> 4) & 1u) | (m & 0xEu));   // (~ X F G)
    }
  }
}

__global__ void k_emit_rows(BatchDev* Bp) {
  const BatchDev B = *Bp;
  ph_emit_rows(B, blockIdx.x, gridDim.x);
}

// ================================================================== finish
// Bookkeeping of the level just built by a RUNNING instance; on a solution,
// the formula is rebuilt from the cache (LTL_BS.cu:561-705).
__device__ void finish_one(InstDev& I) {
  const int k = I.level;
  if (I.on_the_fly) {
    // nothing of the level was stored: its first solving candidate, if any,
    // is the answer (it owns its word: no earlier candidate or level has it)
    I.lcount[k] = 0;
    I.built_cands = I.cands;
    I.built_wins = 0;
    I.built_scanned = 0;
    I.built_sol_known = 1;
    if (I.best_cand != ~0ULL) {
      const uint64_t g = I.best_cand;
      I.lcands[k] = g + 1;
      I.sol_index = g;
      I.res_size = k;
      I.status = ST_FOUND;
      reconstruct(I, k, g);
    } else {
      I.lcands[k] = I.cands;
      I.res_size = k - 1;
      I.status = ST_LIMIT;
    }
    return;
  }
  // the level's figures are read before the record is written (one thread:
  // a load after a store to the record waits for the store)
  const uint64_t cands = I.cands, wins = I.n_wins, newlist = I.n_newlist, tent = I.tent_cap,
                 cap = I.table_mask + 1, best = I.best_sol, keys = I.keys;
  const uint64_t* wlist = I.wins;
  const uint64_t n_below = I.n_below;
  const int no_list = I.no_list;
  const int attempt = I.attempt, sol_known = I.sol_known, max_size = I.max_size,
            counted_below = I.counted_below;
  I.built_cands = cands;
  I.built_wins = wins;
  I.built_scanned = (attempt == 1 && !no_list && newlist <= tent) ? newlist : cap;
  I.built_sol_known = sol_known;
  I.keys = keys + wins;
  if (best != ~0ULL) {
    const uint64_t g = best;
    uint64_t lo = 0, hi = wins;   // first index with wins[idx] >= g
    if (counted_below) {
      lo = n_below;
    } else {
      while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (wlist[mid] < g) lo = mid + 1; else hi = mid;
      }
    }
    I.lcount[k] = lo + 1;
    I.lcands[k] = g + 1;
    I.sol_index = g;
    I.res_size = k;
    I.status = ST_FOUND;
    reconstruct(I, k, g);
  } else {
    I.lcount[k] = wins;
    I.lcands[k] = cands;
    I.res_size = k;
    if (k >= max_size) I.status = ST_NOT_FOUND;
    else I.level = k + 1;
  }
  I.rows_deferred = 0;   // the next level projects its rows afresh
}

__device__ void ph_finish(const BatchDev& B, unsigned bid, unsigned nb) {
  for (int b = bid * blockDim.x + threadIdx.x; b < B.ninst; b += nb * blockDim.x) {
    InstDev& I = B.inst[b];
    if (I.status == ST_RUNNING) finish_one(I);
    B.status_out[b] = make_int2(I.status, I.need);
  }
}

__global__ void k_finish(BatchDev* Bp) {
  const BatchDev B = *Bp;
  ph_finish(B, blockIdx.x, gridDim.x);
}

// ============================================================ level advance
// One CTA.  built != 0: every RUNNING instance whose level was planned (and
// so built by the step that just ran) is finished; then every RUNNING
// instance not yet planned for its current level is planned.  The batch's
// tile and chunk prefixes are rebuilt from the recorded plans, the
// look-back states of k_compact cleared and the work tickets reset.
__global__ void __launch_bounds__(kAdvanceThreads) k_advance(BatchDev* Bp, cudaGraphConditionalHandle handle, int built,
                                                  int loop, unsigned int max_iter) {
  __shared__ int s_run, s_need;
  __shared__ unsigned s_blocks;
  __shared__ unsigned long long s_w3[32][3];
  __shared__ unsigned long long s_carry[3];
  step_entry();
  const BatchDev B = *Bp;
  if (threadIdx.x == 0) {
    s_run = 0;
    s_need = 0;
    s_blocks = 0;
    s_carry[0] = s_carry[1] = s_carry[2] = 0;
  }
  __syncthreads();
  int run = 0, need = 0;
  unsigned blocks = 0;   // CTAs the step's P1 asks for (~0u: every resident CTA)
  for (int base = 0; base < B.ninst; base += blockDim.x) {
    const int b = base + threadIdx.x;
    unsigned long long tiles = 0, chunks = 0, tchunks = 0;
    if (b < B.ninst) {
      InstDev& I = B.inst[b];
      if (built && I.status == ST_RUNNING && I.planned == I.level) {
        if (I.p1_tail) finish_one(I);
        else I.p1_done += I.p1_step;   // a slice of the level's tiles ran
      }
      if (I.status == ST_RUNNING && I.planned != I.level) plan_one(I);
      if (I.status == ST_RUNNING) {
        // this step's slice of P1 tiles: all that remain, or the quota's worth
        const unsigned long long left = I.plan_tiles - I.p1_done;
        unsigned long long step = left;
        if (I.p1_quota && I.cands > I.p1_quota) {
          const unsigned long long q = I.p1_quota * I.plan_tiles / I.cands;
          step = q < 1 ? 1 : (q < left ? q : left);
        }
        I.p1_step = step;
        I.p1_tail = step == left;
        tiles = step;
        const unsigned want = I.p1_blocks ? (unsigned)I.p1_blocks : ~0u;
        blocks = want > blocks ? want : blocks;
        if (I.p1_tail) {
          chunks = (I.plan_words + kCompactWords - 1) / kCompactWords;
          tchunks = I.plan_tchunks;
        }
        run = 1;
      }
      need |= (I.status == ST_NEED_MEM);
      B.status_out[b] = make_int2(I.status, I.need);
    }
    // inclusive prefixes over this block of instances, carried across blocks
    const unsigned long long v[3] = {tiles, chunks, tchunks};
    unsigned long long ex[3], tot[3];
    block_excl_scan3(v, s_w3, ex, tot);
    if (b < B.ninst) {
      B.p1_prefix[b + 1] = s_carry[0] + ex[0] + tiles;
      B.chunk_prefix[b + 1] = s_carry[1] + ex[1] + chunks;
      B.tscan_prefix[b + 1] = s_carry[2] + ex[2] + tchunks;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      s_carry[0] += tot[0];
      s_carry[1] += tot[1];
      s_carry[2] += tot[2];
    }
    __syncthreads();
  }
  if (run) atomicOr(&s_run, 1);
  if (need) atomicOr(&s_need, 1);
  if (blocks) atomicMax(&s_blocks, blocks);
  __syncthreads();
  if (threadIdx.x == 0) {
    B.p1_prefix[0] = 0;
    B.chunk_prefix[0] = 0;
    B.tscan_prefix[0] = 0;
    for (int i = 0; i < 4; ++i) B.tickets[i] = 0;
    B.tickets[kTicketP1Blocks] = s_blocks == ~0u ? 0 : s_blocks;
  }
  __syncthreads();
  const unsigned long long nchunks = s_carry[1];
  for (unsigned long long c = threadIdx.x; c < nchunks; c += blockDim.x) B.chunk_base[c] = 0;
  if (loop && threadIdx.x == 0) {
    const unsigned long long it = ++(*B.loop_iter);
    const bool more = s_run && !s_need && it < max_iter;
    cudaGraphSetConditional(handle, more ? 1u : 0u);
  }
}

// ========================================================= ordered compaction
// Owner bitmap -> ascending owner list I.wins, in one pass.  CTAs take chunks
// of kCompactWords bitmap words in ticket order; each counts its owners,
// publishes the count (flag 1) and then its inclusive prefix (flag 2) in
// chunk_base, and finds its exclusive prefix by looking back over the
// preceding chunks of the instance, a warp at a time (decoupled look-back: a
// chunk waits for its predecessors' counts, which are published as soon as
// they are known, never for their prefixes).  Instances that are not RUNNING
// (the table scan's check asked for memory) are skipped; bitmap words are
// cleared in every case.
constexpr unsigned long long kFlagCount = 1ULL << 62, kFlagPrefix = 2ULL << 62;
constexpr unsigned long long kStateMask = (1ULL << 62) - 1;
constexpr long long kLookbackCycles = 2000000000LL;   // ~1 s: a predecessor that never publishes

__global__ void __launch_bounds__(kCompactThreads) k_compact(BatchDev* Bp) {
  __shared__ unsigned long long s_w[32];
  __shared__ unsigned long long s_c, s_prefix;
  __shared__ int s_ok;
  step_entry();
  const BatchDev B = *Bp;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned long long total = B.chunk_prefix[B.ninst];
  if (blockIdx.x >= total) return;   // no chunk for this CTA (small levels)
  for (;;) {
    if (threadIdx.x == 0) s_c = atomicAdd(B.tickets + 2, 1ULL);
    __syncthreads();
    const unsigned long long c = s_c;
    if (c >= total) break;
    const int b = find_owner(B.chunk_prefix, B.ninst, c);
    InstDev& I = B.inst[b];
    const unsigned long long c0 = B.chunk_prefix[b];
    const uint64_t words = (I.cands + 31) / 32;
    const uint64_t w0 = (c - c0) * kCompactWords;
    uint32_t v[2];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const uint64_t w = w0 + 2 * threadIdx.x + j;
      v[j] = (w < words) ? __ldcg(I.bitmap + w) : 0u;
      if (v[j]) I.bitmap[w] = 0u;
    }
    const unsigned long long cnt = __popc(v[0]) + __popc(v[1]);
    unsigned long long tot;
    const unsigned long long ex = block_excl_scan(cnt, s_w, tot);
    if (threadIdx.x == 0) {
      const int ok = *(volatile int*)&I.status == ST_RUNNING;
      s_ok = ok;
      if (ok && c == c0) {
        atomicExch(B.chunk_base + c, kFlagPrefix | tot);
        s_prefix = 0;
      } else if (ok) {
        atomicExch(B.chunk_base + c, kFlagCount | tot);
      }
    }
    __syncthreads();
    if (s_ok && c != c0 && warp == 0) {
      // look back: lane i reads chunk (p - i); the nearest chunk with a
      // published prefix ends the walk (chunks before the instance's first
      // count as a prefix of 0)
      unsigned long long prefix = 0;
      long long p = (long long)c - 1;
      bool failed = false;
      for (;;) {
        const long long q = p - lane;
        unsigned long long st = kFlagPrefix;
        if (q >= (long long)c0) {
          const long long t0 = clock64();
          st = *(volatile unsigned long long*)(B.chunk_base + q);
          while ((st >> 62) == 0) {
            if (clock64() - t0 > kLookbackCycles) break;
            st = *(volatile unsigned long long*)(B.chunk_base + q);
          }
        }
        if (__any_sync(0xffffffffu, (st >> 62) == 0)) { failed = true; break; }
        const unsigned pm = __ballot_sync(0xffffffffu, (st >> 62) == 2);
        const int stop = pm ? __ffs(pm) - 1 : 31;
        unsigned long long x = lane <= stop ? (st & kStateMask) : 0ULL;
        x = warp_sum(x);
        prefix += __shfl_sync(0xffffffffu, x, 0);
        if (pm) break;
        p -= 32;
      }
      if (lane == 0) {
        if (failed) {
          // a predecessor never published: give up on this instance; the
          // prefix published here keeps successors' writes inside the list
          atomicExch(&I.status, (int)ST_ERROR);
          prefix = 0;
        }
        atomicExch(B.chunk_base + c, kFlagPrefix | (prefix + tot));
        s_prefix = prefix;
      }
    }
    __syncthreads();
    if (s_ok) {
      unsigned long long pos = s_prefix + ex;
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        uint32_t bits = v[j];
        const uint64_t gw = (w0 + 2 * threadIdx.x + j) * 32;
        while (bits) {
          const int bit = __ffs(bits) - 1;
          bits &= bits - 1;
          I.wins[pos++] = gw + bit;
        }
      }
    }
    __syncthreads();
  }
}

// ================================================================ row emission
// Graph solver: the owners' rows appended to the level cache in canonical
// order, solution test (insertInCache LTL_BS.cu:299-329).  Work items are
// kEmitItem consecutive owners of one instance on large levels, kEmitGroup
// on small ones (prefix built by k_table_scan_check, which records the
// choice); a warp takes an item, each lane decodes one owner
// (decode_level: compares with the plan's block bases), then the owners go
// kEmitGroup at a time, lane per trace word, so row reads and writes stay
// coalesced and the loads of a group's owners are in flight together.
__global__ void __launch_bounds__(256, 3) k_emit(BatchDev* Bp) {
  step_entry();
  const BatchDev B = *Bp;
  const unsigned long long total = B.win_prefix[B.ninst];
  const int lane = threadIdx.x & 31;
  const unsigned long long nw = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
  for (unsigned long long item = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; item < total;
       item += nw) {
    const int b = find_owner(B.win_prefix, B.ninst, item);
    InstDev& I = B.inst[b];
    if (I.status != ST_RUNNING) continue;
    const int k = I.level, T = I.T, TP = I.TP;
    const uint64_t per = (uint64_t)I.emit_item;
    const uint64_t o0 = (item - B.win_prefix[b]) * per;
    const uint64_t nwin = I.n_wins;
    const int cnt = (int)(nwin - o0 < per ? nwin - o0 : per);
    // lane l decodes owner o0 + l
    int op = -1;
    const uint64_t* pa = nullptr;
    const uint64_t* pb = nullptr;
    uint64_t g = 0;
    if (lane < cnt) {
      g = __ldcg(I.wins + o0 + lane);
      const Cand cd = decode_level(I, k, g);
      op = cd.op;
      if (op >= 0) {
        pa = row_ptr(I, cd.la, cd.a);
        pb = (op == OP_AND || op == OP_OR || op == OP_U) ? row_ptr(I, cd.lb, cd.b) : pa;
      }
    }
    const uint64_t r0 = I.lstart[k] + o0;
    for (int s0 = 0; s0 < cnt; s0 += kEmitGroup) {
      int ops[kEmitGroup];
      const uint64_t* ra[kEmitGroup];
      const uint64_t* rb[kEmitGroup];
      unsigned miss[kEmitGroup];   // emit_miss OR-ed over the words
#pragma unroll
      for (int u = 0; u < kEmitGroup; ++u) {
        const int src = s0 + u;
        const int o = __shfl_sync(0xffffffffu, op, src & 31);
        ops[u] = src < cnt ? o : -1;
        ra[u] = (const uint64_t*)__shfl_sync(0xffffffffu, (unsigned long long)pa, src & 31);
        rb[u] = (const uint64_t*)__shfl_sync(0xffffffffu, (unsigned long long)pb, src & 31);
        miss[u] = 0u;
      }
      for (int t = lane; t < TP; t += 32) {
        const int L = t < T ? I.len[t] : 0;
        const unsigned lab = (t < T && is_pos(I, t)) ? 1u : 0u;
        const uint64_t lm = len_mask(L);
        uint64_t xa[kEmitGroup], xb[kEmitGroup];
#pragma unroll
        for (int u = 0; u < kEmitGroup; ++u) {
          xa[u] = (ops[u] >= 0 && t < T) ? __ldg(ra[u] + t) : 0ULL;
          xb[u] = (ops[u] >= 0 && t < T) ? __ldg(rb[u] + t) : 0ULL;
        }
#pragma unroll
        for (int u = 0; u < kEmitGroup; ++u) {
          if (ops[u] < 0) continue;
          const uint64_t word = t < T ? apply_w(ops[u], xa[u], xb[u], L) : 0ULL;
          if (t < T) miss[u] |= emit_miss(word, lm, lab);
          I.rows[(r0 + s0 + u) * (uint64_t)TP + t] = word;
        }
      }
#pragma unroll
      for (int u = 0; u < kEmitGroup; ++u) {
        if (ops[u] < 0) continue;
        const unsigned m = __reduce_or_sync(0xffffffffu, miss[u]);
        if (lane == s0 + u) {
          I.origin[r0 + s0 + u] = g;
          if (!(m & 1u)) atomicMin(&I.best_sol, (unsigned long long)g);
          record_unary(I, k, o0 + s0 + u, ((m >> 4) & 1u) | (m & 0xEu));   // (~ X F G)
        }
      }
    }
  }
}

// ======================================================= persistent solver
// A wait longer than this (in SM clock cycles, ~60 s) is treated as a failed
// barrier: the waiting CTA raises ctl[2] and every CTA leaves the kernel.
constexpr long long kBarrierCycles = 120000000000LL;

__device__ bool grid_sync(unsigned int* ctl, unsigned int nb) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int* vgen = ctl + 1;
    volatile unsigned int* verr = ctl + 2;
    const unsigned int gen = *vgen;
    __threadfence();
    const unsigned int arrived = atomicAdd(ctl, 1u) + 1u;
    if (arrived == nb) {
      atomicExch(ctl, 0u);     // no CTA arrives again before the generation moves
      __threadfence();
      atomicAdd(ctl + 1, 1u);
    } else {
      const long long t0 = clock64();
      while (*vgen == gen && *verr == 0) {
        if (clock64() - t0 > kBarrierCycles) {
          atomicExch(ctl + 2, 1u);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    s_ok = (*verr == 0);
  }
  __syncthreads();
  return s_ok != 0;
}

__global__ void __launch_bounds__(kTS) k_solve(BatchDev* Bp, unsigned int max_steps) {
  const BatchDev B = *Bp;
  unsigned int* ctl = B.ctl;
  const unsigned int bid = blockIdx.x, nb = gridDim.x;
  __shared__ int s_more;
  for (unsigned int it = 0; it < max_steps; ++it) {
    ph_plan(B, bid, nb);
    if (!grid_sync(ctl, nb)) return;
    if (bid == 0 && threadIdx.x == 0) ph_plan_prefix(B);
    if (!grid_sync(ctl, nb)) return;
    ph_p1<false>(B);
    if (!grid_sync(ctl, nb)) return;
    ph_table_scan(B, bid, nb);
    if (!grid_sync(ctl, nb)) return;
    ph_chunk_count(B, bid, nb);
    if (!grid_sync(ctl, nb)) return;
    ph_chunk_scan(B, bid, nb);
    if (!grid_sync(ctl, nb)) return;
    ph_chunk_emit(B, bid, nb);
    if (!grid_sync(ctl, nb)) return;
    ph_emit_rows(B, bid, nb);
    if (!grid_sync(ctl, nb)) return;
    ph_finish(B, bid, nb);
    if (!grid_sync(ctl, nb)) return;
    if (bid == 0 && threadIdx.x == 0) {
      int run = 0, need = 0;
      for (int b = 0; b < B.ninst; ++b) {
        const int st = B.status_out[b].x;
        run |= (st == ST_RUNNING);
        need |= (st == ST_NEED_MEM);
      }
      atomicExch(ctl + 3, (run && !need) ? 1u : 0u);
      ++(*B.loop_iter);
    }
    if (!grid_sync(ctl, nb)) return;
    if (threadIdx.x == 0) s_more = *(volatile unsigned int*)(ctl + 3);
    __syncthreads();
    if (!s_more) return;
  }
}

// ========================================================= cluster solver
// One thread-block cluster per instance in flight: the cluster's CTAs run the
// level phases over one instance, separated by the hardware cluster barrier;
// each cluster then pulls the next instance from the queue.  A level above
// the instance's promote_above (or a buffer that must grow) stops the instance
// at a level boundary with NEED_MEM; the host continues it on the whole GPU.
__global__ void __launch_bounds__(kTS) k_cluster(ClusterWork W) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const unsigned int rank = cl.block_rank(), csize = cl.num_blocks();
  const unsigned int slot = blockIdx.x / csize;
  BatchDev B = W.slots[slot];
  __shared__ int s_idx;
  for (;;) {
    if (rank == 0 && threadIdx.x == 0) {
      const unsigned int q = atomicAdd(W.next, 1u);
      s_idx = q < (unsigned int)W.n ? W.order[q] : -1;
    }
    cl.sync();
    const int idx = *cl.map_shared_rank(&s_idx, 0);
    cl.sync();   // rank 0 rewrites s_idx only after every CTA has read it
    if (idx < 0) break;
    B.inst = W.insts + idx;
    B.ninst = 1;
    for (int it = 0; it < kMaxSize + 2; ++it) {
      const int st = *(volatile int*)&B.inst->status;
      cl.sync();   // every CTA has read the status before a phase may change it
      if (st != ST_RUNNING) break;
      ph_plan(B, rank, csize);
      cl.sync();
      if (rank == 0 && threadIdx.x == 0) ph_plan_prefix(B);
      cl.sync();
      ph_p1<false>(B);
      cl.sync();
      ph_table_scan(B, rank, csize);
      cl.sync();
      ph_chunk_count(B, rank, csize);
      cl.sync();
      ph_chunk_scan(B, rank, csize);
      cl.sync();
      ph_chunk_emit(B, rank, csize);
      cl.sync();
      ph_emit_rows(B, rank, csize);
      cl.sync();
      ph_finish(B, rank, csize);
      cl.sync();
    }
  }
}

// ==================================================================== fill
// First buffers of new instances (fill set by the host): empty table (every
// word ~0) and clear owner bitmap, every thread of the grid on one instance
// after the other.
__global__ void k_fill(BatchDev* Bp) {
  const BatchDev B = *Bp;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
  for (int b = 0; b < B.ninst; ++b) {
    const InstDev& I = B.inst[b];
    if (!I.fill || I.status != ST_RUNNING || I.level != 1) continue;
    ulonglong2* tab = reinterpret_cast<ulonglong2*>(I.table);
    const uint64_t nt = (I.table_mask + 1) * (sizeof(Slot) / sizeof(ulonglong2));
    for (uint64_t x = tid; x < nt; x += nth) tab[x] = make_ulonglong2(~0ULL, ~0ULL);
    for (uint64_t x = tid; x < I.bitmap_words; x += nth) I.bitmap[x] = 0u;
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
    if (threadIdx.x == 0) {
      s_first = ~0ULL;
      s_new = 0;
      for (int o = 0; o < 4; ++o) I.uhit[atom_level(I)][o] = 0u;
    }
    if (I.atoms_staged) {
      if (!B.atoms) {   // (never: the host uploads them before this launch)
        __syncthreads();
        if (threadIdx.x == 0) I.status = ST_ERROR;
        continue;
      }
      const uint64_t nw = (uint64_t)I.A * I.TP;
      for (uint64_t w = threadIdx.x; w < nw; w += blockDim.x) I.rows[w] = B.atoms[I.atom_off + w];
    }
    __syncthreads();
    for (int v = threadIdx.x; v < I.A; v += blockDim.x) {
      const uint64_t* row = I.rows + (uint64_t)v * I.TP;
      uint64_t h, l;
      row_key(I, row, h, l);
      int isnew = 0;
      uint64_t idx = slot_hash(h, l) & I.table_mask;
      const int r = insert_min(I.table, I.table_mask, idx, ld_key(I.table + idx), h, l,
                               pay_of(atom_level(I), v), isnew);
      if (r < 0) atomicAdd(&I.probe_fail, 1ULL);
      if (isnew) atomicAdd(&s_new, 1ULL);
      I.origin[v] = v;
      bool sol = true;
      unsigned miss = 0u;
      for (int t = 0; t < I.T; ++t) {
        const unsigned lab = is_pos(I, t) ? 1u : 0u;
        sol = sol && (((row[t] & 1ULL) != 0) == (lab != 0));
        miss |= unary_miss(row[t], len_mask(I.len[t]), lab);
      }
      if (sol) atomicMin(&s_first, (unsigned long long)v);
      record_unary(I, atom_level(I), (uint64_t)v, miss);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      I.fill = 0;
      // the propositions are the level of their cost c1 (1 with unit costs);
      // the levels below it are empty
      const int c1 = atom_level(I);
      I.keys = s_new;
      for (int k = 0; k <= c1; ++k) {
        I.lstart[k] = 0;
        I.lcount[k] = 0;
        I.lcands[k] = 0;
      }
      I.lcount[c1] = I.A;
      I.lcands[c1] = I.A;
      I.res_size = c1;
      if (I.probe_fail) {
        I.status = ST_ERROR;
      } else if (s_first != ~0ULL) {
        I.lcount[c1] = s_first + 1;
        I.lcands[c1] = s_first + 1;
        I.sol_index = s_first;
        I.rpn[0] = (int16_t)s_first;
        I.rpn_len = 1;
        I.status = ST_FOUND;
      } else if (I.max_size <= c1) {
        I.status = ST_NOT_FOUND;
      } else {
        I.level = c1 + 1;
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
