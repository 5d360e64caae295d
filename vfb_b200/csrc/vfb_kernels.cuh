// vfb_kernels.cuh -- kernel entry points of the level step (see vfb_kernels.cu).
#pragma once
#include "vfb_device.cuh"

namespace vfb {

constexpr int kChunkWords = 4096;     // bitmap words per compaction chunk (131072 bits)
constexpr int kChunkThreads = 256;    // threads per compaction CTA
constexpr int kScanThreads = 1024;
constexpr int kScanSlots = 8192;      // hash-set slots per table-scan chunk (at least; more on
                                      // tables of over 2^26 slots, see scan_slots)
constexpr int kScanBatch = 8;         // table-scan entries a thread reads at a time
constexpr int kCompactWords = 512;    // owner-bitmap words per k_compact chunk (16384 candidates)
constexpr int kCompactThreads = 256;  // threads per k_compact CTA (two bitmap words each)
// k_advance threads at most (it loops over larger batches): few enough that
// the one-thread plan and finish keep their state in registers
constexpr int kAdvanceThreads = 256;
constexpr int kTickets = 8;            // words of BatchDev::tickets
constexpr int kTicketP1Blocks = 4;     // tickets[4]: CTAs the step's k_p1 runs (0: all), set by k_advance
constexpr int kEmitGroup = 4;         // owners per warp step of k_emit (their loads in flight together)
constexpr int kEmitItem = 32;         // owners per k_emit work item on large levels (one warp; a lane
                                      // decodes each); small levels take kEmitGroup per item so that
                                      // their few owners still spread over many warps
constexpr unsigned long long kEmitItemFrom = 1ULL << 18;   // owners from which items are kEmitItem

// Global batch descriptor, resident in device memory so that buffer growth
// never invalidates a captured launch sequence.
struct BatchDev {
  InstDev* inst;
  int ninst;
  int pad;
  unsigned long long* p1_prefix;        // [ninst+1] P1 tiles
  unsigned long long* chunk_prefix;     // [ninst+1] owner-bitmap chunks
  unsigned long long* tscan_prefix;     // [ninst+1] table-scan chunks
  unsigned long long* win_prefix;       // [ninst+1] owners of new keys (k_emit_rows), or
                                        // row-emission groups (k_emit)
  unsigned int* chunk_cnt;              // [chunk_cap]
  unsigned long long* chunk_base;       // [chunk_cap] chunk offsets (k_chunk_*), or the
                                        // look-back states of k_compact (flag << 62 | count)
  unsigned long long chunk_cap;
  unsigned long long* tickets;          // [kTickets]: P1 work ticket, scan done counter,
                                        // compaction ticket, (unused), P1 CTAs of the step
  int2* status_out;                     // [ninst] (status, need) mirror for the host
  unsigned long long* loop_iter;        // level steps run by the current device-side loop
  const uint64_t* atoms;                // proposition rows of the call's new instances (one upload),
                                        // copied into each level cache by k_init
  unsigned int* ctl;                    // persistent solver: [0] barrier arrivals, [1] barrier
                                        // generation, [2] error, [3] continue flag
};

// Level step of the graph solver: k_p1, k_table_scan_check, k_compact,
// k_emit, k_advance (k_advance also runs once, with built = 0, before the
// first step of a launch).  k_table_scan_check adds the buffer checks to the
// table scan; k_compact replaces k_chunk_count/scan/emit with one ordered
// pass (decoupled look-back over the chunks); k_advance replaces k_finish +
// k_plan + the loop control.  With loop != 0 it sets the graph's while
// condition: some instance RUNNING, none waiting for memory, fewer than
// max_iter steps.
__global__ void k_advance(BatchDev* B, cudaGraphConditionalHandle handle, int built, int loop,
                          unsigned int max_iter);
__global__ void k_table_scan_check(BatchDev* B);
__global__ void k_compact(BatchDev* B);
__global__ void k_emit(BatchDev* B);

// Level-step kernels of the persistent, cluster and allocation-free solvers,
// launched in this order for every level.
__global__ void k_plan(BatchDev* B);
__global__ void k_p1(BatchDev* B);
// k_p1 with each tile's operand blocks staged by cp.async.bulk (an option:
// VFB_P1_STAGING=bulk).
__global__ void k_p1_bulk(BatchDev* B);
__global__ void k_table_scan(BatchDev* B);
__global__ void k_chunk_count(BatchDev* B);
__global__ void k_chunk_scan(BatchDev* B);
__global__ void k_chunk_emit(BatchDev* B);
__global__ void k_emit_rows(BatchDev* B);
__global__ void k_finish(BatchDev* B);

// Persistent solver: the whole level loop in one cooperative launch (all CTAs
// co-resident), the phases above separated by a bounded grid barrier.  Runs at
// most max_steps levels; stops early when no instance is RUNNING or one needs
// memory.  ctl[2] != 0 afterwards means a barrier timed out.
__global__ void k_solve(BatchDev* B, unsigned int max_steps);

// Cluster solver work list: slots[c] is cluster c's private workspace (one
// instance at a time), insts the instance records, order the queue of record
// indices, next its head.
struct ClusterWork {
  BatchDev* slots;
  InstDev* insts;
  const int* order;
  int n;
  unsigned int* next;
};
__global__ void k_cluster(ClusterWork W);

// Cache-free search (vfb_exhaustive.cu): the instance and the count matrix
// of the formula numbering; formula numbers [lo, hi) of size k are evaluated
// and the smallest solving number lowers *best.
struct ExhDev {
  int A, T;
  uint64_t cnt[kMaxSize + 1][8];   // formulas per size and root operator (7: all of the size)
  uint64_t posmask[2];             // bit t: trace t is positive
  uint8_t len[kMaxTraces];
  uint64_t words[kMaxTraces * 64]; // words[t * A + v]: proposition v on trace t
};
__global__ void k_exhaustive(const ExhDev* P, int k, unsigned long long lo, unsigned long long hi,
                             unsigned long long* best);

// BS stage (vfb_bs.cu): words of the cache rows and of their ~ & |
// combinations, in a slot table of their own.
constexpr int kBsChunkWords = 1024;   // bitmap words per compaction chunk of the BS stage
struct BsDev {
  const uint64_t* rows;            // the instance's level cache (pitch TP)
  int T, TP;
  uint64_t full, target;           // T low bits; the positive traces' bits
  Slot* tab;
  unsigned long long mask;         // table capacity - 1
  uint64_t* vals;                  // entries: words, in canonical order
  uint64_t* org;                   // entries: cache row (base) or candidate index
  uint32_t* bitmap;                // owner bits of the size being built
  unsigned long long* counts;      // owners per chunk
  unsigned long long* offs;        // chunk offsets (exclusive prefix of counts)
  unsigned long long* best;        // first solving candidate of the size
  unsigned long long* fail;        // probe failures
  uint64_t st[kMaxSize + 2], cn[kMaxSize + 2];   // first entry and entries of each size
};
struct BsCand {
  int op;
  uint64_t a, b;   // entry indices of the operands
};

// Candidate g of BS size c -> operator and operand entries.
__host__ __device__ inline BsCand bs_decode(const uint64_t* st, const uint64_t* cn, int c, uint64_t g) {
  BsCand r{-1, 0, 0};
  const uint64_t un = cn[c - 1];
  if (g < un) return BsCand{OP_NOT, st[c - 1] + g, 0};
  g -= un;
  for (int pass = 0; pass < 2; ++pass) {
    for (int i = 1; 2 * i <= c - 1; ++i) {
      const int j = c - 1 - i;
      const uint64_t n = cn[i] * cn[j];
      if (g < n) return BsCand{pass ? OP_OR : OP_AND, st[i] + g / cn[j], st[j] + g % cn[j]};
      g -= n;
    }
  }
  return r;
}

__global__ void k_bs_base(BsDev D, unsigned long long nrows);
__global__ void k_bs_level(BsDev D, int c, unsigned long long cands);
__global__ void k_bs_mark(BsDev D, int c, unsigned long long cap, unsigned long long limit);
__global__ void k_bs_count(BsDev D, unsigned long long nwords);
__global__ void k_bs_emit(BsDev D, int c, unsigned long long nwords, unsigned long long out0);
__global__ void k_bs_bounds(BsDev D, unsigned long long nent, const unsigned long long* rows_at, int n,
                            unsigned long long* out);
__global__ void k_bs_leaves(const InstDev* I, const unsigned long long* rows, int n, int16_t* rpn, int* len);

// Set-up and maintenance kernels.
__global__ void k_fill(BatchDev* B);
__global__ void k_init(BatchDev* B);
__global__ void k_rehash(const Slot* old_tab, unsigned long long old_cap, Slot* new_tab,
                         unsigned long long new_mask, unsigned long long* fail);

}  // namespace vfb
