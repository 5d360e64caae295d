// vfb_kernels.cuh -- kernel entry points of the level step (see vfb_kernels.cu).
#pragma once
#include "vfb_device.cuh"

namespace vfb {

constexpr int kChunkWords = 4096;     // bitmap words per compaction chunk (131072 bits)
constexpr int kChunkThreads = 256;    // threads per compaction CTA
constexpr int kScanThreads = 1024;
constexpr int kScanSlots = 8192;      // hash-set slots per table-scan chunk

// Global batch descriptor, resident in device memory so that buffer growth
// never invalidates a captured launch sequence.
struct BatchDev {
  InstDev* inst;
  int ninst;
  int pad;
  unsigned long long* p1_prefix;        // [ninst+1] P1 tiles
  unsigned long long* chunk_prefix;     // [ninst+1] owner-bitmap chunks
  unsigned long long* tscan_prefix;     // [ninst+1] table-scan chunks
  unsigned long long* win_prefix;       // [ninst+1] owners of new keys
  unsigned int* chunk_cnt;              // [chunk_cap]
  unsigned long long* chunk_base;       // [chunk_cap]
  unsigned long long chunk_cap;
  unsigned long long* tickets;          // [4]: P1 work ticket, scan done counter
  int2* status_out;                     // [ninst] (status, need) mirror for the host
  unsigned long long* loop_iter;        // level steps run by the current device-side loop
  unsigned int* ctl;                    // persistent solver: [0] barrier arrivals, [1] barrier
                                        // generation, [2] error, [3] continue flag
};

// Level-step kernels, launched in this order for every level.
__global__ void k_plan(BatchDev* B);
__global__ void k_p1(BatchDev* B);
__global__ void k_table_scan(BatchDev* B);
__global__ void k_chunk_count(BatchDev* B);
__global__ void k_chunk_scan(BatchDev* B);
__global__ void k_chunk_emit(BatchDev* B);
__global__ void k_emit_rows(BatchDev* B);
__global__ void k_finish(BatchDev* B);
// Device-side level loop: keeps the graph's while-node running while some
// instance is RUNNING, none waits for memory and fewer than max_iter steps ran.
__global__ void k_loop_ctl(BatchDev* B, cudaGraphConditionalHandle handle, unsigned int max_iter);

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

// Set-up and maintenance kernels.
__global__ void k_init(BatchDev* B);
__global__ void k_rehash(const Slot* old_tab, unsigned long long old_cap, Slot* new_tab,
                         unsigned long long new_mask, unsigned long long* fail);

}  // namespace vfb
