// vfb_engine.cu -- host driver of the cached search: instance set-up, the
// level loop, buffer growth, results.  Implements the C ABI of include/vfb.h.
//
// The reference drives one launch per (level, operator, size split, chunk)
// with a blocking device-to-host copy after each (LTL_BS.cu:1226-1488).  Here
// a whole level of every instance in flight is one fixed launch sequence
// (vfb_kernels.cu) that reads its work from device memory.  That sequence is
// captured once as the body of a CUDA-graph while-node: the device keeps
// building levels until every instance is solved, exhausted or needs a larger
// buffer, so a solve is one graph launch and one status read.  The host only
// steps in to grow a buffer (the level is then re-run; every kernel of the
// step is idempotent) and to read the results.  Device buffers come from a
// block cache on top of the stream-ordered pool, so repeated solves neither
// allocate nor re-grow.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <new>
#include <functional>
#include <vector>

#include "vfb_kernels.cuh"
#include "../../include/vfb.h"

namespace vfb {

namespace {

struct InstHost {
  uint64_t sig = 0; // instance signature (capacity hints)
  InstDev d;        // host copy of the device record
  bool active = false;
  vfb_status fail = VFB_OK;
  int accounted = 1;  // last level whose bytes were added to the profile
  bool restart = false;  // batch: evicted for memory (or never fitted): solved alone after the batch
};

// Serving: a request whose first buffers are at most this large is admitted
// past the projected budget when they fit what is actually free.
constexpr uint64_t kLightRequestBytes = 256ull << 20;
// Serving: two or more requests waiting for memory this many steps running
// count as a deadlock (the least advanced one is evicted).
constexpr int kServeWaitSteps = 32;

uint64_t pow2_at_least(uint64_t x) {
  uint64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}
uint64_t pow2_at_most(uint64_t x) {
  uint64_t p = 1;
  while (2 * p <= x) p <<= 1;
  return p;
}

// Kernels of one level step, in launch order (ids index Engine::prof).
enum KId { KP_ADVANCE, KP_P1, KP_TSCAN, KP_COMPACT, KP_EMIT, KP_INIT, KP_REHASH, KP_N };
const char* const kNames[KP_N] = {"k_advance", "k_p1", "k_table_scan", "k_compact", "k_emit", "k_init",
                                  "k_rehash"};
// One launch of the step graph: plan the instances that need it, then build
// one level (the trailing k_advance finishes it and plans the next).
const int kStepSeq[] = {KP_ADVANCE, KP_P1, KP_TSCAN, KP_COMPACT, KP_EMIT, KP_ADVANCE};
constexpr int kStepLen = sizeof(kStepSeq) / sizeof(int);
constexpr int kStepP1 = 1;    // position of k_p1 in kStepSeq
constexpr int kBodyLen = 5;   // kernels of one level inside the device-side loop
constexpr unsigned kMaxLoop = 4 * kMaxSize;
// serving: P1 candidates of one request per step (a larger level takes
// several steps), which bounds the step that every resident request waits for
constexpr uint64_t kServeStepCands = 1ull << 23;
// candidates of one level above which an instance leaves the cluster solver
constexpr unsigned long long kPromoteAbove = 1ULL << 21;

struct Prof {
  uint64_t launches = 0;
  double ms = 0, bytes = 0;
};

}  // namespace

struct Engine {
  int device = 0;
  int verbose = 0;
  int profile = 0;
  size_t mem_limit = 0;
  cudaStream_t stream = nullptr;
  int sms = 0;
  int grid = 0;        // grid-stride CTAs (256 threads)
  int emit_grid = 0;   // k_emit CTAs: two full waves of its resident CTAs
  int p1_grid = 0;     // P1 CTAs
  int adv_threads = 1024;  // k_advance threads (set per captured batch size)
  cudaError_t last_error = cudaSuccess;
  bool use_loop = true;  // device-side while-node available
  // programmatic dependent launch between the kernels of a step (VFB_PDL=1):
  // measured 1-4% slower than plain stream order on every workload here
  bool use_pdl = false;
  // P1 tiles staged by one bulk copy per operand block (VFB_P1_STAGING=bulk)
  // instead of 8-byte asynchronous copies
  bool p1_bulk = false;
  bool single_step = false;  // serving: one level per launch (admission between levels)
  bool use_coop = false;  // whole-GPU persistent cooperative solver (k_solve)
  int coop_grid = 0;
  bool use_cluster = false;  // cluster solver first, whole GPU for promoted instances
  int cluster_size = 0, cluster_slots = 0;
  BatchDev* d_slots = nullptr;
  void* d_slot_mem = nullptr;
  int* d_order = nullptr;
  unsigned int* d_next = nullptr;
  int slot_cap_inst = 0;        // order capacity
  uint64_t slot_chunk_cap = 0;  // chunks per slot
  int slots_built = -1;         // cluster_slots the slot workspace was built for

  // batch workspace
  int ninst_cap = 0;
  BatchDev hB{};
  BatchDev* dB = nullptr;
  InstDev* dInst = nullptr;
  int2* h_status = nullptr;   // pinned mirror of B.status_out
  unsigned int* h_ctl = nullptr;  // pinned mirror of B.ctl
  unsigned long long* d_fail = nullptr;
  uint64_t* h_stage = nullptr;  // pinned upload staging
  size_t h_stage_words = 0;
  uint64_t* d_atoms = nullptr;  // device staging of a batch's proposition rows (one upload)
  InstDev* h_recs = nullptr;    // pinned mirror of a batch's instance records (uploads, results)
  int h_recs_cap = 0;
  size_t d_atoms_words = 0;

  // graphs
  cudaGraphExec_t exec = nullptr;
  int exec_ninst = -1, exec_smem = -1, exec_grid = -1, exec_loop = -1;

  // device block cache: size -> blocks
  std::multimap<size_t, void*> free_blocks;
  std::map<void*, size_t> live_blocks;
  size_t held_bytes = 0;    // live + cached
  size_t cached_bytes = 0;  // blocks in free_blocks
  size_t peak_live = 0;     // most bytes live at once since the last trim

  // Serving arena: a serving session carves its blocks out of one device
  // allocation made when the session opens.  A cudaMallocAsync that has to
  // map fresh memory costs about 10 ms per GB on a B200, and a growth inside
  // a serve step would wait for it while every request of the step waits too.
  // Free ranges are kept by offset; a block takes the smallest range that
  // fits and a released block merges with its free neighbours.  Every user of
  // a block runs on the engine's one stream, so a range released after its
  // last launch is only handed to launches enqueued after that.
  struct Arena {
    char* base = nullptr;
    size_t size = 0;
    std::map<size_t, size_t> free_ranges;   // offset -> bytes

    bool owns(const void* p) const {
      return base && (const char*)p >= base && (const char*)p < base + size;
    }
    void* take(size_t bytes) {
      auto best = free_ranges.end();
      for (auto it = free_ranges.begin(); it != free_ranges.end(); ++it)
        if (it->second >= bytes && (best == free_ranges.end() || it->second < best->second)) best = it;
      if (best == free_ranges.end()) return nullptr;
      const size_t off = best->first, len = best->second;
      free_ranges.erase(best);
      if (len > bytes) free_ranges.emplace(off + bytes, len - bytes);
      return base + off;
    }
    void give(void* p, size_t bytes) {
      size_t off = (size_t)((char*)p - base), len = bytes;
      auto next = free_ranges.lower_bound(off);
      if (next != free_ranges.end() && off + len == next->first) {
        len += next->second;
        next = free_ranges.erase(next);
      }
      if (next != free_ranges.begin()) {
        auto prev = std::prev(next);
        if (prev->first + prev->second == off) {
          prev->second += len;
          return;
        }
      }
      free_ranges.emplace(off, len);
    }
  } arena;

  // per-call counters
  uint64_t c_h2d = 0, c_d2h = 0, c_launch = 0;
  cudaEvent_t ev_t0 = nullptr, ev_t1 = nullptr;
  cudaEvent_t ev_k[kStepLen + 1] = {};
  Prof prof[KP_N];

  // P1 launch shape by level band (zero fields: built-in), copied into every
  // prepared instance
  vfb_tune tune{};
  // autotuner: k_p1 milliseconds and levels per band of the solves running
  // under it (profile_step adds to them when set)
  double* tune_ms = nullptr;
  uint32_t* tune_levels = nullptr;

  ~Engine() { release(); }

  // Records (and with VFB_DEBUG=1 prints) the CUDA error behind a failure.
  vfb_status dev_fail(int line) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) last_error = e;
    const char* dbg = std::getenv("VFB_DEBUG");
    if (dbg && dbg[0] == '1')
      std::fprintf(stderr, "vfb: device error at vfb_engine.cu:%d: %s\n", line,
                   cudaGetErrorString(last_error));
    return VFB_DEVICE_ERROR;
  }

  void release() {
    if (stream) cudaStreamSynchronize(stream);
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
    free_workspace();
    for (auto& kv : free_blocks) cudaFree(kv.second);
    free_blocks.clear();
    for (auto& kv : live_blocks)
      if (!arena.owns(kv.first)) cudaFree(kv.first);
    live_blocks.clear();
    held_bytes = cached_bytes = 0;
    if (arena.base) cudaFree(arena.base);
    arena = Arena{};
    // the device pool keeps freed memory for reuse while the engine lives
    // (release threshold); an engine that ends gives it back to the device
    if (stream) cudaStreamSynchronize(stream);
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
    if (h_status) cudaFreeHost(h_status);
    h_status = nullptr;
    if (h_stage) cudaFreeHost(h_stage);
    h_stage = nullptr;
    if (d_fail) cudaFree(d_fail);
    d_fail = nullptr;
    if (d_atoms) cudaFree(d_atoms);
    d_atoms = nullptr;
    d_atoms_words = 0;
    if (h_recs) cudaFreeHost(h_recs);
    h_recs = nullptr;
    h_recs_cap = 0;
    if (h_ctl) cudaFreeHost(h_ctl);
    h_ctl = nullptr;
    if (d_slots) cudaFree(d_slots);
    if (d_slot_mem) cudaFree(d_slot_mem);
    if (d_order) cudaFree(d_order);
    if (d_next) cudaFree(d_next);
    d_slots = nullptr;
    d_slot_mem = nullptr;
    d_order = nullptr;
    d_next = nullptr;
    if (ev_t0) cudaEventDestroy(ev_t0);
    if (ev_t1) cudaEventDestroy(ev_t1);
    for (auto& e : ev_k)
      if (e) cudaEventDestroy(e);
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
  }

  void free_workspace() {
    auto f = [&](void* p) { if (p) cudaFree(p); };
    f(hB.p1_prefix); f(hB.chunk_prefix); f(hB.tscan_prefix); f(hB.win_prefix);
    f(hB.chunk_cnt); f(hB.chunk_base); f(hB.tickets); f(hB.status_out); f(hB.loop_iter); f(hB.ctl); f(dB);
    f(dInst);
    hB = BatchDev{};
    dB = nullptr;
    dInst = nullptr;
    ninst_cap = 0;
  }

  // ------------------------------------------------------ device blocks
  // Returns a block of at least `bytes`; *got is its real size.  The smallest
  // cached block that fits and is at most 4x the request is reused (its full
  // size becomes the capacity); larger cached blocks stay for larger requests.
  void* dalloc(size_t bytes, size_t* got) {
    if (bytes < 256) bytes = 256;
    if (arena.base) {
      // within a serving session: a range of the arena (256-byte multiples),
      // else (no range fits) the pool below, under the same budget
      const size_t n = (bytes + 255) & ~(size_t)255;
      if (!mem_limit || held_bytes + n <= mem_limit) {
        if (void* p = arena.take(n)) {
          held_bytes += n;
          live_blocks[p] = n;
          *got = n;
          peak_live = std::max(peak_live, held_bytes - cached_bytes);
          return p;
        }
      }
    }
    auto it = free_blocks.lower_bound(bytes);
    if (it != free_blocks.end() && it->first <= 4 * bytes) {
      void* p = it->second;
      *got = it->first;
      cached_bytes -= it->first;
      free_blocks.erase(it);
      live_blocks[p] = *got;
      peak_live = std::max(peak_live, held_bytes - cached_bytes);
      return p;
    }
    // make room: drop cached blocks before exceeding the budget
    while (mem_limit && held_bytes + bytes > mem_limit && !free_blocks.empty()) {
      auto big = std::prev(free_blocks.end());
      cudaFreeAsync(big->second, stream);
      held_bytes -= big->first;
      cached_bytes -= big->first;
      free_blocks.erase(big);
    }
    if (mem_limit && held_bytes + bytes > mem_limit) return nullptr;
    void* p = nullptr;
    if (cudaMallocAsync(&p, bytes, stream) != cudaSuccess) {
      cudaGetLastError();
      // the device itself is full (other contexts hold the rest): give the
      // cached blocks back to the pool and try once more
      if (free_blocks.empty()) return nullptr;
      for (auto& fb : free_blocks) {
        cudaFreeAsync(fb.second, stream);
        held_bytes -= fb.first;
      }
      free_blocks.clear();
      cached_bytes = 0;
      if (cudaMallocAsync(&p, bytes, stream) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
      }
    }
    held_bytes += bytes;
    live_blocks[p] = bytes;
    *got = bytes;
    peak_live = std::max(peak_live, held_bytes - cached_bytes);
    return p;
  }

  // After a call: keep cached at most what the call had live at its peak (the
  // blocks the next call of its kind reuses); the rest, superseded sizes from
  // buffer growth, goes back to the device's memory pool, where other
  // contexts of the process can allocate it.
  void trim_cache() {
    while (cached_bytes > peak_live && !free_blocks.empty()) {
      auto big = std::prev(free_blocks.end());
      cudaFreeAsync(big->second, stream);
      held_bytes -= big->first;
      cached_bytes -= big->first;
      free_blocks.erase(big);
    }
    peak_live = held_bytes - cached_bytes;
  }
  void dfree(void* p) {
    if (!p) return;
    auto it = live_blocks.find(p);
    if (it == live_blocks.end()) return;
    if (arena.owns(p)) {
      arena.give(p, it->second);
      held_bytes -= it->second;
      live_blocks.erase(it);
      return;
    }
    free_blocks.emplace(it->second, p);
    cached_bytes += it->second;
    live_blocks.erase(it);
  }

  vfb_status init(const vfb_opts* o) {
    device = o ? o->device : 0;
    verbose = o ? o->verbose : 0;
    profile = o ? o->profile : 0;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= device) return VFB_DEVICE_ERROR;
    if (cudaSetDevice(device) != cudaSuccess) return VFB_DEVICE_ERROR;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return VFB_DEVICE_ERROR;
    if (prop.major < 10) {
      std::fprintf(stderr, "vfb: device %d is sm_%d%d; this build targets sm_100a\n", device, prop.major,
                   prop.minor);
      return VFB_DEVICE_ERROR;
    }
    sms = prop.multiProcessorCount;
    size_t freeb = 0, total = 0;
    cudaMemGetInfo(&freeb, &total);
    // memory the process's pool holds but has not handed out is available too
    size_t pool_spare = 0;
    {
      cudaMemPool_t dp;
      uint64_t reserved = 0, used = 0;
      if (cudaDeviceGetDefaultMemPool(&dp, device) == cudaSuccess &&
          cudaMemPoolGetAttribute(dp, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
          cudaMemPoolGetAttribute(dp, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess && reserved > used)
        pool_spare = (size_t)(reserved - used);
    }
    mem_limit = (o && o->mem_limit_bytes) ? o->mem_limit_bytes : (size_t)(0.9 * (double)(freeb + pool_spare));
    if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) return VFB_DEVICE_ERROR;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t thr = ~0ULL;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    if (cudaMalloc(&d_fail, sizeof(unsigned long long)) != cudaSuccess) return VFB_DEVICE_ERROR;
    if (cudaMallocHost(&h_ctl, 4 * sizeof(unsigned int)) != cudaSuccess) return VFB_DEVICE_ERROR;
    if (cudaEventCreate(&ev_t0) != cudaSuccess || cudaEventCreate(&ev_t1) != cudaSuccess) return VFB_DEVICE_ERROR;
    for (auto& e : ev_k)
      if (cudaEventCreate(&e) != cudaSuccess) return VFB_DEVICE_ERROR;
    grid = sms * 8;
    {
      // k_emit's items are spread over its CTAs evenly, so a grid that is not
      // a whole number of waves leaves SMs idle in the last one
      int oe = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&oe, k_emit, 256, 0) != cudaSuccess || oe < 1) oe = 1;
      emit_grid = sms * oe * 2;
    }
    const int maxsmem = (kTS * (kMaxTraces + 1) + kTQ * kMaxTraces) * 8;
    if (cudaFuncSetAttribute(k_p1, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsmem) != cudaSuccess)
      return VFB_DEVICE_ERROR;
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, k_p1) != cudaSuccess) return VFB_DEVICE_ERROR;
    if (cudaFuncSetAttribute(k_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsmem) != cudaSuccess)
      return VFB_DEVICE_ERROR;
    if (cudaFuncSetAttribute(k_p1_bulk, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsmem) != cudaSuccess)
      return VFB_DEVICE_ERROR;
    const char* stg = std::getenv("VFB_P1_STAGING");
    p1_bulk = stg && std::strcmp(stg, "bulk") == 0;
    const char* pdl_env = std::getenv("VFB_PDL");
    use_pdl = pdl_env && pdl_env[0] == '1';
    const char* env = std::getenv("VFB_NO_DEVICE_LOOP");
    use_loop = !(env && env[0] == '1') && !profile;
    // level loop: persistent cooperative kernel unless profiling per kernel,
    // the device cannot co-schedule a grid, or VFB_SOLVER=graph asks otherwise
    int coop = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
    const char* sol = std::getenv("VFB_SOLVER");
    use_coop = coop && !profile && sol && std::strcmp(sol, "coop") == 0;
    // the cluster solver (one thread-block cluster per instance) is available
    // with VFB_SOLVER=cluster; measured slower than the level-synchronous
    // graph on single and batched solves, so it is not the default
    use_cluster = !profile && sol && std::strcmp(sol, "cluster") == 0;
    if (use_cluster) {
      if (cudaFuncSetAttribute(k_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsmem) != cudaSuccess)
        use_cluster = false;
      cudaFuncSetAttribute(k_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
      cudaGetLastError();
    }
    return VFB_OK;
  }

  // ------------------------------------------------------------ workspace
  vfb_status ensure_workspace(int ninst, uint64_t chunk_need) {
    if (ninst > ninst_cap || chunk_need > hB.chunk_cap) {
      if (cudaStreamSynchronize(stream) != cudaSuccess) return dev_fail(__LINE__);
      // with room to spare: a later call of the same instances starts from
      // their final capacities (the hints) and needs more chunks at once than
      // this one did; a reallocation costs a synchronisation and a new graph
      const int nc = std::max(ninst, ninst_cap);
      const uint64_t cc = std::max<uint64_t>(2 * chunk_need, hB.chunk_cap);
      BatchDev nb{};
      void* p = nullptr;
      const size_t pre = (size_t)(nc + 1) * sizeof(unsigned long long);
#define WS_ALLOC(field, bytes)                               \
  if (cudaMalloc(&p, (bytes)) != cudaSuccess) return VFB_OOM; \
  nb.field = reinterpret_cast<decltype(nb.field)>(p);
      WS_ALLOC(p1_prefix, pre)
      WS_ALLOC(chunk_prefix, pre)
      WS_ALLOC(tscan_prefix, pre)
      WS_ALLOC(win_prefix, pre)
      WS_ALLOC(chunk_cnt, std::max<uint64_t>(cc, 1) * sizeof(unsigned int))
      WS_ALLOC(chunk_base, std::max<uint64_t>(cc, 1) * sizeof(unsigned long long))
      WS_ALLOC(tickets, kTickets * sizeof(unsigned long long))
      WS_ALLOC(status_out, (size_t)nc * sizeof(int2))
      WS_ALLOC(loop_iter, sizeof(unsigned long long))
      WS_ALLOC(ctl, 4 * sizeof(unsigned int))
#undef WS_ALLOC
      cudaMemset(nb.ctl, 0, 4 * sizeof(unsigned int));
      BatchDev* ndB = nullptr;
      if (cudaMalloc((void**)&ndB, sizeof(BatchDev)) != cudaSuccess) return VFB_OOM;
      InstDev* ndI = nullptr;
      if (cudaMalloc((void**)&ndI, (size_t)nc * sizeof(InstDev)) != cudaSuccess) return VFB_OOM;
      if (dInst && ninst_cap)
        cudaMemcpy(ndI, dInst, (size_t)ninst_cap * sizeof(InstDev), cudaMemcpyDeviceToDevice);
      free_workspace();
      hB = nb;
      hB.chunk_cap = cc;
      hB.atoms = d_atoms;   // (the staging buffer is not part of the workspace)
      dB = ndB;
      dInst = ndI;
      ninst_cap = nc;
      if (h_status) cudaFreeHost(h_status);
      if (cudaMallocHost(&h_status, (size_t)nc * sizeof(int2)) != cudaSuccess) return VFB_OOM;
      if (exec) { cudaGraphExecDestroy(exec); exec = nullptr; }
    }
    hB.inst = dInst;
    hB.ninst = ninst;
    if (cudaMemcpyAsync(dB, &hB, sizeof(BatchDev), cudaMemcpyHostToDevice, stream) != cudaSuccess)
      return dev_fail(__LINE__);
    c_h2d += sizeof(BatchDev);
    return VFB_OK;
  }

  // --------------------------------------------------------- step launch
  // pre: the leading k_advance (plans instances coming from k_init or a
  // growth).  loop: the trailing k_advance sets the while-node's condition.
  // Launch of one kernel of the step; with pdl, as a programmatic dependent of
  // the kernel before it on the stream (the kernels wait for it on entry).
  template <typename... Args>
  void step_launch(bool pdl, void (*kern)(Args...), unsigned grid_x, unsigned block_x, size_t smem,
                   Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid_x);
    cfg.blockDim = dim3(block_x);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kern, args...);
  }

  void launch_step(bool pre, bool timed, int p1_smem, cudaGraphConditionalHandle handle, bool loop) {
    int e = 0;
    // external event nodes keep their timestamps inside a captured graph;
    // between them the kernels are not adjacent, so no programmatic launch
    auto mark = [&]() { if (timed) cudaEventRecordWithFlags(ev_k[e++], stream, cudaEventRecordExternal); };
    const bool pdl = use_pdl && !timed;
    const int lp = loop ? 1 : 0, built0 = 0, built1 = 1;
    unsigned int mx = kMaxLoop;
    mark();
    if (pre) {
      step_launch(false, k_advance, 1u, (unsigned)adv_threads, 0, dB, handle, built0, lp, mx);
      mark();
    }
    step_launch(pdl && pre, p1_bulk ? k_p1_bulk : k_p1, (unsigned)p1_grid, (unsigned)kTS, (size_t)p1_smem, dB);
    mark();
    step_launch(pdl, k_table_scan_check, (unsigned)grid, 256u, 0, dB);
    mark();
    step_launch(pdl, k_compact, (unsigned)(sms * 8), (unsigned)kCompactThreads, 0, dB);
    mark();
    step_launch(pdl, k_emit, (unsigned)emit_grid, 256u, 0, dB);
    mark();
    step_launch(pdl, k_advance, 1u, (unsigned)adv_threads, 0, dB, handle, built1, lp, mx);
    mark();
  }

  // Graph: [k_advance, while: (k_p1, k_table_scan_check, k_compact, k_emit, k_advance)] + status
  // read-back, or one step [k_advance, k_p1, ..., k_advance] + status read-back.
  cudaError_t build_graph(int ninst, int p1_smem) {
    if (exec) { cudaGraphExecDestroy(exec); exec = nullptr; }
    // one thread per instance (whole warps, at most 1024): small batches keep
    // k_advance's block scans short
    adv_threads = std::min(kAdvanceThreads, std::max(32, (ninst + 31) / 32 * 32));
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaGraphCreate(&graph, 0);
    if (e != cudaSuccess) return e;
    bool loop = use_loop && !single_step;
    if (loop) {
      cudaGraphConditionalHandle handle;
      e = cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault);
      cudaGraphNodeParams cp = {};
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = handle;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      // plan node (sets the condition before the first iteration), then the loop
      cudaGraphNode_t pnode = nullptr, cnode;
      if (e == cudaSuccess) {
        e = cudaStreamBeginCaptureToGraph(stream, graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
          k_advance<<<1, adv_threads, 0, stream>>>(dB, handle, 0, 1, kMaxLoop);
          cudaGraph_t out = nullptr;
          e = cudaStreamEndCapture(stream, &out);
        }
        size_t nn = 1;
        if (e == cudaSuccess) e = cudaGraphGetNodes(graph, &pnode, &nn);
      }
      if (e == cudaSuccess) e = cudaGraphAddNode(&cnode, graph, &pnode, 1, &cp);
      if (e == cudaSuccess) {
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        e = cudaStreamBeginCaptureToGraph(stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
          launch_step(false, false, p1_smem, handle, true);
          cudaGraph_t out = nullptr;
          e = cudaStreamEndCapture(stream, &out);
        }
      }
      if (e == cudaSuccess) {
        // status read-back after the loop
        e = cudaStreamBeginCaptureToGraph(stream, graph, &cnode, nullptr, 1, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
          cudaMemcpyAsync(h_status, hB.status_out, (size_t)ninst * sizeof(int2), cudaMemcpyDeviceToHost, stream);
          cudaGraph_t out = nullptr;
          e = cudaStreamEndCapture(stream, &out);
        }
      }
      if (e != cudaSuccess) {
        // no device-side loop on this driver: fall back to one step per launch
        cudaGetLastError();
        cudaGraphDestroy(graph);
        graph = nullptr;
        use_loop = false;
        loop = false;
        e = cudaGraphCreate(&graph, 0);
        if (e != cudaSuccess) return e;
      }
    }
    if (!loop) {
      e = cudaStreamBeginCaptureToGraph(stream, graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) { cudaGraphDestroy(graph); return e; }
      launch_step(true, profile != 0, p1_smem, 0, false);
      cudaMemcpyAsync(h_status, hB.status_out, (size_t)ninst * sizeof(int2), cudaMemcpyDeviceToHost, stream);
      cudaGraph_t out = nullptr;
      e = cudaStreamEndCapture(stream, &out);
      if (e != cudaSuccess) { cudaGraphDestroy(graph); return e; }
    }
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) { exec = nullptr; return e; }
    exec_ninst = ninst;
    exec_smem = p1_smem;
    exec_grid = p1_grid;
    exec_loop = loop;
    return cudaSuccess;
  }

  cudaError_t run(int ninst, int p1_smem) {
    if (use_coop && !single_step) {
      if (coop_grid <= 0) return cudaErrorInvalidConfiguration;
      const unsigned int init_ctl[2] = {0u, 1u};   // error, continue
      cudaMemcpyAsync(hB.ctl + 2, init_ctl, sizeof(init_ctl), cudaMemcpyHostToDevice, stream);
      cudaMemsetAsync(hB.loop_iter, 0, sizeof(unsigned long long), stream);
      unsigned int steps = kMaxLoop;
      void* args[] = {(void*)&dB, (void*)&steps};
      cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_solve, dim3(coop_grid), dim3(kTS), args,
                                                  (size_t)p1_smem, stream);
      if (e != cudaSuccess) return e;
      cudaMemcpyAsync(h_status, hB.status_out, (size_t)ninst * sizeof(int2), cudaMemcpyDeviceToHost, stream);
      cudaMemcpyAsync(h_ctl, hB.ctl, 4 * sizeof(unsigned int), cudaMemcpyDeviceToHost, stream);
      c_h2d += sizeof(init_ctl);
      c_d2h += (uint64_t)ninst * sizeof(int2) + 4 * sizeof(unsigned int);
      return cudaSuccess;
    }
    if (!exec || exec_ninst != ninst || exec_smem != p1_smem || exec_grid != p1_grid ||
        exec_loop != (int)(use_loop && !single_step)) {
      const cudaError_t e = build_graph(ninst, p1_smem);
      if (e != cudaSuccess) return e;
    }
    if (exec_loop) cudaMemsetAsync(hB.loop_iter, 0, sizeof(unsigned long long), stream);
    c_d2h += (uint64_t)ninst * sizeof(int2);
    return cudaGraphLaunch(exec, stream);
  }

  // ------------------------------------------------------- cluster solver
  // Largest cluster (16, else 8) that fits the P1 tile's shared memory; the
  // number of clusters that can be resident at once sets the slot count.
  void pick_cluster(int p1_smem) {
    cluster_size = 0;
    cluster_slots = 0;
    for (int cs : {16, 8}) {
      cudaLaunchConfig_t cfg = {};
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = cs;
      at[0].val.clusterDim.y = 1;
      at[0].val.clusterDim.z = 1;
      cfg.gridDim = dim3(cs);
      cfg.blockDim = dim3(kTS);
      cfg.dynamicSmemBytes = (size_t)p1_smem;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      int nc = 0;
      if (cudaOccupancyMaxActiveClusters(&nc, (const void*)k_cluster, &cfg) == cudaSuccess && nc > 0) {
        cluster_size = cs;
        cluster_slots = nc;
        return;
      }
      cudaGetLastError();
    }
  }

  // Per-slot private workspace (prefix arrays, tickets, chunk arrays).
  vfb_status ensure_slots(int n, uint64_t chunks) {
    if (cluster_slots <= 0) return dev_fail(__LINE__);
    if (n > slot_cap_inst) {
      if (d_order) cudaFree(d_order);
      if (cudaMalloc(&d_order, (size_t)n * sizeof(int)) != cudaSuccess) return VFB_OOM;
      slot_cap_inst = n;
    }
    if (!d_next && cudaMalloc(&d_next, sizeof(unsigned int)) != cudaSuccess) return VFB_OOM;
    // every slot starts on a 256-byte boundary (its arrays hold 8- and 16-byte words)
    const size_t per = (5 * 2 * 8 + 4 * 8 + 16 + 8 + (size_t)chunks * 12 + 64 + 255) & ~size_t(255);
    if (!d_slots || chunks > slot_chunk_cap || cluster_slots != slots_built) {
      if (cudaStreamSynchronize(stream) != cudaSuccess) return dev_fail(__LINE__);
      if (d_slots) cudaFree(d_slots);
      if (d_slot_mem) cudaFree(d_slot_mem);
      d_slots = nullptr;
      d_slot_mem = nullptr;
      if (cudaMalloc(&d_slots, (size_t)cluster_slots * sizeof(BatchDev)) != cudaSuccess) return VFB_OOM;
      if (cudaMalloc(&d_slot_mem, (size_t)cluster_slots * per) != cudaSuccess) return VFB_OOM;
      std::vector<BatchDev> hs(cluster_slots);
      for (int c = 0; c < cluster_slots; ++c) {
        char* m = (char*)d_slot_mem + (size_t)c * per;
        auto take = [&](size_t bytes) { char* r = m; m += (bytes + 15) & ~size_t(15); return r; };
        BatchDev& b = hs[c];
        b = BatchDev{};
        b.p1_prefix = (unsigned long long*)take(16);
        b.chunk_prefix = (unsigned long long*)take(16);
        b.tscan_prefix = (unsigned long long*)take(16);
        b.win_prefix = (unsigned long long*)take(16);
        b.tickets = (unsigned long long*)take(kTickets * sizeof(unsigned long long));
        b.status_out = (int2*)take(16);
        b.loop_iter = (unsigned long long*)take(8);
        b.chunk_cnt = (unsigned int*)take(chunks * 4);
        b.chunk_base = (unsigned long long*)take(chunks * 8);
        b.chunk_cap = chunks;
        b.ninst = 1;
      }
      if (cudaMemcpy(d_slots, hs.data(), hs.size() * sizeof(BatchDev), cudaMemcpyHostToDevice) != cudaSuccess)
        return dev_fail(__LINE__);
      slot_chunk_cap = chunks;
      slots_built = cluster_slots;
    }
    return VFB_OK;
  }

  // Run every active instance through the cluster solver.
  vfb_status run_clusters(std::vector<InstHost>& H, int n, int p1_smem) {
    std::vector<int> order;
    uint64_t chunks = 1;
    for (int i = 0; i < n; ++i) {
      if (!H[i].active) continue;
      order.push_back(i);
      chunks = std::max<uint64_t>(chunks, (H[i].d.bitmap_words + kChunkWords - 1) / kChunkWords + 1);
    }
    if (order.empty()) return VFB_OK;
    vfb_status s = ensure_slots(n, chunks);
    if (s != VFB_OK) return s;
    if (cudaMemcpyAsync(d_order, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice, stream) !=
            cudaSuccess ||
        cudaMemsetAsync(d_next, 0, sizeof(unsigned int), stream) != cudaSuccess)
      return dev_fail(__LINE__);
    c_h2d += order.size() * sizeof(int);
    ClusterWork w{d_slots, dInst, d_order, (int)order.size(), d_next};
    const int slots = std::min<int>(cluster_slots, (int)order.size());
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cluster_size;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(slots * cluster_size);
    cfg.blockDim = dim3(kTS);
    cfg.dynamicSmemBytes = (size_t)p1_smem;
    cfg.stream = stream;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    if (cudaLaunchKernelEx(&cfg, k_cluster, w) != cudaSuccess) return dev_fail(__LINE__);
    ++c_launch;
    // statuses of every instance after the cluster pass
    std::vector<InstDev> recs(n);
    if (cudaMemcpyAsync(recs.data(), dInst, (size_t)n * sizeof(InstDev), cudaMemcpyDeviceToHost, stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess)
      return dev_fail(__LINE__);
    c_d2h += (uint64_t)n * sizeof(InstDev);
    for (int i = 0; i < n; ++i) h_status[i] = make_int2(recs[i].status, recs[i].need);
    return VFB_OK;
  }

  // ------------------------------------------------------ instance buffers
  vfb_status alloc_buffers(InstHost& H, uint64_t rows, uint64_t slots, uint64_t words, uint64_t tents) {
    InstDev& d = H.d;
    size_t g1, g2, g3, g4, g5, g6;
    void* pr = dalloc(rows * (size_t)d.TP * 8, &g1);
    void* po = dalloc(rows * 8, &g2);
    void* pt = dalloc(slots * sizeof(Slot), &g3);
    void* pb = dalloc(words * 4, &g4);
    void* pw = dalloc(tents * 8, &g6);
    g5 = g6;
    if (!pr || !po || !pt || !pb || !pw) {
      dfree(pr); dfree(po); dfree(pt); dfree(pb); dfree(pw);
      return VFB_OOM;
    }
    d.rows = (uint64_t*)pr;
    d.origin = (uint64_t*)po;
    d.row_cap = std::min<uint64_t>(g1 / ((size_t)d.TP * 8), g2 / 8);
    d.table = (Slot*)pt;
    d.table_mask = pow2_at_most(g3 / sizeof(Slot)) - 1;
    d.bitmap = (uint32_t*)pb;
    d.bitmap_words = g4 / 4;
    d.wins = (uint64_t*)pw;
    d.tent_cap = std::min(g5, g6) / 8;
    // small buffers are initialised by k_fill (launched once for all new
    // instances before k_init) in place of two API calls each
    const uint64_t fill_bytes = (d.table_mask + 1) * sizeof(Slot) + d.bitmap_words * 4;
    d.fill = fill_bytes <= kInitFillMax ? 1 : 0;
    if (!d.fill) {
      cudaMemsetAsync(d.table, 0xFF, (d.table_mask + 1) * sizeof(Slot), stream);
      cudaMemsetAsync(d.bitmap, 0, d.bitmap_words * 4, stream);
    }
    return VFB_OK;
  }

  void free_buffers(InstHost& H) {
    InstDev& d = H.d;
    dfree(d.rows);
    dfree(d.origin);
    dfree(d.table);
    dfree(d.bitmap);
    dfree(d.wins);
    d.rows = d.origin = d.wins = nullptr;
    d.table = nullptr;
    d.bitmap = nullptr;
  }

  uint64_t c_grow = 0;   // buffer growths in the current call

  // Final capacities of recently solved instances, keyed by a signature of the
  // instance: a repeated instance starts with the buffers it ended with.
  struct Caps { uint64_t rows, slots, words, tents; };
  std::map<uint64_t, Caps> hints;

  static uint64_t signature(const vfb_instance& in) {
    uint64_t h = 0x9E3779B97F4A7C15ULL ^ ((uint64_t)in.num_vars << 32) ^ ((uint64_t)in.num_traces << 16) ^
                 ((uint64_t)in.num_pos << 8) ^ (uint64_t)in.max_size ^ ((uint64_t)in.rlx_type << 56);
    auto mix = [&](uint64_t x) {
      h ^= x + 0x9E3779B97F4A7C15ULL + (h << 6) + (h >> 2);
      h *= 0xBF58476D1CE4E5B9ULL;
      h ^= h >> 31;
    };
    for (int i = 0; i < in.num_traces; ++i) mix((uint64_t)in.lengths[i]);
    for (size_t i = 0; i < (size_t)in.num_traces * in.num_vars; ++i) mix(in.words[i]);
    return h;
  }

  // Grow whatever the device asked for; the level is then re-run.
  // Device bytes the buffers of one instance occupy.
  static uint64_t inst_bytes(const InstDev& d) {
    return d.row_cap * ((uint64_t)d.TP * 8 + 8) + (d.table_mask + 1) * sizeof(Slot) + d.bitmap_words * 4 +
           d.tent_cap * 8;
  }

  // Bytes an instance is expected to hold once its next level is built: the
  // next level's rows are projected from the last level-over-level growth
  // (clamped to [1, 32]); rows, table slots (kept at most half full) and the
  // owner list scale with them.
  static uint64_t projected_bytes(const InstDev& d) {
    const uint64_t held = inst_bytes(d);
    const int k = d.level;
    if (d.status != ST_RUNNING && d.status != ST_NEED_MEM) return held;
    if (k < 2 || k > (int)kMaxSize) return held;
    const uint64_t last = d.lcount[k - 1], prev = k >= 3 ? d.lcount[k - 2] : d.A;
    double ratio = prev ? (double)last / (double)prev : 1.0;
    ratio = std::min(32.0, std::max(1.0, ratio));
    const uint64_t next = (uint64_t)((double)last * ratio);
    const uint64_t rows = d.lstart[k - 1] + last + next;
    const uint64_t est = rows * ((uint64_t)d.TP * 8 + 8) + pow2_at_least(2 * (d.keys + next)) * sizeof(Slot) +
                         d.bitmap_words * 4 + next * 8;
    return std::max(held, est);
  }

  // cap_bytes > 0: the instance may hold at most that many bytes; a growth
  // past it ends the instance with VFB_LIMIT.
  vfb_status grow(InstHost& H, int idx, uint64_t cap_bytes = 0) {
    ++c_grow;
    InstDev& d = H.d;
    if (cudaMemcpyAsync(&d, dInst + idx, sizeof(InstDev), cudaMemcpyDeviceToHost, stream) != cudaSuccess)
      return dev_fail(__LINE__);
    c_d2h += sizeof(InstDev);
    if (cudaStreamSynchronize(stream) != cudaSuccess) return dev_fail(__LINE__);
    const int need = d.need;
    size_t g1, g2;
    if (std::getenv("VFB_DEBUG"))
      std::fprintf(stderr, "vfb: instance %d level %d needs %d (rows %llu/%llu slots %llu keys %llu words %llu tent %llu)\n",
                   idx, d.level, need, (unsigned long long)d.need_amount[3], (unsigned long long)d.row_cap,
                   (unsigned long long)(d.table_mask + 1), (unsigned long long)d.keys,
                   (unsigned long long)d.need_amount[0], (unsigned long long)d.need_amount[2]);
    if (need & NEED_LIMIT) return VFB_LIMIT;
    if (need & NEED_PROMOTE) d.promote_above = ~0ULL;   // continue on the whole GPU
    // Rows the plan projected (not yet the level's owner count) that the
    // budget cannot hold next to the instance's other buffers are deferred:
    // the level runs without them and its table scan asks for exactly what its
    // owners need (nothing if it settles the solution).  The test depends on
    // the instance alone (never on memory that other instances of a batch or
    // a serving session hold: those wait), so batched and served results stay
    // those of solo solves.
    const bool rows_est = (need & NEED_ROWS) && (need & NEED_ROWS_EST);
    const uint64_t row_bytes = (uint64_t)d.TP * 8 + 8;
    bool rows_wanted = (need & NEED_ROWS) != 0;
    uint64_t add = 0;   // bytes the other buffers grow by
    if (need & NEED_TABLE)
      add += pow2_at_least(std::max<uint64_t>(2 * (d.table_mask + 1), d.need_amount[1])) * sizeof(Slot);
    if (need & NEED_BITMAP) add += std::max<uint64_t>(2 * d.bitmap_words, d.need_amount[0] + d.need_amount[0] / 4) * 4;
    if (need & NEED_LIST) add += std::max<uint64_t>(2 * d.tent_cap, d.need_amount[2] + d.need_amount[2] / 4) * 8;
    const uint64_t non_rows = inst_bytes(d) - d.row_cap * row_bytes + add;
    const uint64_t limit = cap_bytes ? std::min<uint64_t>(cap_bytes, mem_limit ? mem_limit : ~0ULL)
                                     : (mem_limit ? mem_limit : ~0ULL);
    if (cap_bytes && inst_bytes(d) + add > cap_bytes) return VFB_LIMIT;
    const uint64_t rows_min = d.need_amount[3] + d.need_amount[3] / 64;   // the smallest allocation tried
    if (rows_wanted && rows_min * row_bytes + non_rows > limit) {
      if (!rows_est) {
        if (cap_bytes && rows_min * row_bytes + non_rows > cap_bytes) return VFB_LIMIT;
      } else {
        rows_wanted = false;
        d.rows_deferred = 1;
        d.need &= ~(NEED_ROWS | NEED_ROWS_EST);
      }
    }
    // bytes the rows may add under the per-request cap (no cap: unbounded)
    const uint64_t rows_room = cap_bytes ? cap_bytes - inst_bytes(d) - add : ~0ULL;
    if (rows_wanted) {
      const uint64_t exact = d.need_amount[3];
      const uint64_t used = d.lstart[d.level];
      // doubling keeps the number of growths small; when that does not fit
      // (the budget or the per-request cap), the rows asked for and 1/64
      // more are tried before giving up
      const uint64_t tries[2] = {std::max<uint64_t>(2 * d.row_cap, exact + exact / 4), rows_min};
      void* pr = nullptr;
      void* po = nullptr;
      for (int t = 0; t < 2 && !pr; ++t) {
        const uint64_t want = tries[t];
        if ((want - std::min(want, d.row_cap)) * row_bytes > rows_room) continue;
        pr = dalloc(want * (size_t)d.TP * 8, &g1);
        po = pr ? dalloc(want * 8, &g2) : nullptr;
        if (!po) {
          dfree(pr);
          pr = nullptr;
        }
      }
      if (!pr) return VFB_OOM;   // (held by other instances, or the pool is fragmented)
      {
        cudaMemcpyAsync(pr, d.rows, used * (size_t)d.TP * 8, cudaMemcpyDeviceToDevice, stream);
        cudaMemcpyAsync(po, d.origin, used * 8, cudaMemcpyDeviceToDevice, stream);
        dfree(d.rows);
        dfree(d.origin);
        d.rows = (uint64_t*)pr;
        d.origin = (uint64_t*)po;
        d.row_cap = std::min<uint64_t>(g1 / ((size_t)d.TP * 8), g2 / 8);
        d.need &= ~(NEED_ROWS | NEED_ROWS_EST);   // a later part that fails leaves this one done
      }
    }
    if (need & NEED_TABLE) {
      const uint64_t cap = d.table_mask + 1;
      const uint64_t want = pow2_at_least(std::max<uint64_t>(2 * cap, d.need_amount[1]));
      void* pt = dalloc(want * sizeof(Slot), &g1);
      if (!pt) return VFB_OOM;
      const uint64_t slots = pow2_at_most(g1 / sizeof(Slot));
      cudaMemsetAsync(pt, 0xFF, slots * sizeof(Slot), stream);
      cudaMemsetAsync(d_fail, 0, sizeof(unsigned long long), stream);
      k_rehash<<<grid, 256, 0, stream>>>(d.table, cap, (Slot*)pt, slots - 1, d_fail);
      ++c_launch;
      unsigned long long fails = 0;
      cudaMemcpyAsync(&fails, d_fail, sizeof(fails), cudaMemcpyDeviceToHost, stream);
      c_d2h += sizeof(fails);
      if (cudaStreamSynchronize(stream) != cudaSuccess) return dev_fail(__LINE__);
      if (fails) return dev_fail(__LINE__);
      dfree(d.table);
      d.table = (Slot*)pt;
      d.table_mask = slots - 1;
      d.need &= ~NEED_TABLE;
    }
    if (need & NEED_BITMAP) {
      const uint64_t want = std::max<uint64_t>(2 * d.bitmap_words, d.need_amount[0] + d.need_amount[0] / 4);
      void* pb = dalloc(want * 4, &g1);
      if (!pb) return VFB_OOM;
      cudaMemsetAsync(pb, 0, g1 / 4 * 4, stream);
      dfree(d.bitmap);
      d.bitmap = (uint32_t*)pb;
      d.bitmap_words = g1 / 4;
      d.need &= ~NEED_BITMAP;
    }
    if (need & NEED_LIST) {
      const uint64_t want = std::max<uint64_t>(2 * d.tent_cap, d.need_amount[2] + d.need_amount[2] / 4);
      void* pw = dalloc(want * 8, &g1);
      if (!pw) return VFB_OOM;
      dfree(d.wins);
      d.wins = (uint64_t*)pw;
      d.tent_cap = g1 / 8;
      d.need &= ~NEED_LIST;
    }
    d.status = ST_RUNNING;
    d.need = 0;
    d.planned = 0;   // the level is planned again with the new buffers
    if (cudaMemcpyAsync(dInst + idx, &d, sizeof(InstDev), cudaMemcpyHostToDevice, stream) != cudaSuccess)
      return dev_fail(__LINE__);
    c_h2d += sizeof(InstDev);
    return VFB_OK;
  }

  // ----------------------------------------------------------- the solve
  vfb_status prepare(const vfb_instance& in, InstHost& H) {
    InstDev& d = H.d;
    std::memset(&d, 0, sizeof(d));
    const int T = in.num_traces, A = in.num_vars;
    if (T < 1 || T > kMaxTraces || A < 1 || A > VFB_MAX_VARS || in.num_pos < 0 || in.num_pos > T)
      return VFB_LIMIT;
    if (in.max_size < 1 || in.max_size > kMaxSize) return VFB_LIMIT;
    if (!in.words || !in.lengths) return VFB_BAD_INPUT;
    const int rlx = in.rlx_type == 0 ? 3 : in.rlx_type;
    if (rlx < 1 || rlx > 3) return VFB_BAD_INPUT;
    int S = 0;
    for (int i = 0; i < T; ++i) {
      if (in.lengths[i] < 1 || in.lengths[i] > VFB_MAX_LENGTH) return VFB_LIMIT;
      S += in.lengths[i];
    }
    d.T = T;
    d.TP = T + (T & 1);
    d.A = A;
    for (int b = 0; b < kTuneBands; ++b) {
      d.tune_rows[b] = tune.rows[b];
      d.tune_tiles[b] = tune.tiles_log2[b];
      d.tune_blocks[b] = tune.blocks[b];
    }
    d.npos = in.num_pos;
    d.max_size = in.max_size;
    d.lensum = S;
    d.stride1 = 1;
    for (int i = 0; i < T; ++i) {
      d.len[i] = (uint8_t)in.lengths[i];
      if (i < in.num_pos) d.posmask[i >> 6] |= 1ULL << (i & 63);
    }
    // key layout (LTL_BS.cu:30-110): fields concatenated trace-major into 126 bits
    int width[kMaxTraces];
    if (S <= 126) {
      d.key_mode = KEY_CONCAT;
      for (int i = 0; i < T; ++i) width[i] = in.lengths[i];
    } else if (rlx == 1) {
      d.key_mode = KEY_SAMPLED;
      d.stride1 = S / 126;
      for (int i = 0; i < T; ++i) width[i] = (in.lengths[i] + d.stride1 - 1) / d.stride1;
    } else if (rlx == 2) {
      d.key_mode = KEY_CONCAT;
      for (int i = 0; i < T; ++i) width[i] = (126 * in.lengths[i] + S) / S;
    } else {
      d.key_mode = KEY_HASH;
      for (int i = 0; i < T; ++i) width[i] = 0;
    }
    int off = 0;
    for (int i = 0; i < T; ++i) {
      if (d.key_mode == KEY_HASH || off >= 126) {
        d.off[i] = 0;
        d.width[i] = 0;
      } else {
        d.off[i] = (uint8_t)off;
        d.width[i] = (uint8_t)std::min(width[i], 126 - off);
      }
      off += width[i];
    }
    // operator costs of the call (vfb_solve_costs), else unit costs
    for (int c = 0; c < 8; ++c) d.cost[c] = (uint8_t)req_cost[c];
    d.neg_type = req_neg;
    d.weighted = req_neg == 2;
    for (int c = 0; c < 8; ++c) d.weighted |= req_cost[c] > 1;
    if (atom_level(d) > d.max_size) return VFB_BAD_INPUT;
    d.status = ST_RUNNING;
    d.level = 1;
    return VFB_OK;
  }

  // Proposition rows of the instances with buffers (rows[v*TP + t] = words[t*A + v],
  // zero padding).  staged: one copy of every instance's rows into the batch's
  // staging buffer, which k_init copies into each level cache (a call of
  // hundreds of instances makes one upload, not one per instance); else each
  // instance's rows go to its level cache directly.
  vfb_status upload_atoms(const vfb_instance* ins, std::vector<InstHost>& H, int n, bool staged = false) {
    size_t words = 0;
    for (int i = 0; i < n; ++i)
      if (H[i].active && H[i].d.rows) words += (size_t)H[i].d.A * H[i].d.TP;
    if (words > h_stage_words) {
      if (h_stage) cudaFreeHost(h_stage);
      h_stage = nullptr;
      h_stage_words = 0;
      if (cudaMallocHost(&h_stage, words * 8) != cudaSuccess) return VFB_OOM;
      h_stage_words = words;
    }
    size_t o = 0;
    for (int i = 0; i < n; ++i) {
      if (!H[i].active || !H[i].d.rows) continue;   // (not started yet: no buffers)
      const InstDev& d = H[i].d;
      uint64_t* dst = h_stage + o;
      for (int v = 0; v < d.A; ++v) {
        for (int t = 0; t < d.T; ++t) dst[(size_t)v * d.TP + t] = ins[i].words[(size_t)t * d.A + v];
        if (d.TP > d.T) dst[(size_t)v * d.TP + d.T] = 0;
      }
      const size_t nb = (size_t)d.A * d.TP * 8;
      if (staged) {
        H[i].d.atoms_staged = 1;
        H[i].d.atom_off = o;
      } else {
        if (cudaMemcpyAsync(d.rows, dst, nb, cudaMemcpyHostToDevice, stream) != cudaSuccess)
          return dev_fail(__LINE__);
        c_h2d += nb;
      }
      o += (size_t)d.A * d.TP;
    }
    if (staged && o) {
      if (o > d_atoms_words) {
        if (cudaStreamSynchronize(stream) != cudaSuccess) return dev_fail(__LINE__);
        if (d_atoms) cudaFree(d_atoms);
        d_atoms = nullptr;
        d_atoms_words = 0;
        if (cudaMalloc(&d_atoms, o * 8) != cudaSuccess) return VFB_OOM;
        d_atoms_words = o;
      }
      if (cudaMemcpyAsync(d_atoms, h_stage, o * 8, cudaMemcpyHostToDevice, stream) != cudaSuccess)
        return dev_fail(__LINE__);
      c_h2d += o * 8;
    }
    hB.atoms = d_atoms;
    return VFB_OK;
  }

  // bytes each kernel of one level step had to move (see vfb_kernel_stat)
  void account_level(const InstDev& d, int k) {
    const double T8 = 8.0 * d.T;
    const uint64_t* n = d.lcount;
    double operands = (double)n[k - 1] * T8;
    for (int i = 1; 2 * i <= k - 1; ++i) {
      const int j = k - 1 - i;
      operands += (double)(i == j ? n[i] : n[i] + n[j]) * T8;
    }
    // figures of level k as recorded when it was finished
    const double cands = (double)d.built_cands, wins = (double)d.built_wins;
    const double w0 = std::ceil(cands / 32.0) * 4;
    prof[KP_P1].bytes += operands + 32.0 * cands;
    // owner scan: a listed slot costs its list entry and its payload, a full
    // scan every slot; one bitmap word update per owner
    const bool listed = d.built_scanned != d.table_mask + 1;
    prof[KP_TSCAN].bytes += (listed ? 16.0 : 32.0) * (double)d.built_scanned + 4.0 * wins;
    prof[KP_COMPACT].bytes += 2 * w0 + 8.0 * wins;
    if (!d.built_sol_known) prof[KP_EMIT].bytes += wins * (2 * T8 + 8.0 * d.TP + 16);
  }

  void profile_step(int n, std::vector<InstHost>& H) {
    float ms[kStepLen];
    for (int j = 0; j < kStepLen; ++j) {
      ms[j] = 0;
      cudaEventElapsedTime(&ms[j], ev_k[j], ev_k[j + 1]);
      prof[kStepSeq[j]].launches += 1;
      prof[kStepSeq[j]].ms += ms[j];
    }
    std::vector<InstDev> recs(n);
    cudaMemcpy(recs.data(), dInst, (size_t)n * sizeof(InstDev), cudaMemcpyDeviceToHost);
    if (tune_ms) {
      // a step that built a level (not one that stopped for memory): its
      // k_p1 time goes to the band of the level's candidate count
      for (int i = 0; i < n; ++i) {
        const InstDev& d = recs[i];
        if (!H[i].active || d.status == ST_NEED_MEM || d.built_cands == 0) continue;
        const int b = tune_band(d.built_cands);
        tune_ms[b] += ms[kStepP1];
        tune_levels[b] += 1;
      }
    }
    for (int i = 0; i < n; ++i) {
      const InstDev& d = recs[i];
      const int k = d.res_size;
      if (H[i].active && k > H[i].accounted && k >= 2 && k <= kMaxSize &&
          (d.status == ST_FOUND || d.status == ST_NOT_FOUND || d.level == k + 1)) {
        account_level(d, k);
        H[i].accounted = k;
      }
    }
  }

  // The pinned record mirror, grown to n records.
  vfb_status ensure_recs(int n) {
    if (n <= h_recs_cap) return VFB_OK;
    if (cudaStreamSynchronize(stream) != cudaSuccess) return dev_fail(__LINE__);
    if (h_recs) cudaFreeHost(h_recs);
    h_recs = nullptr;
    h_recs_cap = 0;
    if (cudaMallocHost((void**)&h_recs, (size_t)n * sizeof(InstDev)) != cudaSuccess) {
      h_recs = nullptr;
      return VFB_OOM;
    }
    h_recs_cap = n;
    return VFB_OK;
  }

  vfb_status batch(const vfb_instance* ins, int n, vfb_result* out) {
    const auto t0 = std::chrono::steady_clock::now();
    if (n <= 0) return VFB_OK;
    if (cudaSetDevice(device) != cudaSuccess) return dev_fail(__LINE__);
    c_h2d = c_d2h = c_launch = 0;
    cudaEventRecord(ev_t0, stream);
    std::vector<InstHost> H(n);
    int maxTP = 2;
    for (int i = 0; i < n; ++i) {
      std::memset(&out[i], 0, sizeof(vfb_result));
      const vfb_status s = prepare(ins[i], H[i]);
      if (s != VFB_OK) {
        H[i].fail = s;
        H[i].d.status = ST_IDLE;
        continue;
      }
      maxTP = std::max(maxTP, H[i].d.TP);
    }
    const int p1_smem = (kTS * (maxTP + 1) + kTQ * maxTP) * 8;
    int occ = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_p1, kTS, p1_smem);
    p1_grid = sms * std::max(occ, 1);
    if (use_coop) {
      int occ2 = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ2, k_solve, kTS, p1_smem);
      coop_grid = sms * occ2;
      if (coop_grid <= 0) use_coop = false;
    }
    bool clusters = use_cluster;
    if (clusters) {
      pick_cluster(p1_smem);
      clusters = cluster_size > 0;
    }

    vfb_status rc = VFB_OK;
    uint64_t chunk_need = 0;
    for (int i = 0; i < n; ++i) {
      if (H[i].fail != VFB_OK) continue;
      const InstDev& d = H[i].d;
      Caps c0 = clusters ? Caps{1u << 15, 1u << 16, 1u << 16, 1u << 16} : Caps{4096, 1u << 14, 1u << 14, 1u << 13};
      c0.rows = std::max<uint64_t>(c0.rows, (uint64_t)d.A * 16);
      Caps c = c0;
      H[i].sig = signature(ins[i]);
      auto hit = hints.find(H[i].sig);
      if (hit != hints.end()) c = hit->second;
      vfb_status s = alloc_buffers(H[i], c.rows, c.slots, c.words, c.tents);
      // the final sizes of an earlier solve do not all fit at once: start small
      if (s == VFB_OOM && hit != hints.end()) s = alloc_buffers(H[i], c0.rows, c0.slots, c0.words, c0.tents);
      H[i].d.promote_above = clusters ? kPromoteAbove : ~0ULL;
      if (s == VFB_OOM && n > 1 && !clusters) {
        // the instances before it hold the memory: it is solved alone after them
        H[i].d.status = ST_IDLE;
        H[i].active = true;
        H[i].restart = true;
        continue;
      }
      if (s != VFB_OK) { H[i].fail = s; H[i].d.status = ST_IDLE; continue; }
      H[i].active = true;
      chunk_need += (H[i].d.bitmap_words + kCompactWords - 1) / kCompactWords;
    }
    rc = upload_atoms(ins, H, n, true);
    if (rc == VFB_OK) rc = ensure_workspace(n, chunk_need + n);
    if (rc == VFB_OK) rc = ensure_recs(n);
    if (rc == VFB_OK) {
      // the records go up from the pinned mirror (the mirror is not written
      // again before the stream has passed this copy: the results come back
      // into it after the call's last synchronisation)
      for (int i = 0; i < n; ++i) h_recs[i] = H[i].d;
      if (cudaMemcpyAsync(dInst, h_recs, (size_t)n * sizeof(InstDev), cudaMemcpyHostToDevice, stream) !=
          cudaSuccess)
        rc = dev_fail(__LINE__);
      c_h2d += (uint64_t)n * sizeof(InstDev);
    }
    if (rc == VFB_OK) {
      if (profile) cudaEventRecord(ev_k[0], stream);
      k_fill<<<grid, 256, 0, stream>>>(dB);
      k_init<<<std::min(n, grid), 256, 0, stream>>>(dB);
      c_launch += 2;
      if (profile) {
        cudaEventRecord(ev_k[1], stream);
        cudaStreamSynchronize(stream);
        float ms = 0;
        cudaEventElapsedTime(&ms, ev_k[0], ev_k[1]);
        prof[KP_INIT].launches += 1;
        prof[KP_INIT].ms += ms;
      }
    }
    int guard = 0;
    bool first = true;
    if (rc == VFB_OK && clusters) {
      rc = run_clusters(H, n, p1_smem);
      first = false;
    }
    while (rc == VFB_OK) {
      if (!first) {
        bool running = false, grew = false;
        std::vector<int> waiting;
        int nrun = 0;
        for (int i = 0; i < n; ++i)
          if (H[i].active && h_status[i].x == ST_RUNNING) ++nrun;
        for (int i = 0; i < n; ++i) {
          if (!H[i].active) continue;
          const int st = h_status[i].x;
          if (st == ST_RUNNING) running = true;
          if (st == ST_NEED_MEM || st == ST_WAIT) {
            vfb_status g = grow(H[i], i);
            // buffers of instances that are done are not needed any more
            if (g == VFB_OOM && reclaim_finished(H, n)) g = grow(H[i], i);
            if (g == VFB_OOM && (nrun > 0 || grew || held_by_others(H, n, i))) {
              // the memory is held by other instances: this one waits (with
              // whatever part did grow) and tries again when the device loop
              // returns, at the latest when the others are done
              InstDev& d = H[i].d;
              d.status = ST_WAIT;
              if (cudaMemcpyAsync(dInst + i, &d, sizeof(InstDev), cudaMemcpyHostToDevice, stream) != cudaSuccess)
                rc = dev_fail(__LINE__);
              c_h2d += sizeof(InstDev);
              h_status[i].x = ST_WAIT;
              waiting.push_back(i);
              continue;
            }
            if (g == VFB_OOM && !H[i].d.on_the_fly) {
              // the level's rows do not fit the budget: test its candidates as
              // solutions without storing them (LTL_BS onTheFly)
              InstDev& d = H[i].d;
              d.on_the_fly = 1;
              d.status = ST_RUNNING;
              d.need = 0;
              d.planned = 0;
              if (cudaMemcpyAsync(dInst + i, &d, sizeof(InstDev), cudaMemcpyHostToDevice, stream) != cudaSuccess)
                g = dev_fail(__LINE__);
              else
                g = VFB_OK;
              c_h2d += sizeof(InstDev);
            }
            if (g != VFB_OK) {
              // this instance stops; the others carry on
              H[i].fail = g;
              H[i].active = false;
              const int err = ST_ERROR;
              cudaMemcpyAsync(&dInst[i].status, &err, sizeof(int), cudaMemcpyHostToDevice, stream);
              cudaStreamSynchronize(stream);
              c_h2d += sizeof(int);
              if (g == VFB_DEVICE_ERROR) rc = g;
            } else {
              running = grew = true;
            }
          }
          if (st == ST_ERROR) { H[i].fail = VFB_DEVICE_ERROR; H[i].active = false; }
        }
        if (rc != VFB_OK) break;
        const bool pressure = !waiting.empty();
        if (!running && pressure) {
          // every instance with buffers waits for memory the others hold:
          // the least advanced one gives its buffers up and is solved alone
          // after the others (its result is the same, only later)
          int v = waiting[0];
          for (int i : waiting)
            if (H[i].d.level <= H[v].d.level) v = i;
          free_buffers(H[v]);
          H[v].restart = true;
          const int idle = ST_IDLE;
          cudaMemcpyAsync(&dInst[v].status, &idle, sizeof(int), cudaMemcpyHostToDevice, stream);
          c_h2d += sizeof(int);
          h_status[v].x = ST_IDLE;
          running = true;   // the others retry their growth on the next pass
        }
        if (!running || rc != VFB_OK) break;
        if (grew) {
          uint64_t cn = 0;
          for (int i = 0; i < n; ++i)
            if (H[i].d.bitmap) cn += (H[i].d.bitmap_words + kCompactWords - 1) / kCompactWords;
          if (cn + n > hB.chunk_cap) {
            rc = ensure_workspace(n, cn + n);
            if (rc != VFB_OK) break;
          }
        }
      }
      first = false;
      cudaError_t e = run(n, p1_smem);
      if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
      if (e != cudaSuccess) { last_error = e; rc = dev_fail(__LINE__); break; }
      if (use_coop) {
        c_launch += 1;
        if (h_ctl[2] != 0) { rc = dev_fail(__LINE__); break; }
      } else {
        c_launch += exec_loop ? 0 : (uint64_t)kStepLen;
      }
      if (!use_coop && exec_loop) {
        // the plan node, then kBodyLen kernels per loop iteration (each
        // k_advance counts one iteration)
        unsigned long long it = 0;
        cudaMemcpy(&it, hB.loop_iter, sizeof(it), cudaMemcpyDeviceToHost);
        c_d2h += sizeof(it);
        c_launch += it ? 1 + (it - 1) * kBodyLen : 0;
      }
      if (profile) profile_step(n, H);
      if (verbose) report_progress(n);
      // (a bound on host passes: every level and growth of every instance, with
      // room for the waits and restarts of a batch under memory pressure)
      if (++guard > 64 * kMaxSize * std::max(1, n)) { rc = dev_fail(__LINE__); break; }
    }
    // results (into the pinned mirror when it holds the batch)
    std::vector<InstDev> recs_pageable;
    InstDev* recs = h_recs_cap >= n ? h_recs : nullptr;
    if (!recs) {
      recs_pageable.resize(n);
      recs = recs_pageable.data();
    }
    if (cudaMemcpyAsync(recs, dInst, (size_t)n * sizeof(InstDev), cudaMemcpyDeviceToHost, stream) !=
            cudaSuccess) {
      if (rc == VFB_OK) rc = dev_fail(__LINE__);
    }
    c_d2h += (uint64_t)n * sizeof(InstDev);
    cudaEventRecord(ev_t1, stream);
    if (cudaStreamSynchronize(stream) != cudaSuccess && rc == VFB_OK) rc = dev_fail(__LINE__);
    float dev_ms = 0;
    cudaEventElapsedTime(&dev_ms, ev_t0, ev_t1);
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    for (int i = 0; i < n; ++i) {
      vfb_result& r = out[i];
      const InstDev& d = recs[i];
      r.seconds = secs;
      r.device_seconds = dev_ms * 1e-3;
      r.h2d_bytes = c_h2d;
      r.d2h_bytes = c_d2h;
      r.kernel_launches = c_launch;
      if (H[i].fail != VFB_OK && !H[i].d.rows) {
        r.status = H[i].fail;
        continue;
      }
      r.size = d.res_size;
      const int top = std::min(d.res_size, (int)kMaxSize);
      uint64_t tot = 0;
      for (int k = 1; k <= top; ++k) {
        r.level_rows[k] = d.lcount[k];
        r.level_cands[k] = d.lcands[k];
        tot += d.lcount[k];
      }
      r.total_rows = tot;
      if (d.status == ST_FOUND) {
        r.status = VFB_OK;
        r.rpn_len = d.rpn_len;
        for (int j = 0; j < d.rpn_len && j < kMaxSize; ++j) r.rpn[j] = d.rpn[j];
        r.solution_index = d.sol_index;
        if (d.rpn_len < 1 || rpn_cost(d, d.rpn, d.rpn_len) != d.res_size) r.status = VFB_DEVICE_ERROR;
      } else if (d.status == ST_NOT_FOUND) {
        r.status = VFB_NOT_FOUND;
      } else if (d.status == ST_LIMIT) {
        r.status = VFB_LIMIT;   // the on-the-fly level held no solution; sizes are the stored levels
      } else {
        r.status = H[i].fail != VFB_OK ? H[i].fail : (rc != VFB_OK ? rc : VFB_DEVICE_ERROR);
        // the level in progress is not complete: report the finished ones
        if (r.size >= 1 && d.level <= r.size) {
          r.total_rows -= r.level_rows[r.size];
          r.level_rows[r.size] = 0;
          r.level_cands[r.size] = 0;
          r.size = std::max(0, r.size - 1);
        }
      }
    }
    if (bs_max > 0 && rc == VFB_OK) {
      for (int i = 0; i < n; ++i) {
        if (!H[i].d.rows || recs[i].status != ST_NOT_FOUND || bs_max <= recs[i].max_size) continue;
        const vfb_status s = bs_stage(i, recs[i], out[i]);
        if (s != VFB_OK) out[i].status = s;
      }
      float ms2 = 0;
      cudaEventRecord(ev_t1, stream);
      cudaStreamSynchronize(stream);
      cudaEventElapsedTime(&ms2, ev_t0, ev_t1);
      const double secs2 = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      for (int i = 0; i < n; ++i) {
        out[i].device_seconds = ms2 * 1e-3;
        out[i].seconds = secs2;
        out[i].kernel_launches = c_launch;
      }
    }
    for (int i = 0; i < n; ++i) {
      // (an instance whose buffers were reclaimed during the call has its
      // final capacities in its record all the same)
      if (H[i].fail == VFB_OK && (recs[i].status == ST_FOUND || recs[i].status == ST_NOT_FOUND)) {
        if (hints.size() > 4096) hints.clear();
        hints[H[i].sig] = Caps{recs[i].row_cap, recs[i].table_mask + 1, recs[i].bitmap_words, recs[i].tent_cap};
      }
      if (H[i].d.rows) free_buffers(H[i]);
    }
    trim_cache();
    // evicted instances, and ones whose first buffers did not fit, are solved
    // alone now that the others' buffers are free
    if (rc == VFB_OK) {
      std::vector<int> later;
      for (int i = 0; i < n; ++i)
        if (H[i].restart) later.push_back(i);
      for (int i : later) {
        vfb_result r;
        const vfb_status s = batch(&ins[i], 1, &r);
        out[i] = r;
        if (s != VFB_OK) out[i].status = s;
      }
    }
    return rc;
  }

  // Frees the buffers of instances whose search is over (their results are in
  // their device records); returns whether anything was freed.  Not while a
  // BS stage is to follow: it reads the cached rows.
  // Whether an instance other than i still holds buffers and has not finished.
  bool held_by_others(const std::vector<InstHost>& H, int n, int i) const {
    for (int j = 0; j < n; ++j) {
      if (j == i || !H[j].d.rows) continue;
      const int st = h_status[j].x;
      if (st == ST_RUNNING || st == ST_NEED_MEM || st == ST_WAIT) return true;
    }
    return false;
  }

  bool reclaim_finished(std::vector<InstHost>& H, int n) {
    if (bs_max > 0) return false;
    bool any = false;
    for (int j = 0; j < n; ++j) {
      if (!H[j].d.rows) continue;
      const int st = h_status[j].x;
      if (st == ST_FOUND || st == ST_NOT_FOUND || st == ST_LIMIT) {
        free_buffers(H[j]);
        any = true;
      }
    }
    return any;
  }

  void report_progress(int n) {
    for (int i = 0; i < n; ++i) {
      InstDev d;
      if (cudaMemcpy(&d, dInst + i, sizeof(InstDev), cudaMemcpyDeviceToHost) != cudaSuccess) return;
      if (d.status == ST_NEED_MEM) continue;
      const int k = d.res_size;
      if (k < 1 || k > kMaxSize) continue;
      for (int j = 2; j <= k; ++j)
        std::fprintf(stderr, "Length %-2d | (all) | CheckedLTLs: %-13llu | UniqueCS: %-12llu\n", j,
                     (unsigned long long)d.lcands[j], (unsigned long long)d.lcount[j]);
    }
  }

  // ============================================================ serving
  // A session keeps `cap` instance slots resident on the device.  Each step
  // admits queued requests into free slots (while the projected memory fits),
  // builds one level of every active instance with the captured step graph,
  // grows buffers where asked, and hands back finished results.
  struct Pending {
    uint64_t tag;
    vfb_instance in;
    std::vector<uint64_t> words;
    std::vector<int> lengths;
    bool evicted = false;   // gave its slot up for memory: waits until no request waits
  };
  struct Session {
    int cap = 0;
    std::vector<InstHost> H;
    std::vector<uint64_t> tag;
    std::vector<char> busy;
    std::deque<Pending> queue;
    std::vector<uint64_t> proj;   // projected bytes of each busy slot after its next level
    std::vector<Pending> req;     // the request each busy slot holds (requeued if it is evicted)
    std::vector<int> waited;      // consecutive steps each busy slot has waited for memory
    bool pressure = false;        // some request waited for memory in the last step
    uint64_t evictions = 0;       // requests evicted and queued again (memory held by the others)
    InstDev* h_inst = nullptr;    // pinned mirror of the slot records
    int p1_smem = 0;
    double budget_frac = 0.8;     // admission: projected bytes of all slots <= budget_frac * budget
    uint64_t request_bytes = 0;   // per-request cap (0: a quarter of the budget)
    uint64_t step_cands = 0;      // P1 candidates per request per step (0: whole levels)
  } sv;

  // Admission fraction, per-request byte cap and per-step candidate slice of
  // the serving session.
  vfb_status serve_limits(double budget_frac, uint64_t request_bytes, uint64_t step_candidates) {
    if (!(budget_frac > 0.0 && budget_frac <= 1.0)) return VFB_BAD_INPUT;
    sv_budget_frac = budget_frac;
    sv_request_bytes = request_bytes;
    sv_step_cands = step_candidates;
    sv.budget_frac = budget_frac;
    sv.request_bytes = request_bytes;
    sv.step_cands = step_candidates;
    return VFB_OK;
  }
  double sv_budget_frac = 0.8;
  uint64_t sv_request_bytes = 0;
  uint64_t sv_step_cands = kServeStepCands;

  vfb_status serve_open(int slots, int max_traces) {
    if (slots <= 0) return VFB_BAD_INPUT;
    if (cudaSetDevice(device) != cudaSuccess) return dev_fail(__LINE__);
    serve_close();
    sv.cap = slots;
    sv.H.assign(slots, InstHost{});
    sv.tag.assign(slots, 0);
    sv.busy.assign(slots, 0);
    sv.proj.assign(slots, 0);
    sv.req.clear();
    sv.req.resize(slots);
    sv.waited.assign(slots, 0);
    sv.budget_frac = sv_budget_frac;
    sv.request_bytes = sv_request_bytes ? sv_request_bytes : (uint64_t)(mem_limit / 4);
    sv.step_cands = sv_step_cands;
    open_arena();
    if (cudaMallocHost(&sv.h_inst, (size_t)slots * sizeof(InstDev)) != cudaSuccess) {
      sv.h_inst = nullptr;
      return VFB_OOM;
    }
    const int tp = std::max(2, std::min(max_traces, (int)kMaxTraces) + (max_traces & 1));
    sv.p1_smem = (kTS * (tp + 1) + kTQ * tp) * 8;
    int occ = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_p1, kTS, sv.p1_smem);
    p1_grid = sms * std::max(occ, 1);
    vfb_status rc = ensure_workspace(slots, (uint64_t)slots * 8);
    if (rc != VFB_OK) return rc;
    std::vector<InstDev> idle(slots);
    std::memset(idle.data(), 0, idle.size() * sizeof(InstDev));
    if (cudaMemcpyAsync(dInst, idle.data(), idle.size() * sizeof(InstDev), cudaMemcpyHostToDevice, stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess)
      return dev_fail(__LINE__);
    single_step = true;
    return VFB_OK;
  }

  // The arena of a serving session: the budget less what is live, in one
  // allocation (halved until it can be had, down to 1 GB; without one, blocks
  // come from the pool as in a solve).  The cached blocks go back to the pool
  // first, since the arena takes their memory.
  void open_arena() {
    if (arena.base) return;
    for (auto& kv : free_blocks) cudaFreeAsync(kv.second, stream);
    free_blocks.clear();
    held_bytes -= cached_bytes;
    cached_bytes = 0;
    const size_t gran = (size_t)1 << 21;
    size_t want = mem_limit > held_bytes ? (mem_limit - held_bytes) & ~(gran - 1) : 0;
    size_t least = (size_t)1 << 30;
    // VFB_SERVE_ARENA_MB caps the arena (a small one makes most blocks come
    // from the pool: the path a fragmented arena takes)
    if (const char* cap = std::getenv("VFB_SERVE_ARENA_MB")) {
      const size_t mb = (size_t)std::strtoull(cap, nullptr, 10);
      if (mb) {
        want = std::min(want, (mb << 20) & ~(gran - 1));
        least = std::min(least, want);
      }
    }
    void* p = nullptr;
    while (want >= least && want > 0) {
      if (cudaMallocAsync(&p, want, stream) == cudaSuccess) break;
      cudaGetLastError();
      p = nullptr;
      want = (want / 2) & ~(gran - 1);
    }
    if (!p || cudaStreamSynchronize(stream) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    arena.base = (char*)p;
    arena.size = want;
    arena.free_ranges.clear();
    arena.free_ranges.emplace(0, want);
  }

  // Gives the arena back to the pool once none of its blocks is live.
  void close_arena() {
    if (!arena.base) return;
    for (auto& kv : live_blocks)
      if (arena.owns(kv.first)) return;
    cudaFreeAsync(arena.base, stream);
    arena = Arena{};
  }

  void serve_close() {
    for (int i = 0; i < sv.cap; ++i)
      if (sv.busy[i] && sv.H[i].d.rows) free_buffers(sv.H[i]);
    if (sv.h_inst) cudaFreeHost(sv.h_inst);
    sv = Session{};
    close_arena();
    trim_cache();
    single_step = false;
    if (exec) { cudaGraphExecDestroy(exec); exec = nullptr; }
  }

  vfb_status serve_submit(const vfb_instance* in, uint64_t tag) {
    if (!in || !in->words || !in->lengths || in->num_traces < 1 || in->num_vars < 1) return VFB_BAD_INPUT;
    Pending p;
    p.tag = tag;
    p.in = *in;
    p.words.assign(in->words, in->words + (size_t)in->num_traces * in->num_vars);
    p.lengths.assign(in->lengths, in->lengths + in->num_traces);
    p.in.words = p.words.data();
    p.in.lengths = p.lengths.data();
    sv.queue.push_back(std::move(p));
    sv.queue.back().in.words = sv.queue.back().words.data();
    sv.queue.back().in.lengths = sv.queue.back().lengths.data();
    return VFB_OK;
  }

  // Result of a finished slot (same fields as vfb_solve's).
  void slot_result(const InstDev& d, const InstHost& H, vfb_result& r) {
    std::memset(&r, 0, sizeof(r));
    r.size = d.res_size;
    const int top = std::min(d.res_size, (int)kMaxSize);
    uint64_t tot = 0;
    for (int k = 1; k <= top; ++k) {
      r.level_rows[k] = d.lcount[k];
      r.level_cands[k] = d.lcands[k];
      tot += d.lcount[k];
    }
    r.total_rows = tot;
    if (d.status == ST_FOUND) {
      r.status = VFB_OK;
      r.rpn_len = d.rpn_len;
      for (int j = 0; j < d.rpn_len && j < kMaxSize; ++j) r.rpn[j] = d.rpn[j];
      r.solution_index = d.sol_index;
    } else if (d.status == ST_NOT_FOUND) {
      r.status = VFB_NOT_FOUND;
    } else if (d.status == ST_LIMIT) {
      r.status = VFB_LIMIT;
    } else {
      r.status = H.fail != VFB_OK ? H.fail : VFB_DEVICE_ERROR;
      if (r.size >= 1 && d.level <= r.size) {
        r.total_rows -= r.level_rows[r.size];
        r.level_rows[r.size] = 0;
        r.level_cands[r.size] = 0;
        r.size = std::max(0, r.size - 1);
      }
    }
  }

  vfb_status serve_step(vfb_served* done, int cap_done, int* ndone, int* active, int* queued) {
    *ndone = 0;
    if (sv.cap <= 0) return VFB_BAD_INPUT;
    if (cudaSetDevice(device) != cudaSuccess) return dev_fail(__LINE__);
    // 1. admission, while the projected bytes of all slots fit the budget;
    // with no slot busy the head of the queue is always admitted
    bool admitted = false;
    uint64_t committed = 0;
    int nbusy = 0;
    for (int i = 0; i < sv.cap; ++i)
      if (sv.busy[i]) { committed += sv.proj[i]; ++nbusy; }
    const double budget = sv.budget_frac * (double)mem_limit;
    const uint64_t live = held_bytes - cached_bytes;
    for (int i = 0; i < sv.cap && !sv.queue.empty(); ++i) {
      if (sv.busy[i]) continue;
      // past the projected budget only a light request still goes in, when
      // its first buffers fit the memory budget beside what is live now
      const bool over = mem_limit && nbusy > 0 && (double)committed > budget;
      Pending& p = sv.queue.front();
      // an evicted request comes back once no request waits for memory
      // (else it would take memory the waiting ones need and be evicted again)
      if (p.evicted && sv.pressure && nbusy > 0) break;
      InstHost& H = sv.H[i];
      H = InstHost{};
      vfb_status s = prepare(p.in, H);
      const int tp = p.in.num_traces + (p.in.num_traces & 1);
      if (s == VFB_OK && (kTS * (tp + 1) + kTQ * tp) * 8 > sv.p1_smem) s = VFB_LIMIT;
      if (s == VFB_OK) {
        Caps c{4096, 1u << 14, 1u << 14, 1u << 13};
        c.rows = std::max<uint64_t>(c.rows, (uint64_t)H.d.A * 16);
        H.sig = signature(p.in);
        auto hit = hints.find(H.sig);
        if (hit != hints.end()) {
          const Caps& h = hit->second;
          const uint64_t hb = h.rows * ((uint64_t)H.d.TP * 8 + 8) + h.slots * sizeof(Slot) + h.words * 4 + h.tents * 8;
          if (hb <= sv.request_bytes) c = h;
        }
        if (over) {
          const uint64_t cb = c.rows * ((uint64_t)H.d.TP * 8 + 8) + c.slots * sizeof(Slot) + c.words * 4 + c.tents * 8;
          if (cb > kLightRequestBytes || live + cb > mem_limit) {
            H = InstHost{};
            break;
          }
        }
        s = alloc_buffers(H, c.rows, c.slots, c.words, c.tents);
        if (s == VFB_OOM && nbusy > 0) {
          // the memory is held by the requests on the device: admit later
          H = InstHost{};
          break;
        }
        H.d.promote_above = ~0ULL;
        H.d.p1_quota = sv.step_cands;
      }
      if (s == VFB_OK) {
        std::vector<InstHost> one(1);
        one[0] = H;
        one[0].active = true;
        s = upload_atoms(&p.in, one, 1);
        if (s == VFB_OK &&
            cudaMemcpyAsync(dInst + i, &H.d, sizeof(InstDev), cudaMemcpyHostToDevice, stream) != cudaSuccess)
          s = dev_fail(__LINE__);
        if (s == VFB_OK && cudaStreamSynchronize(stream) != cudaSuccess) s = dev_fail(__LINE__);
      }
      if (s != VFB_OK) {
        // refused: report it as finished with that status
        if (H.d.rows) free_buffers(H);
        if (*ndone < cap_done) {
          std::memset(&done[*ndone], 0, sizeof(vfb_served));
          done[*ndone].tag = p.tag;
          done[*ndone].result.status = s;
          ++*ndone;
        }
        sv.queue.pop_front();
        continue;
      }
      H.active = true;
      sv.busy[i] = 1;
      sv.tag[i] = p.tag;
      sv.proj[i] = inst_bytes(H.d);
      committed += sv.proj[i];
      ++nbusy;
      sv.req[i] = std::move(sv.queue.front());
      sv.req[i].in.words = sv.req[i].words.data();
      sv.req[i].in.lengths = sv.req[i].lengths.data();
      sv.queue.pop_front();
      admitted = true;
    }
    if (admitted) {
      k_fill<<<grid, 256, 0, stream>>>(dB);
      k_init<<<std::min(sv.cap, grid), 256, 0, stream>>>(dB);
      c_launch += 2;
    }
    // 2. one level for every active instance
    int running = 0;
    for (int i = 0; i < sv.cap; ++i) running += sv.busy[i];
    if (running) {
      uint64_t cn = 0;
      for (int i = 0; i < sv.cap; ++i)
        if (sv.busy[i]) cn += (sv.H[i].d.bitmap_words + kCompactWords - 1) / kCompactWords;
      if (cn + sv.cap > hB.chunk_cap) {
        const vfb_status s = ensure_workspace(sv.cap, cn + sv.cap);
        if (s != VFB_OK) return s;
      }
      cudaError_t e = run(sv.cap, sv.p1_smem);
      if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
      if (e != cudaSuccess) { last_error = e; return dev_fail(__LINE__); }
      ++c_launch;
    }
    // 3. growth and 4. harvest.  A growth that finds the device memory held
    // by other requests waits: the record (with whatever part did grow) goes
    // back to the device still asking, and the growth is tried again after
    // the next step.  When no request can go on (every busy one waits and
    // none finished), the waiting request with the fewest levels built is
    // evicted and queued again at the front, to restart once memory frees;
    // a request that waits alone cannot grow at all and goes on as a solo
    // solve would, its level tested on the fly.  Results stay those of solo
    // solves.
    std::vector<int> fin, waiting;
    bool progress = false;
    for (int i = 0; i < sv.cap; ++i) {
      if (!sv.busy[i]) continue;
      const int st = h_status[i].x;
      if (st == ST_NEED_MEM) {
        const vfb_status g = grow(sv.H[i], i, sv.request_bytes);
        if (g == VFB_OOM) {
          InstDev& d = sv.H[i].d;
          d.status = ST_NEED_MEM;
          if (cudaMemcpyAsync(dInst + i, &d, sizeof(InstDev), cudaMemcpyHostToDevice, stream) != cudaSuccess)
            return dev_fail(__LINE__);
          c_h2d += sizeof(InstDev);
          waiting.push_back(i);
          ++sv.waited[i];
        } else if (g != VFB_OK) {
          sv.H[i].fail = g;
          const int err = ST_ERROR;
          cudaMemcpyAsync(&dInst[i].status, &err, sizeof(int), cudaMemcpyHostToDevice, stream);
          fin.push_back(i);
        } else {
          progress = true;
          sv.waited[i] = 0;
        }
      } else if (st == ST_FOUND || st == ST_NOT_FOUND || st == ST_ERROR || st == ST_LIMIT) {
        fin.push_back(i);
      } else if (st == ST_RUNNING) {
        progress = true;
      }
    }
    // requests that wait for one another while others keep the device busy
    // (light requests, which free little) are a deadlock too once it lasts
    sv.pressure = !waiting.empty();
    int longest = 0;
    for (int i : waiting) longest = std::max(longest, sv.waited[i]);
    const bool stuck = waiting.size() >= 2 && longest >= kServeWaitSteps;
    if ((!progress || stuck) && fin.empty() && !waiting.empty()) {
      if (waiting.size() == 1) {
        const int i = waiting[0];
        InstDev& d = sv.H[i].d;
        d.on_the_fly = 1;
        d.status = ST_RUNNING;
        d.need = 0;
        d.planned = 0;
        if (cudaMemcpyAsync(dInst + i, &d, sizeof(InstDev), cudaMemcpyHostToDevice, stream) != cudaSuccess)
          return dev_fail(__LINE__);
        c_h2d += sizeof(InstDev);
      } else {
        int v = waiting[0];
        for (int i : waiting)
          if (sv.H[i].d.level <= sv.H[v].d.level) v = i;
        free_buffers(sv.H[v]);
        sv.H[v] = InstHost{};
        sv.busy[v] = 0;
        for (int i : waiting) sv.waited[i] = 0;
        sv.req[v].evicted = true;
        sv.queue.push_front(std::move(sv.req[v]));
        sv.queue.front().in.words = sv.queue.front().words.data();
        sv.queue.front().in.lengths = sv.queue.front().lengths.data();
        const int idle = ST_IDLE;
        cudaMemcpyAsync(&dInst[v].status, &idle, sizeof(int), cudaMemcpyHostToDevice, stream);
        ++sv.evictions;
      }
    }
    for (int i : fin) {
      if (*ndone >= cap_done) break;
      InstDev d;
      if (cudaMemcpyAsync(&d, dInst + i, sizeof(InstDev), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
          cudaStreamSynchronize(stream) != cudaSuccess)
        return dev_fail(__LINE__);
      vfb_served& out = done[(*ndone)++];
      out.tag = sv.tag[i];
      slot_result(d, sv.H[i], out.result);
      if (d.status == ST_FOUND || d.status == ST_NOT_FOUND) {
        if (hints.size() > 4096) hints.clear();
        hints[sv.H[i].sig] = Caps{d.row_cap, d.table_mask + 1, d.bitmap_words, d.tent_cap};
      }
      free_buffers(sv.H[i]);
      sv.H[i] = InstHost{};
      sv.busy[i] = 0;
      const int idle = ST_IDLE;
      cudaMemcpyAsync(&dInst[i].status, &idle, sizeof(int), cudaMemcpyHostToDevice, stream);
    }
    // 5. projections for the next admission (only needed while requests wait)
    int act = 0;
    for (int i = 0; i < sv.cap; ++i) act += sv.busy[i];
    if (act && !sv.queue.empty() && mem_limit) {
      if (cudaMemcpyAsync(sv.h_inst, dInst, (size_t)sv.cap * sizeof(InstDev), cudaMemcpyDeviceToHost, stream) !=
          cudaSuccess)
        return dev_fail(__LINE__);
      if (cudaStreamSynchronize(stream) != cudaSuccess) return dev_fail(__LINE__);
      for (int i = 0; i < sv.cap; ++i)
        if (sv.busy[i]) sv.proj[i] = projected_bytes(sv.h_inst[i]);
    } else {
      cudaStreamSynchronize(stream);
    }
    if (active) *active = act;
    if (queued) *queued = (int)sv.queue.size();
    return VFB_OK;
  }

  // ================================================================ BS stage
  // After instance i (record d) found nothing up to its max size: ~ & |
  // combinations of its cached formulas over their step-0 vectors, sizes up to
  // bs_max (kernels in vfb_bs.cu).  Fills r's sizes above max_size; the
  // instance's buffers must still be held.
  int bs_max = 0;   // set by vfb_solve_bs for the call
  int req_cost[8] = {1, 1, 1, 1, 1, 1, 1, 1};   // set by vfb_solve_costs for the call
  int req_neg = 1;

  // Cost of an RPN formula under an instance's operator costs.
  static int rpn_cost(const InstDev& d, const int16_t* rpn, int n) {
    int c = 0;
    for (int j = 0; j < n; ++j) c += rpn[j] >= 0 ? atom_level(d) : op_cost(d, -rpn[j] - 1);
    return c;
  }

  vfb_status bs_stage(int i, const InstDev& d, vfb_result& r) {
    const int K = d.max_size, T = d.T;
    if (T > 64 || bs_max > kMaxSize) return VFB_LIMIT;
    for (int c = 0; c < 8; ++c)
      if (d.cost[c] > 1) return VFB_BAD_INPUT;   // the BS stage uses unit costs
    const uint64_t nrows = d.lstart[K] + d.lcount[K];
    BsDev D;
    std::memset(&D, 0, sizeof(D));
    D.rows = d.rows;
    D.T = T;
    D.TP = d.TP;
    D.full = T == 64 ? ~0ULL : ((1ULL << T) - 1);
    D.target = d.npos == 64 ? ~0ULL : ((1ULL << d.npos) - 1);
    std::vector<void*> held;
    auto take = [&](size_t bytes) -> void* {
      size_t g = 0;
      void* p = dalloc(bytes, &g);
      if (p) held.push_back(p);
      return p;
    };
    auto release = [&]() { for (void* p : held) dfree(p); held.clear(); };
    vfb_status rc = VFB_OK;
    // entries of the base and of every size: at most one per cache row or candidate
    uint64_t ent_cap = nrows + 1024, slots = pow2_at_least(4 * ent_cap), words_cap = (nrows + 31) / 32 + 1;
    uint64_t chunk_cap = (words_cap + kBsChunkWords - 1) / kBsChunkWords + 1;
    D.tab = (Slot*)take(slots * sizeof(Slot));
    D.vals = (uint64_t*)take(ent_cap * 8);
    D.org = (uint64_t*)take(ent_cap * 8);
    D.bitmap = (uint32_t*)take(words_cap * 4);
    D.counts = (unsigned long long*)take(chunk_cap * 8);
    D.offs = (unsigned long long*)take(chunk_cap * 8);
    D.best = (unsigned long long*)take(64);
    D.fail = D.best + 1;
    unsigned long long* bnd = (unsigned long long*)take(2 * (kMaxSize + 2) * 8);
    if (!D.tab || !D.vals || !D.org || !D.bitmap || !D.counts || !D.offs || !D.best || !bnd) {
      release();
      return VFB_OOM;
    }
    D.mask = slots - 1;
    cudaMemsetAsync(D.tab, 0xFF, slots * sizeof(Slot), stream);
    cudaMemsetAsync(D.bitmap, 0, words_cap * 4, stream);
    cudaMemsetAsync(D.best, 0xFF, 8, stream);
    cudaMemsetAsync(D.fail, 0, 8, stream);
    const int g256 = sms * 8;
    std::vector<unsigned long long> hcount;
    // compaction of the owner bits below nbits into entries from out0
    auto compact = [&](int c, uint64_t nbits, uint64_t out0, uint64_t& n_out) -> vfb_status {
      const uint64_t nwords = (nbits + 31) / 32;
      const unsigned chunks = (unsigned)((nwords + kBsChunkWords - 1) / kBsChunkWords);
      if (chunks == 0) { n_out = 0; return VFB_OK; }
      k_bs_count<<<chunks, 256, 0, stream>>>(D, (unsigned long long)nwords);
      hcount.assign(chunks, 0);
      if (cudaMemcpyAsync(hcount.data(), D.counts, chunks * 8, cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
          cudaStreamSynchronize(stream) != cudaSuccess)
        return dev_fail(__LINE__);
      unsigned long long run = 0;
      for (unsigned j = 0; j < chunks; ++j) { const unsigned long long x = hcount[j]; hcount[j] = run; run += x; }
      if (out0 + run > ent_cap) return VFB_OOM;
      cudaMemcpyAsync(D.offs, hcount.data(), chunks * 8, cudaMemcpyHostToDevice, stream);
      k_bs_emit<<<chunks, 256, 0, stream>>>(D, c, (unsigned long long)nwords, (unsigned long long)out0);
      c_launch += 2;
      n_out = run;
      return VFB_OK;
    };
    // base entries: the rows' words, first occurrence in row order
    k_bs_base<<<g256, 256, 0, stream>>>(D, (unsigned long long)nrows);
    k_bs_mark<<<g256, 256, 0, stream>>>(D, 0, (unsigned long long)slots, (unsigned long long)nrows);
    c_launch += 2;
    uint64_t nent = 0;
    rc = compact(0, nrows, 0, nent);
    unsigned long long fails = 0;
    if (rc == VFB_OK) {
      std::vector<unsigned long long> at(K + 1), pos(K + 1);
      for (int c = 1; c <= K; ++c) at[c - 1] = d.lstart[c];
      at[K] = nrows;
      cudaMemcpyAsync(bnd, at.data(), (K + 1) * 8, cudaMemcpyHostToDevice, stream);
      k_bs_bounds<<<1, 64, 0, stream>>>(D, (unsigned long long)nent, bnd, K + 1, bnd + kMaxSize + 2);
      ++c_launch;
      cudaMemcpyAsync(pos.data(), bnd + kMaxSize + 2, (K + 1) * 8, cudaMemcpyDeviceToHost, stream);
      cudaMemcpyAsync(&fails, D.fail, 8, cudaMemcpyDeviceToHost, stream);
      if (cudaStreamSynchronize(stream) != cudaSuccess) rc = dev_fail(__LINE__);
      for (int c = 1; c <= K; ++c) {
        D.st[c] = pos[c - 1];
        D.cn[c] = pos[c] - pos[c - 1];
      }
    }
    if (rc == VFB_OK && fails) rc = VFB_LIMIT;
    uint64_t total_bs = 0;
    unsigned long long best = ~0ULL;
    int c = K;
    for (c = K + 1; rc == VFB_OK && c <= bs_max; ++c) {
      // candidates of size c, in 128 bits against overflow
      unsigned __int128 cands = D.cn[c - 1];
      for (int a = 1; 2 * a <= c - 1; ++a) cands += 2 * (unsigned __int128)D.cn[a] * D.cn[c - 1 - a];
      if (cands >= ((unsigned __int128)1 << 40)) { rc = VFB_LIMIT; break; }
      const uint64_t nc = (uint64_t)cands;
      // room: entries, table (at most half full), bitmap
      if (nent + nc > ent_cap) {
        const uint64_t want = nent + nc + 1024;
        size_t g1 = 0, g2 = 0;
        void* nv = dalloc(want * 8, &g1);
        void* no = nv ? dalloc(want * 8, &g2) : nullptr;
        if (!nv || !no) { dfree(nv); rc = VFB_OOM; break; }
        cudaMemcpyAsync(nv, D.vals, nent * 8, cudaMemcpyDeviceToDevice, stream);
        cudaMemcpyAsync(no, D.org, nent * 8, cudaMemcpyDeviceToDevice, stream);
        for (void*& p : held) {
          if (p == D.vals) { dfree(p); p = nv; }
          else if (p == D.org) { dfree(p); p = no; }
        }
        D.vals = (uint64_t*)nv;
        D.org = (uint64_t*)no;
        ent_cap = want;
      }
      if (2 * (nent + nc) > slots) {
        const uint64_t ns = pow2_at_least(4 * (nent + nc));
        size_t g1 = 0;
        void* pt = dalloc(ns * sizeof(Slot), &g1);
        if (!pt) { rc = VFB_OOM; break; }
        cudaMemsetAsync(pt, 0xFF, ns * sizeof(Slot), stream);
        cudaMemsetAsync(D.fail, 0, 8, stream);
        k_rehash<<<grid, 256, 0, stream>>>(D.tab, slots, (Slot*)pt, ns - 1, D.fail);
        ++c_launch;
        for (void*& p : held)
          if (p == D.tab) { dfree(p); p = pt; }
        D.tab = (Slot*)pt;
        slots = ns;
        D.mask = ns - 1;
      }
      const uint64_t nw = (nc + 31) / 32 + 1;
      if (nw > words_cap) {
        size_t g1 = 0, g2 = 0, g3 = 0;
        void* pb = dalloc(nw * 4, &g1);
        const uint64_t ncap = (nw + kBsChunkWords - 1) / kBsChunkWords + 1;
        void* pc = pb ? dalloc(ncap * 8, &g2) : nullptr;
        void* po = pc ? dalloc(ncap * 8, &g3) : nullptr;
        if (!pb || !pc || !po) { dfree(pb); dfree(pc); rc = VFB_OOM; break; }
        cudaMemsetAsync(pb, 0, nw * 4, stream);
        for (void*& p : held) {
          if (p == D.bitmap) { dfree(p); p = pb; }
          else if (p == D.counts) { dfree(p); p = pc; }
          else if (p == D.offs) { dfree(p); p = po; }
        }
        D.bitmap = (uint32_t*)pb;
        D.counts = (unsigned long long*)pc;
        D.offs = (unsigned long long*)po;
        words_cap = nw;
        chunk_cap = ncap;
      }
      cudaMemsetAsync(D.best, 0xFF, 8, stream);
      k_bs_level<<<g256, 256, 0, stream>>>(D, c, (unsigned long long)nc);
      ++c_launch;
      cudaMemcpyAsync(&best, D.best, 8, cudaMemcpyDeviceToHost, stream);
      cudaMemcpyAsync(&fails, D.fail, 8, cudaMemcpyDeviceToHost, stream);
      if (cudaStreamSynchronize(stream) != cudaSuccess) { rc = dev_fail(__LINE__); break; }
      if (fails) { rc = VFB_LIMIT; break; }
      // new entries: the owners (below the solving candidate, if any)
      const uint64_t lim = best != ~0ULL ? best : nc;
      k_bs_mark<<<g256, 256, 0, stream>>>(D, c, (unsigned long long)slots, (unsigned long long)lim);
      ++c_launch;
      uint64_t nnew = 0;
      rc = compact(c, lim, nent, nnew);
      if (rc != VFB_OK) break;
      D.st[c] = nent;
      D.cn[c] = nnew;
      nent += nnew;
      r.level_rows[c] = nnew + (best != ~0ULL ? 1 : 0);
      r.level_cands[c] = best != ~0ULL ? best + 1 : nc;
      r.size = c;
      total_bs += r.level_rows[c];
      if (best != ~0ULL) break;
    }
    if (rc == VFB_OK && best != ~0ULL) {
      // the formula: the solving candidate's tree over BS entries; its leaves
      // are cache rows, rebuilt on the device
      const int cs = r.size;
      std::vector<uint64_t> orgs;
      auto org_of = [&](uint64_t e) -> uint64_t {
        uint64_t v = 0;
        cudaMemcpy(&v, D.org + e, 8, cudaMemcpyDeviceToHost);
        return v;
      };
      auto size_of = [&](uint64_t e) -> int {
        for (int k = 1; k < cs; ++k)
          if (e >= D.st[k] && e < D.st[k] + D.cn[k]) return k;
        return -1;
      };
      struct Node { int op; int leaf; uint64_t a, b; };
      std::vector<unsigned long long> leaves;
      std::vector<int16_t> tokens;   // >= 0: leaf index + 1000; < 0: operator
      std::function<bool(int, uint64_t, bool)> walk = [&](int k, uint64_t key, bool is_cand) -> bool {
        // key: candidate index at size k (is_cand) or an entry index
        uint64_t g = key;
        if (!is_cand) {
          k = size_of(key);
          if (k < 0) return false;
          g = org_of(key);
          if (k <= K) {
            leaves.push_back(g);   // g: cache row
            tokens.push_back((int16_t)(1000 + leaves.size() - 1));
            return true;
          }
        }
        const BsCand cd = bs_decode(D.st, D.cn, k, g);
        if (cd.op < 0) return false;
        if (!walk(0, cd.a, false)) return false;
        if (cd.op != OP_NOT && !walk(0, cd.b, false)) return false;
        tokens.push_back((int16_t)(-(1 + cd.op)));
        return true;
      };
      if (!walk(cs, best, true) || leaves.size() > (size_t)kMaxSize) {
        rc = dev_fail(__LINE__);
      } else {
        const int nl = (int)leaves.size();
        unsigned long long* dl = (unsigned long long*)take(nl * 8);
        int16_t* drpn = (int16_t*)take((size_t)nl * kMaxSize * 2);
        int* dlen = (int*)take(nl * 4);
        if (!dl || !drpn || !dlen) {
          rc = VFB_OOM;
        } else {
          cudaMemcpyAsync(dl, leaves.data(), nl * 8, cudaMemcpyHostToDevice, stream);
          k_bs_leaves<<<1, 32, 0, stream>>>(dInst + i, dl, nl, drpn, dlen);
          ++c_launch;
          std::vector<int16_t> lr((size_t)nl * kMaxSize);
          std::vector<int> ll(nl);
          cudaMemcpyAsync(lr.data(), drpn, lr.size() * 2, cudaMemcpyDeviceToHost, stream);
          cudaMemcpyAsync(ll.data(), dlen, nl * 4, cudaMemcpyDeviceToHost, stream);
          if (cudaStreamSynchronize(stream) != cudaSuccess) rc = dev_fail(__LINE__);
          int n = 0;
          for (int16_t tk : tokens) {
            if (rc != VFB_OK) break;
            if (tk >= 1000) {
              const int li = tk - 1000;
              if (ll[li] <= 0 || n + ll[li] > kMaxSize) { rc = dev_fail(__LINE__); break; }
              for (int j = 0; j < ll[li]; ++j) r.rpn[n++] = lr[(size_t)li * kMaxSize + j];
            } else {
              if (n >= kMaxSize) { rc = dev_fail(__LINE__); break; }
              r.rpn[n++] = tk;
            }
          }
          if (rc == VFB_OK && n == cs) {
            r.rpn_len = n;
            r.solution_index = best;
            r.status = VFB_OK;
          } else if (rc == VFB_OK) {
            rc = dev_fail(__LINE__);
          }
        }
      }
    } else if (rc == VFB_OK) {
      r.status = VFB_NOT_FOUND;
    }
    r.total_rows += total_bs;
    release();
    return rc;
  }

  // ============================================================ cache-free search
  // Formula numbers of each size in order (ltl_nocache.cu:319-446), one launch
  // per range of kExhRange numbers; the first range with a solution gives the
  // first solution of the numbering.  Sizes whose count passes 2^62 end the
  // search with VFB_LIMIT.
  static constexpr unsigned long long kExhRange = 1ull << 28;

  static void exh_decode_host(uint64_t n, int k, const uint64_t (*cnt)[8], int16_t* rpn) {
    if (k == 1) { rpn[0] = (int16_t)n; return; }
    int op = 0;
    while (op < OP_U && n >= cnt[k][op]) n -= cnt[k][op++];
    rpn[k - 1] = (int16_t)(-(1 + op));
    const int sub = k - 1;
    if (op == OP_NOT || op == OP_X || op == OP_F || op == OP_G) {
      exh_decode_host(n, sub, cnt, rpn);
      return;
    }
    int left = 1;
    while (left < sub - 1 && n >= cnt[left][7] * cnt[sub - left][7]) {
      n -= cnt[left][7] * cnt[sub - left][7];
      ++left;
    }
    const uint64_t nr = cnt[sub - left][7];
    exh_decode_host(n / nr, left, cnt, rpn);
    exh_decode_host(n % nr, sub - left, cnt, rpn + left);
  }

  vfb_status exhaustive(const vfb_instance& in, vfb_result& r) {
    const auto t0 = std::chrono::steady_clock::now();
    std::memset(&r, 0, sizeof(r));
    c_h2d = c_d2h = c_launch = 0;
    if (cudaSetDevice(device) != cudaSuccess) return r.status = dev_fail(__LINE__);
    const int T = in.num_traces, A = in.num_vars, K = in.max_size;
    if (T < 1 || T > kMaxTraces || A < 1 || A > VFB_MAX_VARS || in.num_pos < 0 || in.num_pos > T ||
        K < 1 || K > kMaxSize)
      return r.status = VFB_LIMIT;
    if (!in.words || !in.lengths) return r.status = VFB_BAD_INPUT;
    std::vector<ExhDev> hv(1);
    ExhDev& h = hv[0];
    std::memset(&h, 0, sizeof(h));
    h.A = A;
    h.T = T;
    for (int t = 0; t < T; ++t) {
      if (in.lengths[t] < 1 || in.lengths[t] > VFB_MAX_LENGTH) return r.status = VFB_LIMIT;
      h.len[t] = (uint8_t)in.lengths[t];
      if (t < in.num_pos) h.posmask[t >> 6] |= 1ULL << (t & 63);
      const uint64_t m = in.lengths[t] >= 64 ? ~0ULL : ((1ULL << in.lengths[t]) - 1);
      for (int v = 0; v < A; ++v) h.words[(size_t)t * A + v] = in.words[(size_t)t * A + v] & m;
    }
    // count matrix (generateMatrix ltl_nocache.cu:248-287) in 128 bits; the
    // search stops before the first size that does not fit 62 bits
    typedef unsigned __int128 u128;
    u128 c[kMaxSize + 1][8];
    std::memset(c, 0, sizeof(c));
    c[1][7] = (u128)A;
    if (K >= 2) { c[2][0] = c[2][3] = c[2][4] = c[2][5] = (u128)A; c[2][7] = 4 * (u128)A; }
    for (int i = 3; i <= K; ++i) {
      u128 un = c[i - 1][7], com = 0, ncom = 0;
      for (int j = 1; j <= (i - 1) / 2; ++j) com += c[j][7] * c[i - j - 1][7];
      for (int j = 1; j <= i - 2; ++j) ncom += c[j][7] * c[i - j - 1][7];
      c[i][0] = c[i][3] = c[i][4] = c[i][5] = un;
      c[i][1] = c[i][2] = com;
      c[i][6] = ncom;
      c[i][7] = 4 * un + 2 * com + ncom;
    }
    int kfit = 0;
    for (int i = 1; i <= K; ++i) {
      if (c[i][7] >= ((u128)1 << 62)) break;
      kfit = i;
    }
    for (int i = 1; i <= kfit; ++i)
      for (int o = 0; o < 8; ++o) h.cnt[i][o] = (uint64_t)c[i][o];
    size_t g1 = 0, g2 = 0;
    void* pd = dalloc(sizeof(ExhDev), &g1);
    void* pb = pd ? dalloc(sizeof(unsigned long long), &g2) : nullptr;
    if (!pd || !pb) { dfree(pd); return r.status = VFB_OOM; }
    ExhDev* dP = (ExhDev*)pd;
    unsigned long long* dBest = (unsigned long long*)pb;
    cudaEventRecord(ev_t0, stream);
    vfb_status rc = VFB_OK;
    if (cudaMemcpyAsync(dP, &h, sizeof(ExhDev), cudaMemcpyHostToDevice, stream) != cudaSuccess ||
        cudaMemsetAsync(dBest, 0xFF, sizeof(unsigned long long), stream) != cudaSuccess)
      rc = dev_fail(__LINE__);
    c_h2d += sizeof(ExhDev);
    unsigned long long best = ~0ULL;
    int found_k = 0;
    for (int k = 1; k <= kfit && rc == VFB_OK && !found_k; ++k) {
      const unsigned long long total = h.cnt[k][7];
      for (unsigned long long lo = 0; lo < total; lo += kExhRange) {
        const unsigned long long hi = std::min(total, lo + kExhRange);
        const unsigned long long nthreads = hi - lo;
        const unsigned blocks = (unsigned)std::min<unsigned long long>((nthreads + 255) / 256,
                                                                       (unsigned long long)sms * 16);
        k_exhaustive<<<blocks, 256, 0, stream>>>(dP, k, lo, hi, dBest);
        ++c_launch;
        if (cudaMemcpyAsync(&best, dBest, sizeof(best), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
            cudaStreamSynchronize(stream) != cudaSuccess) {
          rc = dev_fail(__LINE__);
          break;
        }
        c_d2h += sizeof(best);
        if (best != ~0ULL) {
          r.level_cands[k] = best + 1;
          found_k = k;
          break;
        }
        r.level_cands[k] = hi;
      }
      r.size = k;
    }
    cudaEventRecord(ev_t1, stream);
    cudaStreamSynchronize(stream);
    float ms = 0;
    cudaEventElapsedTime(&ms, ev_t0, ev_t1);
    dfree(pd);
    dfree(pb);
    if (rc != VFB_OK) return r.status = rc;
    r.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    r.device_seconds = ms * 1e-3;
    r.h2d_bytes = c_h2d;
    r.d2h_bytes = c_d2h;
    r.kernel_launches = c_launch;
    if (found_k) {
      exh_decode_host(best, found_k, h.cnt, r.rpn);
      r.rpn_len = found_k;
      r.solution_index = best;
      r.size = found_k;
      return r.status = VFB_OK;
    }
    return r.status = (kfit < K) ? VFB_LIMIT : VFB_NOT_FOUND;
  }

  // ------------------------------------------------------------ autotuner
  vfb_status tune_set(const vfb_tune* t) {
    if (!t) {
      tune = vfb_tune{};
      return VFB_OK;
    }
    for (int b = 0; b < kTuneBands; ++b) {
      const int r = t->rows[b];
      if (r > 32 || (r & (r - 1)) != 0) return VFB_BAD_INPUT;   // (above kTQ acts as kTQ)
      if (t->tiles_log2[b] > 40) return VFB_BAD_INPUT;
    }
    tune = *t;
    return VFB_OK;
  }

  static bool same_result(const vfb_result& a, const vfb_result& b) {
    if (a.status != b.status || a.size != b.size || a.rpn_len != b.rpn_len ||
        a.solution_index != b.solution_index || a.total_rows != b.total_rows)
      return false;
    for (int i = 0; i < a.rpn_len && i < VFB_MAX_SIZE; ++i)
      if (a.rpn[i] != b.rpn[i]) return false;
    for (int k = 0; k <= VFB_MAX_SIZE; ++k)
      if (a.level_rows[k] != b.level_rows[k] || a.level_cands[k] != b.level_cands[k]) return false;
    return true;
  }

  // Solves the sample under each candidate shape with every kernel of the
  // level step timed; per band, the shape with the least k_p1 time wins.
  vfb_status autotune(const vfb_instance* sample, int n, int reps, vfb_tune* out) {
    if (!sample || n <= 0 || reps < 1) return VFB_BAD_INPUT;
    struct Shape { uint8_t rows, tiles; uint16_t blocks; };
    std::vector<Shape> shapes;
    for (int r : {2, 4, 8, 16})
      for (int t : {8, 10, 12, 14})
        for (int b : {0, sms}) shapes.push_back(Shape{(uint8_t)r, (uint8_t)t, (uint16_t)b});
    const int sv_profile = profile;
    const bool sv_loop = use_loop, sv_coop = use_coop, sv_cluster = use_cluster;
    Prof sv_prof[KP_N];
    std::memcpy(sv_prof, prof, sizeof(prof));
    profile = 1;
    use_loop = use_coop = use_cluster = false;
    if (exec) { cudaGraphExecDestroy(exec); exec = nullptr; }
    tune = vfb_tune{};
    vfb_status rc = VFB_OK;
    // reference results (and buffers at their final sizes) under the built-in shape
    std::vector<vfb_result> want(n);
    for (int i = 0; i < n && rc == VFB_OK; ++i) {
      const vfb_status s = batch(&sample[i], 1, &want[i]);
      if (s != VFB_OK) rc = s;
    }
    const size_t ns = shapes.size();
    std::vector<double> best(ns * kTuneBands, 0.0);
    std::vector<uint32_t> lv(ns * kTuneBands, 0);
    for (size_t c = 0; c < ns && rc == VFB_OK; ++c) {
      for (int b = 0; b < kTuneBands; ++b) {
        tune.rows[b] = shapes[c].rows;
        tune.tiles_log2[b] = shapes[c].tiles;
        tune.blocks[b] = shapes[c].blocks;
      }
      for (int r = 0; r < reps && rc == VFB_OK; ++r) {
        double acc[kTuneBands] = {};
        uint32_t lev[kTuneBands] = {};
        tune_ms = acc;
        tune_levels = lev;
        for (int i = 0; i < n && rc == VFB_OK; ++i) {
          vfb_result got;
          const vfb_status s = batch(&sample[i], 1, &got);
          if (s != VFB_OK) rc = s;
          else if (!same_result(got, want[i])) rc = dev_fail(__LINE__);
        }
        tune_ms = nullptr;
        tune_levels = nullptr;
        for (int b = 0; b < kTuneBands; ++b) {
          double& m = best[c * kTuneBands + b];
          if (r == 0 || acc[b] < m) m = acc[b];
          lv[c * kTuneBands + b] = lev[b];
        }
      }
    }
    vfb_tune res{};
    if (rc == VFB_OK) {
      size_t dflt = 0;
      for (size_t c = 0; c < ns; ++c)
        if (shapes[c].rows == kTQDefault && (1 << shapes[c].tiles) == kP1TileTarget && shapes[c].blocks == 0)
          dflt = c;
      for (int b = 0; b < kTuneBands; ++b) {
        if (lv[dflt * kTuneBands + b] == 0) continue;
        size_t w = dflt;
        for (size_t c = 0; c < ns; ++c)
          if (best[c * kTuneBands + b] < best[w * kTuneBands + b]) w = c;
        if (w != dflt) {
          res.rows[b] = shapes[w].rows;
          res.tiles_log2[b] = shapes[w].tiles;
          res.blocks[b] = shapes[w].blocks;
        }
        res.ms[b] = (float)best[w * kTuneBands + b];
        res.ms_default[b] = (float)best[dflt * kTuneBands + b];
        res.levels[b] = lv[dflt * kTuneBands + b];
      }
    }
    profile = sv_profile;
    use_loop = sv_loop;
    use_coop = sv_coop;
    use_cluster = sv_cluster;
    std::memcpy(prof, sv_prof, sizeof(prof));
    if (exec) { cudaGraphExecDestroy(exec); exec = nullptr; }
    tune = rc == VFB_OK ? res : vfb_tune{};
    if (out && rc == VFB_OK) *out = res;
    return rc;
  }

  int profile_read(vfb_kernel_stat* outp, int cap) {
    int m = 0;
    for (int k = 0; k < KP_N && m < cap; ++k) {
      if (!prof[k].launches) continue;
      vfb_kernel_stat& s = outp[m++];
      std::memset(&s, 0, sizeof(s));
      std::snprintf(s.name, sizeof(s.name), "%s", kNames[k]);
      s.launches = prof[k].launches;
      s.ms = prof[k].ms;
      s.bytes = prof[k].bytes;
    }
    return m;
  }
};

}  // namespace vfb

// =================================================================== C ABI
using vfb::Engine;

extern "C" {

const char* vfb_status_str(vfb_status s) {
  switch (s) {
    case VFB_OK: return "ok";
    case VFB_NOT_FOUND: return "not found";
    case VFB_LIMIT: return "outside supported limits";
    case VFB_OOM: return "device memory budget exhausted";
    case VFB_DEVICE_ERROR: return "device error";
    case VFB_TIMEOUT: return "timeout";
    case VFB_BAD_INPUT: return "bad input";
  }
  return "unknown";
}

vfb_status vfb_create(void** ctx, const vfb_opts* opts) {
  if (!ctx) return VFB_BAD_INPUT;
  *ctx = nullptr;
  Engine* e = new (std::nothrow) Engine();
  if (!e) return VFB_OOM;
  const vfb_status s = e->init(opts);
  if (s != VFB_OK) {
    delete e;
    return s;
  }
  *ctx = e;
  return VFB_OK;
}

void vfb_destroy(void* ctx) { delete static_cast<Engine*>(ctx); }

vfb_status vfb_solve(void* ctx, const vfb_instance* inst, vfb_result* out) {
  if (!ctx || !inst || !out) return VFB_BAD_INPUT;
  const vfb_status rc = static_cast<Engine*>(ctx)->batch(inst, 1, out);
  return rc != VFB_OK ? rc : out->status;
}

vfb_status vfb_solve_costs(void* ctx, const vfb_instance* inst, const int* costs, int neg_type, vfb_result* out) {
  if (!ctx || !inst || !out || !costs) return VFB_BAD_INPUT;
  if (neg_type != 1 && neg_type != 2) return VFB_BAD_INPUT;
  for (int c = 0; c < 8; ++c)
    if (costs[c] < 1 || costs[c] > VFB_MAX_SIZE) return VFB_BAD_INPUT;
  Engine* e = static_cast<Engine*>(ctx);
  for (int c = 0; c < 8; ++c) e->req_cost[c] = costs[c];
  e->req_neg = neg_type;
  const vfb_status rc = e->batch(inst, 1, out);
  for (int c = 0; c < 8; ++c) e->req_cost[c] = 1;
  e->req_neg = 1;
  return rc != VFB_OK ? rc : out->status;
}

vfb_status vfb_solve_bs(void* ctx, const vfb_instance* inst, int bs_max_size, vfb_result* out) {
  if (!ctx || !inst || !out) return VFB_BAD_INPUT;
  if (bs_max_size < 1 || bs_max_size > VFB_MAX_SIZE) return VFB_BAD_INPUT;
  Engine* e = static_cast<Engine*>(ctx);
  e->bs_max = bs_max_size;
  const vfb_status rc = e->batch(inst, 1, out);
  e->bs_max = 0;
  return rc != VFB_OK ? rc : out->status;
}

vfb_status vfb_solve_exhaustive(void* ctx, const vfb_instance* inst, vfb_result* out) {
  if (!ctx || !inst || !out) return VFB_BAD_INPUT;
  return static_cast<Engine*>(ctx)->exhaustive(*inst, *out);
}

vfb_status vfb_batch_solve(void* ctx, const vfb_instance* inst, int n, vfb_result* out) {
  if (!ctx || (n > 0 && (!inst || !out)) || n < 0) return VFB_BAD_INPUT;
  return static_cast<Engine*>(ctx)->batch(inst, n, out);
}

vfb_status vfb_serve_open(void* ctx, int slots, int max_traces) {
  if (!ctx) return VFB_BAD_INPUT;
  return static_cast<Engine*>(ctx)->serve_open(slots, max_traces);
}

vfb_status vfb_serve_limits(void* ctx, double budget_frac, uint64_t request_bytes, uint64_t step_candidates) {
  if (!ctx) return VFB_BAD_INPUT;
  return static_cast<Engine*>(ctx)->serve_limits(budget_frac, request_bytes, step_candidates);
}

vfb_status vfb_serve_submit(void* ctx, const vfb_instance* inst, uint64_t tag) {
  if (!ctx) return VFB_BAD_INPUT;
  return static_cast<Engine*>(ctx)->serve_submit(inst, tag);
}

vfb_status vfb_serve_step(void* ctx, vfb_served* done, int cap, int* ndone, int* active, int* queued) {
  if (!ctx || !done || !ndone || cap <= 0) return VFB_BAD_INPUT;
  return static_cast<Engine*>(ctx)->serve_step(done, cap, ndone, active, queued);
}

void vfb_serve_close(void* ctx) {
  if (ctx) static_cast<Engine*>(ctx)->serve_close();
}

vfb_status vfb_tune_set(void* ctx, const vfb_tune* tune) {
  if (!ctx) return VFB_BAD_INPUT;
  return static_cast<Engine*>(ctx)->tune_set(tune);
}

vfb_status vfb_tune_get(void* ctx, vfb_tune* tune) {
  if (!ctx || !tune) return VFB_BAD_INPUT;
  *tune = static_cast<Engine*>(ctx)->tune;
  return VFB_OK;
}

vfb_status vfb_autotune(void* ctx, const vfb_instance* sample, int n, int reps, vfb_tune* out) {
  if (!ctx) return VFB_BAD_INPUT;
  return static_cast<Engine*>(ctx)->autotune(sample, n, reps, out);
}

int vfb_profile_read(void* ctx, vfb_kernel_stat* out, int cap) {
  if (!ctx || !out || cap <= 0) return 0;
  return static_cast<Engine*>(ctx)->profile_read(out, cap);
}

void vfb_profile_reset(void* ctx) {
  if (!ctx) return;
  Engine* e = static_cast<Engine*>(ctx);
  for (auto& p : e->prof) p = vfb::Prof{};
}

}  // extern "C"
