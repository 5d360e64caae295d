// vfb_noalloc.cu -- vfb_solve_noalloc: a solve that allocates nothing.
//
// For callers that must not allocate device memory while they run: code that
// executes while another component owns the device heap through its own
// allocator (a serving process that reserved all memory up front, a
// framework whose pool must not be bypassed), latency-critical loops that
// cannot afford the implicit synchronisation of cudaMalloc/cudaFree, and
// environments where the driver heap is closed after start-up.  vfb_solve
// cannot serve them: its context allocates a stream, events, pinned staging
// and growing device buffers.
//
// This entry point runs the same level-step kernels as vfb_solve, but every
// device buffer they use -- the per-instance record, the level cache, the
// hash set, the owner bitmap, the owner list and the batch
// workspace -- is carved out of one file-scope static device array of
// kScratchBytes.  Buffers never grow: a search that needs more room than the
// array provides stops with VFB_OOM and a message on stderr.  Nothing is
// allocated on the host either (uploads and read-backs use the caller's
// memory and the legacy default stream).
//
// The array belongs to the module: every GPU that loads the library holds it
// until the process exits.  All calls share it and it keeps the last call's
// contents, so each call clears what must start empty (hash set, bitmap,
// counters).  Calls that overlap on the GPU (from several host threads, or
// with other work on the default stream of the same device) race on the
// array; serialise them.  The first call on a device resolves the array's
// device address (cudaGetSymbolAddress with that device current) and sets the
// P1 kernel's shared-memory limit; make that first call before any stream
// capture begins.  The address is remembered with the CUDA context it was
// resolved in: after a device reset (a new primary context) the next call
// resolves it again, so it never writes through an address of a context that
// is gone.
//
// Capacity: besides the fixed parts (hash set of 2^19 slots, 16 MiB; bitmap
// of 2^25 candidates, 4 MiB; owner list of 2^19 entries, 4 MiB), about 40 MiB
// of level cache: rows = that space / (8 * TP + 8) bytes, TP = traces rounded
// up to even (about 127,000 characteristic sets at 40 traces, 40,000 at 128),
// and at most about 2^18 distinct keys (the hash set is planned at most half
// full, counting the next level's projected keys).
#include <cstdio>
#include <cstring>
#include <mutex>

#include "vfb_kernels.cuh"
#include "../../include/vfb.h"

namespace vfb {
namespace {

constexpr size_t kScratchBytes = 64ull << 20;   // VFB_NOALLOC_SCRATCH_BYTES in vfb.h
constexpr uint64_t kNaSlots = 1ull << 19;        // hash-set slots (16 MiB)
constexpr uint64_t kNaWords = 1ull << 20;        // candidate-bitmap words (32 Mi candidates)
constexpr uint64_t kNaTents = 1ull << 19;        // owner-list entries

__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
unsigned char* g_base[kMaxDevices] = {};
void* g_base_ctx[kMaxDevices] = {};   // context each address was resolved in
std::mutex g_mu;

// The driver's cuCtxGetCurrent, looked up through the runtime so that the
// library does not link the driver library itself.  nullptr if unavailable.
using CtxGetCurrentFn = int (*)(void**);
CtxGetCurrentFn ctx_get_current() {
  static const CtxGetCurrentFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return static_cast<CtxGetCurrentFn>(nullptr);
    }
    return reinterpret_cast<CtxGetCurrentFn>(p);
  }();
  return fn;
}

void* current_context() {
  void* c = nullptr;
  const CtxGetCurrentFn fn = ctx_get_current();
  if (fn && fn(&c) != 0) c = nullptr;
  return c;
}

// Device address of g_scratch for device `dev` (current).  The host-side
// symbol is only a stand-in and must never be passed to a kernel.  Resolved
// on the first call on a device and again whenever the current context is not
// the one it was resolved in (the device was reset since).
vfb_status scratch_base(int dev, unsigned char** out) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (dev < 0 || dev >= kMaxDevices) return VFB_DEVICE_ERROR;
  void* ctx = g_base[dev] ? current_context() : nullptr;
  if (!g_base[dev] || ctx != g_base_ctx[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      g_base[dev] = nullptr;
      return VFB_DEVICE_ERROR;
    }
    const int smem = (kTS * (kMaxTraces + 1) + kTQ * kMaxTraces) * 8;
    if (cudaFuncSetAttribute(k_p1, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess) {
      cudaGetLastError();
      g_base[dev] = nullptr;
      return VFB_DEVICE_ERROR;
    }
    g_base[dev] = static_cast<unsigned char*>(p);
    g_base_ctx[dev] = current_context();   // (the lookup above made the context current)
  }
  *out = g_base[dev];
  return VFB_OK;
}

// Proposition rows from the caller's trace-major words (words[t*A + v] ->
// rows[v*TP + t], zero in the padding column).
__global__ void k_na_rows(const uint64_t* __restrict__ words, int T, int A, int TP, uint64_t* __restrict__ rows) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A * TP; i += gridDim.x * blockDim.x) {
    const int v = i / TP, t = i - v * TP;
    rows[i] = t < T ? words[(size_t)t * A + v] : 0ULL;
  }
}

struct Carver {
  unsigned char* base;
  size_t off = 0;
  template <typename T>
  T* take(size_t count) {
    off = (off + 255) & ~size_t(255);
    T* p = reinterpret_cast<T*>(base + off);
    off += count * sizeof(T);
    return p;
  }
};

// Problem fields of the instance record (same rules as the engine's set-up:
// key layout of LTL_BS.cu:30-110).
vfb_status fill_problem(const vfb_instance& in, InstDev& d) {
  std::memset(&d, 0, sizeof(d));
  d.mask_off = 1;   // no level re-runs here: P1 never skips operators
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
  d.npos = in.num_pos;
  d.max_size = in.max_size;
  d.lensum = S;
  d.stride1 = 1;
  for (int i = 0; i < T; ++i) {
    d.len[i] = (uint8_t)in.lengths[i];
    if (i < in.num_pos) d.posmask[i >> 6] |= 1ULL << (i & 63);
  }
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
      d.width[i] = (uint8_t)(width[i] < 126 - off ? width[i] : 126 - off);
    }
    off += width[i];
  }
  d.status = ST_RUNNING;
  d.level = 1;
  d.promote_above = ~0ULL;   // no cluster pass here: never hand the instance on
  return VFB_OK;
}

const char* need_text(int need) {
  if (need & NEED_ROWS) return "level cache";
  if (need & NEED_TABLE) return "hash set";
  if (need & NEED_BITMAP) return "candidate bitmap";
  if (need & NEED_LIST) return "owner list";
  return "index range";
}

}  // namespace
}  // namespace vfb

using namespace vfb;

extern "C" vfb_status vfb_solve_noalloc(const vfb_instance* inst, vfb_result* out) {
  if (!inst || !out) return VFB_BAD_INPUT;
  std::memset(out, 0, sizeof(*out));
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return out->status = VFB_DEVICE_ERROR;
  unsigned char* base = nullptr;
  vfb_status s = scratch_base(dev, &base);
  if (s != VFB_OK) return out->status = s;
  InstDev d;
  s = fill_problem(*inst, d);
  if (s != VFB_OK) return out->status = s;

  // carve the static array
  Carver cv{base};
  BatchDev* dB = cv.take<BatchDev>(1);
  InstDev* dI = cv.take<InstDev>(1);
  BatchDev hB{};
  hB.inst = dI;
  hB.ninst = 1;
  hB.p1_prefix = cv.take<unsigned long long>(2);
  hB.chunk_prefix = cv.take<unsigned long long>(2);
  hB.tscan_prefix = cv.take<unsigned long long>(2);
  hB.win_prefix = cv.take<unsigned long long>(2);
  hB.tickets = cv.take<unsigned long long>(kTickets);
  hB.status_out = cv.take<int2>(1);
  hB.loop_iter = cv.take<unsigned long long>(1);
  hB.chunk_cap = kNaWords / kChunkWords + 2;
  hB.chunk_cnt = cv.take<unsigned int>(hB.chunk_cap);
  hB.chunk_base = cv.take<unsigned long long>(hB.chunk_cap);
  d.table = cv.take<Slot>(kNaSlots);
  d.table_mask = kNaSlots - 1;
  d.bitmap = cv.take<uint32_t>(kNaWords);
  d.bitmap_words = kNaWords;
  d.wins = cv.take<uint64_t>(kNaTents);
  d.tent_cap = kNaTents;
  uint64_t* stage = cv.take<uint64_t>((size_t)d.T * d.A);   // the caller's words, as given
  const size_t used = ((cv.off + 255) & ~size_t(255)) + 512;   // + alignment of the last two carves
  const size_t per_row = (size_t)d.TP * 8 + 8;                  // row words + origin index
  if (used >= kScratchBytes || (kScratchBytes - used) / per_row < (size_t)d.A) {
    std::fprintf(stderr, "vfb_solve_noalloc: %d propositions x %d traces do not fit the %zu-byte static scratch\n",
                 d.A, d.T, kScratchBytes);
    return out->status = VFB_OOM;
  }
  const uint64_t rows = (kScratchBytes - used) / per_row;
  d.origin = cv.take<uint64_t>(rows);
  d.rows = cv.take<uint64_t>(rows * d.TP);
  d.row_cap = rows;

  // reset what must start empty, upload the instance
  uint64_t h2d = 0, d2h = 0, launches = 0;
  cudaStream_t st = 0;
  bool ok = cudaMemsetAsync(d.table, 0xFF, kNaSlots * sizeof(Slot), st) == cudaSuccess &&
            cudaMemsetAsync(d.bitmap, 0, kNaWords * 4, st) == cudaSuccess;
  // one copy of the words, turned into proposition rows on the device
  ok = ok && cudaMemcpy(stage, inst->words, (size_t)d.T * d.A * 8, cudaMemcpyHostToDevice) == cudaSuccess;
  h2d += (uint64_t)d.T * d.A * 8;
  if (ok) {
    k_na_rows<<<(d.A * d.TP + 255) / 256, 256, 0, st>>>(stage, d.T, d.A, d.TP, d.rows);
    ++launches;
    ok = cudaGetLastError() == cudaSuccess;
  }
  ok = ok && cudaMemcpy(dI, &d, sizeof(InstDev), cudaMemcpyHostToDevice) == cudaSuccess &&
       cudaMemcpy(dB, &hB, sizeof(BatchDev), cudaMemcpyHostToDevice) == cudaSuccess;
  h2d += sizeof(InstDev) + sizeof(BatchDev);
  if (!ok) return out->status = VFB_DEVICE_ERROR;

  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int g = sms * 8, gc = sms * 2;
  const int p1_smem = (kTS * (d.TP + 1) + kTQ * d.TP) * 8;
  int occ = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_p1, kTS, p1_smem);
  const int p1_grid = sms * (occ > 0 ? occ : 1);

  k_init<<<1, 256, 0, st>>>(dB);
  ++launches;
  int2 status{ST_RUNNING, 0};
  for (int step = 0; step <= kMaxSize + 1; ++step) {
    if (cudaMemcpy(&status, hB.status_out, sizeof(int2), cudaMemcpyDeviceToHost) != cudaSuccess)
      return out->status = VFB_DEVICE_ERROR;
    d2h += sizeof(int2);
    if (status.x != ST_RUNNING) break;
    k_plan<<<1, 1024, 0, st>>>(dB);
    k_p1<<<p1_grid, kTS, p1_smem, st>>>(dB);
    k_table_scan<<<g, 256, 0, st>>>(dB);
    k_chunk_count<<<gc, 256, 0, st>>>(dB);
    k_chunk_scan<<<1, kScanThreads, 0, st>>>(dB);
    k_chunk_emit<<<gc, kChunkThreads, 0, st>>>(dB);
    k_emit_rows<<<g, 256, 0, st>>>(dB);
    k_finish<<<1, 256, 0, st>>>(dB);
    launches += 8;
    if (cudaGetLastError() != cudaSuccess) return out->status = VFB_DEVICE_ERROR;
  }
  InstDev r;
  if (cudaMemcpy(&r, dI, sizeof(InstDev), cudaMemcpyDeviceToHost) != cudaSuccess)
    return out->status = VFB_DEVICE_ERROR;
  d2h += sizeof(InstDev);
  out->h2d_bytes = h2d;
  out->d2h_bytes = d2h;
  out->kernel_launches = launches;
  if (r.status == ST_NEED_MEM) {
    std::fprintf(stderr,
                 "vfb_solve_noalloc: size %d needs a larger %s than the %zu-byte static scratch holds; "
                 "use vfb_solve\n",
                 r.level, need_text(r.need), kScratchBytes);
    out->status = VFB_OOM;
  } else if (r.status == ST_FOUND) {
    out->status = VFB_OK;
  } else if (r.status == ST_NOT_FOUND) {
    out->status = VFB_NOT_FOUND;
  } else {
    out->status = VFB_DEVICE_ERROR;
  }
  // sizes completed (a stopped search reports the finished ones only)
  int top = r.res_size;
  if (out->status == VFB_OOM || out->status == VFB_DEVICE_ERROR) top = r.level - 1;
  if (top > kMaxSize) top = kMaxSize;
  out->size = top > 0 ? top : 0;
  uint64_t tot = 0;
  for (int k = 1; k <= top; ++k) {
    out->level_rows[k] = r.lcount[k];
    out->level_cands[k] = r.lcands[k];
    tot += r.lcount[k];
  }
  out->total_rows = tot;
  if (out->status == VFB_OK) {
    out->rpn_len = r.rpn_len;
    for (int j = 0; j < r.rpn_len && j < kMaxSize; ++j) out->rpn[j] = r.rpn[j];
    out->solution_index = r.sol_index;
  }
  return out->status;
}
