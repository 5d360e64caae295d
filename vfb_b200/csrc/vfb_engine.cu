// vfb_engine.cu -- host driver of the cached search: instance set-up, the
// level loop, buffer growth, results.  Implements the C ABI of include/vfb.h.
//
// The reference drives one launch per (level, operator, size split, chunk)
// with a blocking device-to-host copy after each (LTL_BS.cu:1226-1488).  Here
// a whole level of every instance in flight is one fixed launch sequence
// (vfb_kernels.cu), captured once as a CUDA graph; the host only reads a
// per-instance (status, need) word after each level and grows a buffer when
// a kernel asked for more room.  All buffers come from the device's
// stream-ordered memory pool, which keeps freed memory for the next solve.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "vfb_kernels.cuh"
#include "../../include/vfb.h"

namespace vfb {

namespace {

struct InstHost {
  InstDev d;        // host copy of the device record
  size_t bytes = 0; // device bytes held by this instance
  bool active = false;
  vfb_status fail = VFB_OK;
};

uint64_t pow2_at_least(uint64_t x) {
  uint64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

}  // namespace

struct Engine {
  int device = 0;
  int verbose = 0;
  size_t mem_limit = 0;
  cudaStream_t stream = nullptr;
  cudaMemPool_t pool = nullptr;
  int sms = 0;
  int grid = 0;        // grid-stride CTAs (256 threads)
  int p1_grid = 0;     // P1 CTAs
  int p1_smem_max = 0;
  cudaError_t last_error = cudaSuccess;

  // batch workspace
  int ninst_cap = 0;
  BatchDev hB{};
  BatchDev* dB = nullptr;
  InstDev* dInst = nullptr;
  int2* h_status = nullptr;   // pinned mirror of B.status_out
  unsigned long long* d_fail = nullptr;

  // graph of one level step
  cudaGraphExec_t step_exec = nullptr;
  int step_ninst = -1, step_smem = -1, step_grid = -1;

  size_t used_bytes = 0;

  ~Engine() { release(); }

  void release() {
    if (step_exec) cudaGraphExecDestroy(step_exec);
    step_exec = nullptr;
    free_workspace();
    if (h_status) cudaFreeHost(h_status);
    h_status = nullptr;
    if (d_fail) cudaFree(d_fail);
    d_fail = nullptr;
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
  }

  void free_workspace() {
    auto f = [&](void* p) { if (p) cudaFreeAsync(p, stream); };
    f(hB.p1_prefix); f(hB.chunk_prefix0); f(hB.chunk_prefix1); f(hB.tent_prefix); f(hB.win_prefix);
    f(hB.chunk_cnt); f(hB.chunk_base); f(hB.tickets); f(hB.status_out); f(dB); f(dInst);
    hB = BatchDev{};
    dB = nullptr;
    dInst = nullptr;
    ninst_cap = 0;
    if (stream) cudaStreamSynchronize(stream);
  }

  cudaError_t dalloc(void** p, size_t bytes) {
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    if (mem_limit && used_bytes + bytes > mem_limit) return cudaErrorMemoryAllocation;
    cudaError_t e = cudaMallocAsync(p, bytes, stream);
    if (e == cudaSuccess) used_bytes += bytes;
    return e;
  }
  void dfree(void* p, size_t bytes) {
    if (p) {
      cudaFreeAsync(p, stream);
      used_bytes -= std::min(used_bytes, bytes);
    }
  }

  vfb_status init(const vfb_opts* o) {
    device = o ? o->device : 0;
    verbose = o ? o->verbose : 0;
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
    mem_limit = (o && o->mem_limit_bytes) ? o->mem_limit_bytes : (size_t)(0.9 * (double)freeb);
    if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) return VFB_DEVICE_ERROR;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t thr = ~0ULL;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    if (cudaMalloc(&d_fail, sizeof(unsigned long long)) != cudaSuccess) return VFB_DEVICE_ERROR;
    grid = sms * 8;
    p1_smem_max = 0;
    // P1 must be able to hold the largest staged tile (128 traces)
    const int maxsmem = (kTS * (kMaxTraces + 1) + kTQ * kMaxTraces) * 8;
    if (cudaFuncSetAttribute(k_p1, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsmem) != cudaSuccess)
      return VFB_DEVICE_ERROR;
    // a quick launch of a trivial kernel proves the image runs on this device
    if (cudaFuncGetAttributes(&fattr_, k_p1) != cudaSuccess) return VFB_DEVICE_ERROR;
    return VFB_OK;
  }
  cudaFuncAttributes fattr_{};

  // ------------------------------------------------------------ workspace
  vfb_status ensure_workspace(int ninst, uint64_t chunk_need) {
    if (ninst > ninst_cap || chunk_need > hB.chunk_cap) {
      const int nc = std::max(ninst, ninst_cap);
      const uint64_t cc = std::max<uint64_t>(chunk_need, hB.chunk_cap);
      BatchDev nb{};
      void* p = nullptr;
      const size_t pre = (size_t)(nc + 1) * sizeof(unsigned long long);
#define WS_ALLOC(field, bytes)                                            \
  if (cudaMallocAsync(&p, (bytes), stream) != cudaSuccess) return VFB_OOM; \
  nb.field = reinterpret_cast<decltype(nb.field)>(p);
      WS_ALLOC(p1_prefix, pre)
      WS_ALLOC(chunk_prefix0, pre)
      WS_ALLOC(chunk_prefix1, pre)
      WS_ALLOC(tent_prefix, pre)
      WS_ALLOC(win_prefix, pre)
      WS_ALLOC(chunk_cnt, std::max<uint64_t>(cc, 1) * sizeof(unsigned int))
      WS_ALLOC(chunk_base, std::max<uint64_t>(cc, 1) * sizeof(unsigned long long))
      WS_ALLOC(tickets, 4 * sizeof(unsigned long long))
      WS_ALLOC(status_out, (size_t)nc * sizeof(int2))
#undef WS_ALLOC
      BatchDev* ndB = nullptr;
      if (cudaMallocAsync((void**)&ndB, sizeof(BatchDev), stream) != cudaSuccess) return VFB_OOM;
      InstDev* ndI = nullptr;
      if (cudaMallocAsync((void**)&ndI, (size_t)nc * sizeof(InstDev), stream) != cudaSuccess) return VFB_OOM;
      if (dInst && ninst_cap)
        cudaMemcpyAsync(ndI, dInst, (size_t)ninst_cap * sizeof(InstDev), cudaMemcpyDeviceToDevice, stream);
      free_workspace_keep_stream();
      hB = nb;
      hB.chunk_cap = cc;
      dB = ndB;
      dInst = ndI;
      ninst_cap = nc;
      if (h_status) cudaFreeHost(h_status);
      if (cudaMallocHost(&h_status, (size_t)nc * sizeof(int2)) != cudaSuccess) return VFB_OOM;
      if (step_exec) { cudaGraphExecDestroy(step_exec); step_exec = nullptr; }
    }
    hB.inst = dInst;
    hB.ninst = ninst;
    if (cudaMemcpyAsync(dB, &hB, sizeof(BatchDev), cudaMemcpyHostToDevice, stream) != cudaSuccess)
      return VFB_DEVICE_ERROR;
    return VFB_OK;
  }

  void free_workspace_keep_stream() {
    auto f = [&](void* p) { if (p) cudaFreeAsync(p, stream); };
    f(hB.p1_prefix); f(hB.chunk_prefix0); f(hB.chunk_prefix1); f(hB.tent_prefix); f(hB.win_prefix);
    f(hB.chunk_cnt); f(hB.chunk_base); f(hB.tickets); f(hB.status_out); f(dB); f(dInst);
  }

  // --------------------------------------------------------- step launch
  void launch_step(int ninst, int p1_smem) {
    const int g = grid;
    k_plan<<<1, 1024, 0, stream>>>(dB);
    k_p1<<<p1_grid, kTS, p1_smem, stream>>>(dB);
    for (int phase = 0; phase < 2; ++phase) {
      if (phase == 1) k_verify<<<g, 256, 0, stream>>>(dB);
      k_chunk_count<<<g, 256, 0, stream>>>(dB, phase);
      k_chunk_scan<<<std::min(ninst, g), kScanThreads, 0, stream>>>(dB, phase);
      k_chunk_emit<<<g, kChunkThreads, 0, stream>>>(dB, phase);
    }
    k_emit_rows<<<g, 256, 0, stream>>>(dB);
    k_finish<<<(ninst + 255) / 256, 256, 0, stream>>>(dB);
    cudaMemcpyAsync(h_status, hB.status_out, (size_t)ninst * sizeof(int2), cudaMemcpyDeviceToHost, stream);
  }

  cudaError_t run_step(int ninst, int p1_smem) {
    if (!step_exec || step_ninst != ninst || step_smem != p1_smem || step_grid != p1_grid) {
      if (step_exec) { cudaGraphExecDestroy(step_exec); step_exec = nullptr; }
      cudaGraph_t graph;
      cudaError_t e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) return e;
      launch_step(ninst, p1_smem);
      e = cudaStreamEndCapture(stream, &graph);
      if (e != cudaSuccess) return e;
      e = cudaGraphInstantiate(&step_exec, graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) { step_exec = nullptr; return e; }
      step_ninst = ninst;
      step_smem = p1_smem;
      step_grid = p1_grid;
    }
    return cudaGraphLaunch(step_exec, stream);
  }

  // ------------------------------------------------------ instance buffers
  vfb_status alloc_buffers(InstHost& H, uint64_t rows, uint64_t slots, uint64_t words, uint64_t tents) {
    InstDev& d = H.d;
    void* p;
    const size_t rb = rows * (size_t)d.TP * 8, ob = rows * 8, tb = slots * sizeof(Slot), bb = words * 4,
                 eb = tents * 8;
    if (dalloc(&p, rb) != cudaSuccess) return VFB_OOM;
    d.rows = (uint64_t*)p;
    if (dalloc(&p, ob) != cudaSuccess) return VFB_OOM;
    d.origin = (uint64_t*)p;
    if (dalloc(&p, tb) != cudaSuccess) return VFB_OOM;
    d.table = (Slot*)p;
    if (dalloc(&p, bb) != cudaSuccess) return VFB_OOM;
    d.bitmap = (uint32_t*)p;
    if (dalloc(&p, eb) != cudaSuccess) return VFB_OOM;
    d.tent = (uint64_t*)p;
    if (dalloc(&p, eb) != cudaSuccess) return VFB_OOM;
    d.wins = (uint64_t*)p;
    cudaMemsetAsync(d.table, 0xFF, tb, stream);
    cudaMemsetAsync(d.bitmap, 0, bb, stream);
    cudaMemsetAsync(d.rows, 0, rb, stream);
    d.row_cap = rows;
    d.table_mask = slots - 1;
    d.bitmap_words = words;
    d.tent_cap = tents;
    H.bytes = rb + ob + tb + bb + 2 * eb;
    return VFB_OK;
  }

  void free_buffers(InstHost& H) {
    InstDev& d = H.d;
    dfree(d.rows, d.row_cap * (size_t)d.TP * 8);
    dfree(d.origin, d.row_cap * 8);
    dfree(d.table, (d.table_mask + 1) * sizeof(Slot));
    dfree(d.bitmap, d.bitmap_words * 4);
    dfree(d.tent, d.tent_cap * 8);
    dfree(d.wins, d.tent_cap * 8);
    d.rows = d.origin = d.tent = d.wins = nullptr;
    d.table = nullptr;
    d.bitmap = nullptr;
    H.bytes = 0;
  }

  // Grow whatever the device asked for; the level is then re-run.
  vfb_status grow(InstHost& H, int idx) {
    InstDev& d = H.d;
    if (cudaMemcpyAsync(&d, dInst + idx, sizeof(InstDev), cudaMemcpyDeviceToHost, stream) != cudaSuccess)
      return VFB_DEVICE_ERROR;
    if (cudaStreamSynchronize(stream) != cudaSuccess) return VFB_DEVICE_ERROR;
    const int need = d.need;
    void* p;
    if (need & NEED_LIMIT) return VFB_LIMIT;
    if (need & NEED_ROWS) {
      const uint64_t want = std::max<uint64_t>(2 * d.row_cap, d.need_amount[3] + d.need_amount[3] / 4);
      const uint64_t used = d.lstart[d.level];
      if (dalloc(&p, want * (size_t)d.TP * 8) != cudaSuccess) return VFB_OOM;
      uint64_t* nr = (uint64_t*)p;
      cudaMemcpyAsync(nr, d.rows, used * (size_t)d.TP * 8, cudaMemcpyDeviceToDevice, stream);
      if (dalloc(&p, want * 8) != cudaSuccess) { dfree(nr, want * (size_t)d.TP * 8); return VFB_OOM; }
      uint64_t* no = (uint64_t*)p;
      cudaMemcpyAsync(no, d.origin, used * 8, cudaMemcpyDeviceToDevice, stream);
      dfree(d.rows, d.row_cap * (size_t)d.TP * 8);
      dfree(d.origin, d.row_cap * 8);
      H.bytes += (want - d.row_cap) * ((size_t)d.TP * 8 + 8);
      d.rows = nr;
      d.origin = no;
      d.row_cap = want;
    }
    if (need & NEED_TABLE) {
      const uint64_t cap = d.table_mask + 1;
      const uint64_t want = pow2_at_least(std::max<uint64_t>(2 * cap, d.need_amount[1]));
      if (dalloc(&p, want * sizeof(Slot)) != cudaSuccess) return VFB_OOM;
      Slot* nt = (Slot*)p;
      cudaMemsetAsync(nt, 0xFF, want * sizeof(Slot), stream);
      cudaMemsetAsync(d_fail, 0, sizeof(unsigned long long), stream);
      k_rehash<<<grid, 256, 0, stream>>>(d.table, cap, nt, want - 1, d_fail);
      unsigned long long fails = 0;
      cudaMemcpyAsync(&fails, d_fail, sizeof(fails), cudaMemcpyDeviceToHost, stream);
      if (cudaStreamSynchronize(stream) != cudaSuccess) return VFB_DEVICE_ERROR;
      if (fails) return VFB_DEVICE_ERROR;
      dfree(d.table, cap * sizeof(Slot));
      H.bytes += (want - cap) * sizeof(Slot);
      d.table = nt;
      d.table_mask = want - 1;
    }
    if (need & NEED_BITMAP) {
      const uint64_t want = std::max<uint64_t>(2 * d.bitmap_words, d.need_amount[0] + d.need_amount[0] / 4);
      if (dalloc(&p, want * 4) != cudaSuccess) return VFB_OOM;
      cudaMemsetAsync(p, 0, want * 4, stream);
      dfree(d.bitmap, d.bitmap_words * 4);
      H.bytes += (want - d.bitmap_words) * 4;
      d.bitmap = (uint32_t*)p;
      d.bitmap_words = want;
    }
    if (need & NEED_TENT) {
      const uint64_t want = std::max<uint64_t>(2 * d.tent_cap, d.need_amount[2] + d.need_amount[2] / 4);
      void* q;
      if (dalloc(&p, want * 8) != cudaSuccess) return VFB_OOM;
      if (dalloc(&q, want * 8) != cudaSuccess) { dfree(p, want * 8); return VFB_OOM; }
      dfree(d.tent, d.tent_cap * 8);
      dfree(d.wins, d.tent_cap * 8);
      H.bytes += (want - d.tent_cap) * 16;
      d.tent = (uint64_t*)p;
      d.wins = (uint64_t*)q;
      d.tent_cap = want;
    }
    d.status = ST_RUNNING;
    d.need = 0;
    if (cudaMemcpyAsync(dInst + idx, &d, sizeof(InstDev), cudaMemcpyHostToDevice, stream) != cudaSuccess)
      return VFB_DEVICE_ERROR;
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
    d.status = ST_RUNNING;
    d.level = 1;
    return VFB_OK;
  }

  vfb_status upload_atoms(const vfb_instance& in, InstHost& H, std::vector<uint64_t>& staging) {
    const InstDev& d = H.d;
    staging.assign((size_t)d.A * d.TP, 0ULL);
    for (int v = 0; v < d.A; ++v)
      for (int t = 0; t < d.T; ++t) staging[(size_t)v * d.TP + t] = in.words[(size_t)t * d.A + v];
    if (cudaMemcpyAsync(d.rows, staging.data(), staging.size() * 8, cudaMemcpyHostToDevice, stream) !=
        cudaSuccess)
      return VFB_DEVICE_ERROR;
    // the copy reads pageable memory: it completes before the call returns
    return VFB_OK;
  }

  vfb_status batch(const vfb_instance* ins, int n, vfb_result* out) {
    const auto t0 = std::chrono::steady_clock::now();
    if (n <= 0) return VFB_OK;
    if (cudaSetDevice(device) != cudaSuccess) return VFB_DEVICE_ERROR;
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

    vfb_status rc = VFB_OK;
    std::vector<uint64_t> staging;
    uint64_t chunk_need = 0;
    for (int i = 0; i < n && rc == VFB_OK; ++i) {
      if (H[i].fail != VFB_OK) continue;
      const InstDev& d = H[i].d;
      const uint64_t rows = std::max<uint64_t>(4096, (uint64_t)d.A * 16);
      const vfb_status s = alloc_buffers(H[i], rows, 1 << 14, 1 << 14, 1 << 13);
      if (s != VFB_OK) { H[i].fail = s; H[i].d.status = ST_IDLE; continue; }
      const vfb_status u = upload_atoms(ins[i], H[i], staging);
      if (u != VFB_OK) { rc = u; break; }
      H[i].active = true;
      chunk_need += (H[i].d.bitmap_words + kChunkWords - 1) / kChunkWords;
    }
    if (rc == VFB_OK) rc = ensure_workspace(n, chunk_need + n);
    if (rc == VFB_OK) {
      std::vector<InstDev> recs(n);
      for (int i = 0; i < n; ++i) recs[i] = H[i].d;
      if (cudaMemcpyAsync(dInst, recs.data(), (size_t)n * sizeof(InstDev), cudaMemcpyHostToDevice, stream) !=
          cudaSuccess)
        rc = VFB_DEVICE_ERROR;
      if (cudaStreamSynchronize(stream) != cudaSuccess) rc = VFB_DEVICE_ERROR;
    }
    if (rc == VFB_OK) {
      k_init<<<std::min(n, grid), 256, 0, stream>>>(dB);
      if (cudaMemcpyAsync(h_status, hB.status_out, (size_t)n * sizeof(int2), cudaMemcpyDeviceToHost, stream) !=
              cudaSuccess ||
          cudaStreamSynchronize(stream) != cudaSuccess)
        rc = VFB_DEVICE_ERROR;
    }
    int guard = 0;
    while (rc == VFB_OK) {
      bool running = false;
      for (int i = 0; i < n; ++i) {
        if (!H[i].active) continue;
        const int st = h_status[i].x;
        if (st == ST_RUNNING) running = true;
        if (st == ST_NEED_MEM) {
          const vfb_status g = grow(H[i], i);
          if (g != VFB_OK) {
            // this instance stops; the others carry on
            H[i].fail = g;
            H[i].active = false;
            InstDev& d = H[i].d;
            d.status = ST_ERROR;
            cudaMemcpyAsync(&dInst[i].status, &d.status, sizeof(int), cudaMemcpyHostToDevice, stream);
            if (g == VFB_DEVICE_ERROR) rc = g;
          } else {
            running = true;
          }
        }
        if (st == ST_ERROR) { H[i].fail = VFB_DEVICE_ERROR; H[i].active = false; }
      }
      if (!running || rc != VFB_OK) break;
      // the bitmap compaction needs room for every instance's chunks
      uint64_t cn = 0;
      for (int i = 0; i < n; ++i)
        if (H[i].d.bitmap) cn += (H[i].d.bitmap_words + kChunkWords - 1) / kChunkWords;
      if (cn + n > hB.chunk_cap) {
        rc = ensure_workspace(n, cn + n);
        if (rc != VFB_OK) break;
      }
      cudaError_t e = run_step(n, p1_smem);
      if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
      if (e != cudaSuccess) { last_error = e; rc = VFB_DEVICE_ERROR; break; }
      if (verbose) report_progress(n);
      if (++guard > 64 * kMaxSize) { rc = VFB_DEVICE_ERROR; break; }
    }
    // results
    std::vector<InstDev> recs(n);
    if (cudaMemcpyAsync(recs.data(), dInst, (size_t)n * sizeof(InstDev), cudaMemcpyDeviceToHost, stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess) {
      if (rc == VFB_OK) rc = VFB_DEVICE_ERROR;
    }
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    for (int i = 0; i < n; ++i) {
      vfb_result& r = out[i];
      const InstDev& d = recs[i];
      r.seconds = secs;
      if (H[i].fail != VFB_OK && !(H[i].d.rows)) {
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
        if (d.rpn_len != d.res_size) r.status = VFB_DEVICE_ERROR;
      } else if (d.status == ST_NOT_FOUND) {
        r.status = VFB_NOT_FOUND;
      } else {
        r.status = H[i].fail != VFB_OK ? H[i].fail : (rc != VFB_OK ? rc : VFB_DEVICE_ERROR);
        // level counts of the last level are not final
        if (r.size >= 1 && d.status != ST_FOUND) {
          r.total_rows -= r.level_rows[r.size];
          r.level_rows[r.size] = 0;
          r.level_cands[r.size] = 0;
          r.size = std::max(0, r.size - 1);
        }
      }
    }
    for (int i = 0; i < n; ++i)
      if (H[i].d.rows) free_buffers(H[i]);
    cudaStreamSynchronize(stream);
    return rc;
  }

  void report_progress(int n) {
    for (int i = 0; i < n; ++i) {
      InstDev d;
      if (cudaMemcpy(&d, dInst + i, sizeof(InstDev), cudaMemcpyDeviceToHost) != cudaSuccess) return;
      if (d.status == ST_NEED_MEM) continue;
      const int k = d.res_size;
      if (k < 1 || k > kMaxSize) continue;
      std::fprintf(stderr, "Length %-2d | (all) | CheckedLTLs: %-13llu | UniqueCS: %-12llu\n", k,
                   (unsigned long long)d.lcands[k], (unsigned long long)d.lcount[k]);
    }
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

vfb_status vfb_batch_solve(void* ctx, const vfb_instance* inst, int n, vfb_result* out) {
  if (!ctx || (n > 0 && (!inst || !out)) || n < 0) return VFB_BAD_INPUT;
  return static_cast<Engine*>(ctx)->batch(inst, n, out);
}

}  // extern "C"
