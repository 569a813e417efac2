// Shared device helpers and the context definition of libspexgpu.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "spexgpu.h"  // include/ is on the include path

// ---------------------------------------------------------------------------
// context

struct spx_ctx {
  int device = 0;
  int num_sms = 0;
  int cc_major = 0, cc_minor = 0;
  cudaStream_t stream = nullptr;   // main compute stream
  cudaStream_t copy_stream = nullptr;
  cudaStream_t prep_stream = nullptr;  // split-path operand preparation, overlapped
  cudaEvent_t sev[5] = {};             // split path: start, prep done x2, accumulation done x2
  spx_options opt{};
  std::string err;
  int* d_status = nullptr;         // device error word (0 = ok), see spx_status_*
  // grow-only device workspace, carved per call
  void* ws = nullptr;
  size_t ws_bytes = 0;
  // pinned host staging for pageable host arrays
  void* pinned = nullptr;
  size_t pinned_bytes = 0;
  cudaEvent_t ev[12] = {};          // 2-7: host-path chunk copies / frees (3 buffers), 8-9: tuners
  // optional per-kernel timing: marks recorded on the stream, summed after a sync
  bool timing = false;
  std::vector<cudaEvent_t> mark_pool;
  std::vector<int> mark_kind;
  size_t nmarks = 0;
  // split-path tuning table, one entry per (N bucket, pair bucket, nw)
  std::vector<spx_tune_entry> tune;
  // captured batched schedules, keyed by the batch signature (least recently used first out)
  struct BatchGraph {
    uint64_t key;
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    uint64_t last_use;
    void* mem;  // device memory the graph's persistent schedule owns (or NULL)
  };
  std::vector<BatchGraph> graphs;
  uint64_t graph_clock = 0;
  void* dn = nullptr;  // dense-solver handle of the dielectric inversion, made on first use
  // role profile of the persistent schedule (spx_pb_profile_*)
  unsigned long long* d_prof = nullptr;
  bool prof_on = false;
};

namespace spx {

// device status codes written by kernels into ctx->d_status
enum : int { kStatusOk = 0, kStatusTimeout = 1, kStatusBadLaunch = 2 };

// Tile code of the persistent schedule (tile columns + 256 x pipeline stages) when no
// tuning entry names one: 64 x 80 complex tiles, three stages.
constexpr int kPbDefaultTile = 80 + 3 * 256;

int set_error(spx_ctx* ctx, int code, const std::string& msg);
int check_cuda(spx_ctx* ctx, cudaError_t e, const char* what);
// Makes sure the workspace holds `bytes`; returns SPX_OK or SPX_ENOMEM.
int ensure_workspace(spx_ctx* ctx, size_t bytes);
int ensure_pinned(spx_ctx* ctx, size_t bytes);
// Reads and clears the device status word (synchronises `stream`).
int collect_status(spx_ctx* ctx, cudaStream_t stream, const char* what);
// Records a timing mark of `kind` (0 = operand preparation, 1 = band-pair
// accumulation, 2 = end) when ctx->timing is set.
void timing_mark(spx_ctx* ctx, cudaStream_t s, int kind);
// Sums the intervals between consecutive marks per kind (after a sync) and clears them.
void timing_collect(spx_ctx* ctx, double* ms_prep, double* ms_gram);
inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
// Carves 256-byte aligned pieces off a scratch range; ok turns false when it runs out.
struct Carve {
  char* p;
  size_t left;
  bool ok = true;
  template <class T>
  T* take(size_t n) {
    const size_t bytes = align_up(sizeof(T) * std::max<size_t>(n, 1), 256);
    if (bytes > left) {
      ok = false;
      return nullptr;
    }
    T* r = reinterpret_cast<T*>(p);
    p += bytes;
    left -= bytes;
    return r;
  }
};
inline cudaStream_t pick_stream(spx_ctx* ctx, void* s) {
  return s ? (cudaStream_t)s : ctx->stream;
}

// ---------------------------------------------------------------------------
// device helpers (sm_90+ PTX: mbarrier, bulk async copies, global timer)

#if defined(__CUDACC__)
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: returns false (and records a timeout in *status) if the phase
// with `parity` has not completed within `timeout_ns`. Polls with try_wait and
// looks at the clock and at the other CTAs' status only every 64 polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t timeout_ns,
                                          int* status) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (uint32_t n = 1;; ++n) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((n & 63) == 0) {
      if (global_ns() - t0 > timeout_ns) {
        atomicCAS(status, 0, (int)kStatusTimeout);
        return false;
      }
      if (*((volatile int*)status) != 0) return false;  // another CTA gave up
    }
  }
}
// The same bounded wait for warps that idle for long stretches (an epilogue waiting
// for a whole tile): the thread sleeps inside try_wait between polls.
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(2000u)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_idle(uint64_t* bar, uint32_t parity,
                                               uint64_t timeout_ns, int* status) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (uint32_t n = 1;; ++n) {
    if (mbar_try_wait_sleep(bar, parity)) return true;
    if ((n & 15) == 0) {
      if (global_ns() - t0 > timeout_ns) {
        atomicCAS(status, 0, (int)kStatusTimeout);
        return false;
      }
      if (*((volatile int*)status) != 0) return false;
    }
  }
}
// Bounded wait used only on the way out after a failure: waits for copies
// already issued to land, ignoring the status word, for at most timeout_ns.
__device__ __forceinline__ void mbar_drain(uint64_t* bar, uint32_t parity, uint64_t timeout_ns) {
  uint64_t t0 = global_ns();
  while (!mbar_try_wait(bar, parity))
    if (global_ns() - t0 > timeout_ns) return;
}
// 1-D bulk copy global -> shared through the TMA engine, completing on `bar`.
// dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
#endif

}  // namespace spx
