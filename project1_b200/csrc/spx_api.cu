// C ABI of libspexgpu: contexts, errors, and the chi0 accumulation driver.
//
// The driver replaces the packet loop body of `susceptibility`
// (src/susceptibility.f:751-1276): for each slab of band pairs it computes the
// FP64 weights (K6, :950-975) and accumulates the weighted Gram into the packed
// Hermitian output (K1 FP64 or K2 split precision, :1182-1240). Host-pointer
// calls stream cprod to the device slab by slab on a copy stream, double
// buffered, so that transfer and tensor-core work overlap; the slab is the
// analogue of the reference's MEM packet (:659-713), sized from device memory
// instead of the MEM keyword.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "spx_common.cuh"

namespace spx {

int launch_weights(spx_ctx*, int64_t, int64_t, const double*, const double*, double, int,
                   const double*, double*, cudaStream_t);
int launch_scale(spx_ctx*, double*, int64_t, double, cudaStream_t);
int launch_hilbert_weights(spx_ctx*, int64_t, int, int, const double*, int64_t, const double*,
                           double, double, double*, int64_t, cudaStream_t);
int launch_gen_normal(spx_ctx*, uint64_t, uint32_t, int64_t, int64_t, double, double*,
                      cudaStream_t);
int launch_gen_cmatrix(spx_ctx*, uint64_t, uint32_t, int64_t, int64_t, int64_t, int64_t,
                       double, double*, cudaStream_t);
int launch_chi0_fp64(spx_ctx*, const double2*, int64_t, int64_t, int, const double*, int64_t,
                     int, double2*, cudaStream_t, int);
int split_chi0_slab(spx_ctx*, const double2*, int64_t, int64_t, int, const double*, int64_t,
                    int, double2*, void*, size_t, cudaStream_t, int*, int variant, int slab);
size_t split_workspace_bytes(int64_t P, int N, int nw);
size_t split_workspace_bytes(int64_t P, int N, int nw, int slab);
size_t split_workspace_bytes_real(int64_t P, int N, int nw);
size_t pb_single_bytes(int64_t P, int N, int nw, int slab);
int pb_single(spx_ctx* ctx, const double2* M, int64_t ldc, int64_t P, int N, const double* ediff,
              const double* wscale, double scale_all, int nw, const double* omega, double2* out,
              int tile, int slab, char* scratch, size_t scratch_bytes, cudaStream_t s, int* launches);

// The split variant and slab a call of this shape runs with: the context's forced
// variant, else the tuning table's, else one CTA per 64 x 80 tile with 32768-pair slabs.
static void split_choice(spx_ctx* ctx, int N, int64_t P, int nw, int* variant, int* slab, int* tile) {
  *variant = ctx->opt.split_variant;
  *slab = 0;
  *tile = kPbDefaultTile;
  spx_tune_entry te;
  if (*variant == 0 && spx_tune_lookup(ctx, N, P, nw, &te) == SPX_OK) {
    *variant = te.variant;
    *slab = te.slab_pairs;
    if (te.tile) *tile = te.tile;
  }
}

// Scratch of the split path for a call of this shape (the persistent schedule's
// buffers when that is the variant in force).
static size_t split_scratch_bytes(spx_ctx* ctx, int64_t P, int N, int nw) {
  int variant, slab, tile;
  split_choice(ctx, N, P, nw, &variant, &slab, &tile);
  // a slab below P takes two buffers of that slab, which can exceed one buffer of
  // P pairs (P = 16000 at 8192-pair slabs)
  size_t b = split_workspace_bytes(P, N, nw);
  if (slab > 0) b = std::max(b, split_workspace_bytes(P, N, nw, slab));
  // the host path runs the plan chosen for the whole array on shorter chunks: every
  // entry for this width sizes the scratch for its slab and kernel
  bool persistent = variant == 3;
  for (const auto& e : ctx->tune) {
    if (e.nw != nw || e.variant == 4) continue;
    if (e.variant == 3) persistent = true;
    if (e.slab_pairs > 0) b = std::max(b, split_workspace_bytes(P, N, nw, e.slab_pairs));
  }
  if (persistent) b = std::max(b, pb_single_bytes(P, N, nw, 32768));
  return b;
}
int split_chi0_real_slab(spx_ctx*, const double*, int64_t, int64_t, int, const double*, int64_t,
                         int, double*, void*, size_t, cudaStream_t, int*);
int launch_chi0_fp64_real(spx_ctx*, const double*, int64_t, int64_t, int, const double*, int64_t,
                          int, double*, cudaStream_t);

void timing_mark(spx_ctx* ctx, cudaStream_t s, int kind) {
  if (!ctx->timing) return;
  if (ctx->nmarks == ctx->mark_pool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    ctx->mark_pool.push_back(e);
    ctx->mark_kind.push_back(0);
  }
  cudaEventRecord(ctx->mark_pool[ctx->nmarks], s);
  ctx->mark_kind[ctx->nmarks] = kind;
  ++ctx->nmarks;
}

void timing_collect(spx_ctx* ctx, double* ms_prep, double* ms_gram) {
  double prep = 0, gram = 0;
  for (size_t k = 0; k + 1 < ctx->nmarks; ++k) {
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->mark_pool[k], ctx->mark_pool[k + 1]);
    if (ctx->mark_kind[k] == 0) prep += ms;
    if (ctx->mark_kind[k] == 1) gram += ms;
  }
  ctx->nmarks = 0;
  if (ms_prep) *ms_prep = prep;
  if (ms_gram) *ms_gram = gram;
}

int set_error(spx_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return code;
}

int check_cuda(spx_ctx* ctx, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return SPX_OK;
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  if (e == cudaErrorMemoryAllocation) return set_error(ctx, SPX_ENOMEM, m);
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
    return set_error(ctx, SPX_ENODEV, m);
  return set_error(ctx, SPX_ECUDA, m);
}

int ensure_workspace(spx_ctx* ctx, size_t bytes) {
  if (bytes <= ctx->ws_bytes) return SPX_OK;
  if (ctx->opt.workspace_limit > 0 && bytes > (size_t)ctx->opt.workspace_limit)
    return set_error(ctx, SPX_ENOMEM,
                     "workspace of " + std::to_string(bytes) + " bytes exceeds workspace_limit");
  if (ctx->ws) {
    cudaFree(ctx->ws);
    ctx->ws = nullptr;
    ctx->ws_bytes = 0;
  }
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error(ctx, SPX_ENOMEM,
                     "cudaMalloc of " + std::to_string(bytes) + " bytes failed: " +
                         cudaGetErrorString(e));
  }
  ctx->ws = p;
  ctx->ws_bytes = bytes;
  return SPX_OK;
}

int ensure_pinned(spx_ctx* ctx, size_t bytes) {
  if (bytes <= ctx->pinned_bytes) return SPX_OK;
  if (ctx->pinned) {
    cudaFreeHost(ctx->pinned);
    ctx->pinned = nullptr;
    ctx->pinned_bytes = 0;
  }
  void* p = nullptr;
  cudaError_t e = cudaMallocHost(&p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error(ctx, SPX_ENOMEM, "cudaMallocHost failed: " + std::string(cudaGetErrorString(e)));
  }
  ctx->pinned = p;
  ctx->pinned_bytes = bytes;
  return SPX_OK;
}

int collect_status(spx_ctx* ctx, cudaStream_t stream, const char* what) {
  int h = 0;
  int rc = check_cuda(ctx, cudaMemcpyAsync(&h, ctx->d_status, sizeof(int),
                                           cudaMemcpyDeviceToHost, stream),
                      what);
  if (rc) return rc;
  rc = check_cuda(ctx, cudaStreamSynchronize(stream), what);
  if (rc) return rc;
  if (h != 0) {
    cudaMemsetAsync(ctx->d_status, 0, sizeof(int), stream);
    cudaStreamSynchronize(stream);
    if (h == kStatusTimeout)
      return set_error(ctx, SPX_ETIMEOUT,
                       std::string(what) + ": a device-side wait exceeded its time limit");
    return set_error(ctx, SPX_ECUDA, std::string(what) + ": device status " + std::to_string(h));
  }
  return SPX_OK;
}

static bool is_pinned_or_device(const void* p, bool* device) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    *device = false;
    return false;
  }
  *device = a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
  return a.type != cudaMemoryTypeUnregistered;
}

// Validates the arguments shared by both accumulation entry points.
static int check_chi0_args(spx_ctx* ctx, const double* cprod, int64_t ldc, int64_t npair,
                           int32_t nbas, const double* ediff, int32_t nw, const double* omega,
                           int32_t precision, const double* susceph) {
  if (!ctx) return SPX_EINVAL;
  if (npair < 0 || nbas < 0 || nw < 0) return set_error(ctx, SPX_EINVAL, "negative size");
  if (npair > 0 && nbas > 0 && nw > 0) {
    if (!cprod || !ediff || !omega || !susceph)
      return set_error(ctx, SPX_EINVAL, "null array argument");
    if (ldc < npair) return set_error(ctx, SPX_EINVAL, "ldc < npair");
  }
  if (nbas > 46340) return set_error(ctx, SPX_EINVAL, "nbas too large for packed indexing");
  if (precision != SPX_FP64 && precision != SPX_SPLIT)
    return set_error(ctx, SPX_EINVAL, "unknown precision");
  return SPX_OK;
}

// Accumulates one slab of band pairs already on the device into the device
// output. `W` is workspace for npair*nw weights (ldw = round_up(npair, 16)).
// `plan` (variant, slab, tile), when given, replaces the per-call choice: a caller
// that streams one array in chunks keeps one kernel and one slab size for all of it.
static int chi0_slab(spx_ctx* ctx, const double2* M, int64_t ldc, int64_t P, int N,
                     const double* ediff, const double* wscale, double scale_all, int nw,
                     const double* omega, int precision, double2* out, double* W,
                     void* split_ws, size_t split_ws_bytes, cudaStream_t s, int* launches,
                     const int* plan = nullptr) {
  const int64_t ldw = (int64_t)align_up((size_t)std::max<int64_t>(P, 1), 16);
  timing_mark(ctx, s, 0);
  int rc = launch_weights(ctx, P, ldw, ediff, wscale, scale_all, nw, omega, W, s);
  if (rc) return rc;
  ++*launches;
  if (precision == SPX_FP64) {
    timing_mark(ctx, s, 1);
    rc = launch_chi0_fp64(ctx, M, ldc, P, N, W, ldw, nw, out, s, 8);
    ++*launches;
  } else {
    // kernel variant and slab from the context's tuning table when the caller left
    // the variant open and the table has this shape (smaller slabs need less scratch)
    int variant, slab, tile;
    if (plan) variant = plan[0], slab = plan[1], tile = plan[2];
    else split_choice(ctx, N, P, nw, &variant, &slab, &tile);
    if (variant == 3) {
      // the persistent schedule forms its weights from ediff itself
      timing_mark(ctx, s, 1);
      rc = pb_single(ctx, M, ldc, P, N, ediff, wscale, scale_all, nw, omega, out, tile,
                     slab > 0 ? slab : 32768, (char*)split_ws, split_ws_bytes, s, launches);
    } else {
      // the split path marks its own preparation / accumulation phases
      rc = split_chi0_slab(ctx, M, ldc, P, N, W, ldw, nw, out, split_ws, split_ws_bytes, s,
                           launches, variant == 3 ? 0 : variant, slab);
    }
  }
  timing_mark(ctx, s, 2);
  return rc;
}

}  // namespace spx

using namespace spx;

// ---------------------------------------------------------------------------

extern "C" int spx_abi_version(void) { return SPX_ABI_VERSION; }

extern "C" const char* spx_strerror(int s) {
  switch (s) {
    case SPX_OK: return "ok";
    case SPX_EINVAL: return "invalid argument";
    case SPX_ENOMEM: return "out of memory";
    case SPX_ECUDA: return "CUDA error";
    case SPX_ETIMEOUT: return "device wait timed out";
    case SPX_ENOTSUP: return "not supported";
    case SPX_ENODEV: return "no CUDA device";
    default: return "unknown status";
  }
}

extern "C" int spx_ctx_create(int device, const spx_options* opt, spx_ctx** out) {
  if (!out) return SPX_EINVAL;
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    return SPX_ENODEV;
  }
  if (device < 0 || device >= n) return SPX_EINVAL;
  spx_ctx* ctx = new spx_ctx();
  if (opt) {
    size_t sz = opt->struct_size > 0 ? std::min<size_t>(opt->struct_size, sizeof(spx_options))
                                     : sizeof(spx_options);
    std::memcpy(&ctx->opt, opt, sz);
  }
  ctx->device = device;
  int rc;
  if ((rc = check_cuda(ctx, cudaSetDevice(device), "cudaSetDevice"))) {
    delete ctx;
    return rc;
  }
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, device);
  ctx->num_sms = prop.multiProcessorCount;
  ctx->cc_major = prop.major;
  ctx->cc_minor = prop.minor;
  if (prop.major != 10) {
    delete ctx;
    return SPX_ENOTSUP;  // kernels are built for sm_100a only
  }
  if ((rc = check_cuda(ctx, cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking),
                       "stream")) ||
      (rc = check_cuda(ctx, cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking),
                       "stream")) ||
      (rc = check_cuda(ctx, cudaStreamCreateWithFlags(&ctx->prep_stream, cudaStreamNonBlocking),
                       "stream")) ||
      (rc = check_cuda(ctx, cudaMalloc(&ctx->d_status, sizeof(int)), "status word")) ||
      (rc = check_cuda(ctx, cudaMemset(ctx->d_status, 0, sizeof(int)), "status word"))) {
    spx_ctx_destroy(ctx);
    return rc;
  }
  for (auto& ev : ctx->ev) cudaEventCreate(&ev);
  for (auto& ev : ctx->sev) cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
  *out = ctx;
  return SPX_OK;
}

namespace spx {
void dielec_release(spx_ctx* ctx);
}

extern "C" int spx_ctx_destroy(spx_ctx* ctx) {
  if (!ctx) return SPX_EINVAL;
  cudaSetDevice(ctx->device);
  spx::dielec_release(ctx);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
  if (ctx->prep_stream) cudaStreamSynchronize(ctx->prep_stream);
  for (auto& ev : ctx->ev)
    if (ev) cudaEventDestroy(ev);
  for (auto& ev : ctx->sev)
    if (ev) cudaEventDestroy(ev);
  for (auto& ev : ctx->mark_pool) cudaEventDestroy(ev);
  for (auto& g : ctx->graphs) {
    cudaGraphExecDestroy(g.exec);
    cudaGraphDestroy(g.graph);
    if (g.mem) cudaFree(g.mem);
  }
  if (ctx->ws) cudaFree(ctx->ws);
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  if (ctx->d_status) cudaFree(ctx->d_status);
  if (ctx->d_prof) cudaFree(ctx->d_prof);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  if (ctx->prep_stream) cudaStreamDestroy(ctx->prep_stream);
  delete ctx;
  return SPX_OK;
}

extern "C" const char* spx_last_error(const spx_ctx* ctx) {
  return ctx ? ctx->err.c_str() : "null context";
}

extern "C" int spx_ctx_synchronize(spx_ctx* ctx) {
  if (!ctx) return SPX_EINVAL;
  cudaSetDevice(ctx->device);
  int rc = check_cuda(ctx, cudaStreamSynchronize(ctx->copy_stream), "synchronize");
  if (rc) return rc;
  return collect_status(ctx, ctx->stream, "synchronize");
}

extern "C" int spx_weights_dev(spx_ctx* ctx, int64_t npair, const double* ediff,
                               const double* wscale, double scale_all, int32_t nw,
                               const double* omega, double* w, void* stream) {
  if (!ctx) return SPX_EINVAL;
  if (npair < 0 || nw < 0) return set_error(ctx, SPX_EINVAL, "negative size");
  if (npair == 0 || nw == 0) return SPX_OK;
  if (!ediff || !omega || !w) return set_error(ctx, SPX_EINVAL, "null array argument");
  cudaSetDevice(ctx->device);
  return launch_weights(ctx, npair, npair, ediff, wscale, scale_all, nw, omega, w,
                        pick_stream(ctx, stream));
}

extern "C" int spx_scale_dev(spx_ctx* ctx, double* z, int64_t n, double factor, void* stream) {
  if (!ctx) return SPX_EINVAL;
  if (n < 0) return set_error(ctx, SPX_EINVAL, "negative size");
  if (n > 0 && !z) return set_error(ctx, SPX_EINVAL, "null array argument");
  cudaSetDevice(ctx->device);
  return launch_scale(ctx, z, n, factor, pick_stream(ctx, stream));
}

extern "C" int spx_gen_normal_dev(spx_ctx* ctx, uint64_t seed, uint32_t stream_id,
                                  int64_t offset, int64_t n, double scale, double* out,
                                  void* stream) {
  if (!ctx) return SPX_EINVAL;
  if (n < 0 || offset < 0) return set_error(ctx, SPX_EINVAL, "negative size");
  if (n > 0 && !out) return set_error(ctx, SPX_EINVAL, "null array argument");
  cudaSetDevice(ctx->device);
  return launch_gen_normal(ctx, seed, stream_id, offset, n, scale, out,
                           pick_stream(ctx, stream));
}

extern "C" int spx_gen_cmatrix_dev(spx_ctx* ctx, uint64_t seed, uint32_t stream_id,
                                   int64_t rows, int64_t cols, int64_t ld, int64_t col0,
                                   double scale, double* out, void* stream) {
  if (!ctx) return SPX_EINVAL;
  if (rows < 0 || cols < 0 || col0 < 0) return set_error(ctx, SPX_EINVAL, "negative size");
  if (rows > 0 && cols > 0 && (!out || ld < rows))
    return set_error(ctx, SPX_EINVAL, "bad output array");
  cudaSetDevice(ctx->device);
  return launch_gen_cmatrix(ctx, seed, stream_id, rows, cols, ld, col0, scale, out,
                            pick_stream(ctx, stream));
}

extern "C" int spx_chi0_accumulate_dev(spx_ctx* ctx, const double* cprod, int64_t ldc,
                                       int64_t npair, int32_t nbas, const double* ediff,
                                       const double* wscale, double scale_all, int32_t nw,
                                       const double* omega, int32_t precision,
                                       double* susceph, void* stream, spx_chi0_stats* stats) {
  int rc = check_chi0_args(ctx, cprod, ldc, npair, nbas, ediff, nw, omega, precision, susceph);
  if (rc) return rc;
  cudaSetDevice(ctx->device);
  auto t0 = std::chrono::steady_clock::now();
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->precision = precision;
    stats->flops = 8.0 * (double)nbas * nbas * (double)npair * nw;
  }
  if (npair == 0 || nbas == 0 || nw == 0) return SPX_OK;
  cudaStream_t s = pick_stream(ctx, stream);
  const int64_t ldw = (int64_t)align_up((size_t)npair, 16);
  size_t wbytes = align_up(sizeof(double) * (size_t)ldw * nw, 256);
  size_t sbytes = precision == SPX_SPLIT ? split_scratch_bytes(ctx, npair, nbas, nw) : 0;
  if ((rc = ensure_workspace(ctx, wbytes + sbytes))) return rc;
  double* W = (double*)ctx->ws;
  void* sws = (char*)ctx->ws + wbytes;
  int launches = 0;
  ctx->timing = stats != nullptr;
  ctx->nmarks = 0;
  rc = chi0_slab(ctx, reinterpret_cast<const double2*>(cprod), ldc, npair, nbas, ediff, wscale,
                 scale_all, nw, omega, precision, reinterpret_cast<double2*>(susceph), W, sws,
                 sbytes, s, &launches);
  ctx->timing = false;
  if (rc) return rc;
  if (stats) {
    rc = collect_status(ctx, s, "chi0_accumulate_dev");
    if (rc) return rc;
    timing_collect(ctx, &stats->ms_prep, &stats->ms_gram);
    stats->kernel_launches = launches;
    stats->ms_total =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  return SPX_OK;
}

// -DINV build: real cprod and real packed susceph (MCOMPLEX_dp = real_dp,
// src/cppmacro.h:53-64; re(k) = cprod(k,i)*cprod(k,j), src/susceptibility.f:1197).
extern "C" int spx_chi0_accumulate_real_dev(spx_ctx* ctx, const double* cprod, int64_t ldc,
                                            int64_t npair, int32_t nbas, const double* ediff,
                                            const double* wscale, double scale_all, int32_t nw,
                                            const double* omega, int32_t precision,
                                            double* susceph, void* stream, spx_chi0_stats* stats) {
  int rc = check_chi0_args(ctx, cprod, ldc, npair, nbas, ediff, nw, omega, precision, susceph);
  if (rc) return rc;
  cudaSetDevice(ctx->device);
  auto t0 = std::chrono::steady_clock::now();
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->precision = precision;
    stats->flops = 2.0 * (double)nbas * nbas * (double)npair * nw;
  }
  if (npair == 0 || nbas == 0 || nw == 0) return SPX_OK;
  cudaStream_t s = pick_stream(ctx, stream);
  const int64_t ldw = (int64_t)align_up((size_t)npair, 16);
  const size_t wbytes = align_up(sizeof(double) * (size_t)ldw * nw, 256);
  const size_t sbytes = precision == SPX_SPLIT ? split_workspace_bytes_real(npair, nbas, nw) : 0;
  // the FP64 kernel streams M with 2-D tensor copies: columns must start on 16 bytes,
  // otherwise M goes through an aligned copy first
  const bool realign = precision == SPX_FP64 && ((ldc & 1) || ((uintptr_t)cprod & 15));
  const int64_t ldm = realign ? (int64_t)align_up((size_t)npair, 2) : ldc;
  const size_t mbytes = realign ? align_up(sizeof(double) * (size_t)ldm * nbas, 256) : 0;
  if ((rc = ensure_workspace(ctx, wbytes + sbytes + mbytes))) return rc;
  double* W = (double*)ctx->ws;
  void* sws = (char*)ctx->ws + wbytes;
  const double* M = cprod;
  if (realign) {
    double* Mc = (double*)((char*)ctx->ws + wbytes + sbytes);
    if ((rc = check_cuda(ctx, cudaMemcpy2DAsync(Mc, sizeof(double) * ldm, cprod, sizeof(double) * ldc,
                                                sizeof(double) * npair, nbas, cudaMemcpyDeviceToDevice, s),
                         "align cprod")))
      return rc;
    M = Mc;
  }
  int launches = 0;
  ctx->timing = stats != nullptr;
  ctx->nmarks = 0;
  timing_mark(ctx, s, 0);
  rc = launch_weights(ctx, npair, ldw, ediff, wscale, scale_all, nw, omega, W, s);
  ++launches;
  if (!rc) {
    if (precision == SPX_FP64) {
      timing_mark(ctx, s, 1);
      rc = launch_chi0_fp64_real(ctx, M, ldm, npair, nbas, W, ldw, nw, susceph, s);
      ++launches;
    } else {
      rc = split_chi0_real_slab(ctx, M, ldm, npair, nbas, W, ldw, nw, susceph, sws, sbytes, s, &launches);
    }
  }
  timing_mark(ctx, s, 2);
  ctx->timing = false;
  if (rc) return rc;
  if (stats) {
    rc = collect_status(ctx, s, "chi0_accumulate_real_dev");
    if (rc) return rc;
    timing_collect(ctx, &stats->ms_prep, &stats->ms_gram);
    stats->kernel_launches = launches;
    stats->ms_total =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  return SPX_OK;
}

// Copies columns [0, nbas) of rows [p0, p0+len) of a host cprod(ldc, nbas) into a
// dense pinned slab (len, nbas), using `nthr` host threads.
static void gather_slab(const double* cprod, int64_t ldc, int64_t p0, int64_t len, int nbas,
                        double* dst, int nthr) {
  auto work = [&](int t) {
    for (int c = t; c < nbas; c += nthr)
      std::memcpy(dst + 2 * (int64_t)c * len, cprod + 2 * ((int64_t)c * ldc + p0),
                  sizeof(double) * 2 * (size_t)len);
  };
  std::vector<std::thread> th;
  for (int t = 1; t < nthr; ++t) th.emplace_back(work, t);
  work(0);
  for (auto& x : th) x.join();
}

extern "C" int spx_chi0_accumulate(spx_ctx* ctx, const double* cprod, int64_t ldc,
                                   int64_t npair, int32_t nbas, const double* ediff,
                                   const double* wscale, double scale_all, int32_t nw,
                                   const double* omega, int32_t precision, double* susceph,
                                   spx_chi0_stats* stats) {
  int rc = check_chi0_args(ctx, cprod, ldc, npair, nbas, ediff, nw, omega, precision, susceph);
  if (rc) return rc;
  cudaSetDevice(ctx->device);
  auto t0 = std::chrono::steady_clock::now();
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->precision = precision;
    stats->flops = 8.0 * (double)nbas * nbas * (double)npair * nw;
  }
  if (npair == 0 || nbas == 0 || nw == 0) return SPX_OK;
  bool dev = false;
  const bool pinned = is_pinned_or_device(cprod, &dev);
  if (dev) return set_error(ctx, SPX_EINVAL, "cprod is a device pointer; use spx_chi0_accumulate_dev");

  // One split kernel and slab size for the whole array (chosen for npair), so that
  // the chunks' exact slabs are the device call's: chunk boundaries stay on
  // multiples of that slab and the result equals the device call's bit for bit.
  int plan[3] = {0, 0, kPbDefaultTile};
  if (precision == SPX_SPLIT) split_choice(ctx, nbas, npair, nw, &plan[0], &plan[1], &plan[2]);
  const int64_t align = precision == SPX_SPLIT ? (plan[1] > 0 ? plan[1] : 32768) : 16384;
  // slab size: band pairs per streamed chunk
  // By default the first chunk is short, since its copy overlaps nothing; the
  // chunks then grow by an eighth each time, up to 262144 pairs (a chunk's copy, about
  // 0.35-0.4 us per pair at N = 1200 over PCIe 5, against about 0.32-0.38 us of
  // accumulation), and halve again over the last quarter or so, so that little
  // accumulation is left once the last copy has landed. Pageable arrays keep
  // 65536-pair chunks so that their pinned staging stays small.
  const bool ramp = ctx->opt.chunk_pairs <= 0;
  int64_t slab = ctx->opt.chunk_pairs > 0 ? ctx->opt.chunk_pairs : (pinned ? 262144 : 65536);
  slab = std::min<int64_t>(slab, npair);
  slab = (int64_t)align_up((size_t)slab, 16);
  const int64_t first = ramp ? std::min<int64_t>(slab, (int64_t)align_up(16384, (size_t)align)) : slab;
  const int nslab_buf = 3;  // chunk k's copy waits only for chunk k-3's accumulation
  const int64_t npack = (int64_t)nbas * (nbas + 1) / 2;
  const size_t out_bytes = align_up(sizeof(double) * 2 * (size_t)npack * nw, 256);
  const size_t slab_bytes = align_up(sizeof(double) * 2 * (size_t)slab * nbas, 256);
  const size_t e_bytes = align_up(sizeof(double) * (size_t)slab, 256);
  const size_t om_bytes = align_up(sizeof(double) * (size_t)nw, 256);
  const size_t w_bytes = align_up(sizeof(double) * (size_t)slab * nw, 256);
  const size_t s_bytes = precision == SPX_SPLIT ? split_scratch_bytes(ctx, slab, nbas, nw) : 0;
  size_t total = out_bytes + nslab_buf * (slab_bytes + 2 * e_bytes) + om_bytes + w_bytes + s_bytes;
  if ((rc = ensure_workspace(ctx, total))) return rc;
  char* base = (char*)ctx->ws;
  double2* d_out = (double2*)base;
  base += out_bytes;
  double2* d_slab[nslab_buf];
  double* d_e[nslab_buf];
  double* d_ws[nslab_buf];
  for (int b = 0; b < nslab_buf; ++b) {
    d_slab[b] = (double2*)base;
    base += slab_bytes;
    d_e[b] = (double*)base;
    base += e_bytes;
    d_ws[b] = (double*)base;
    base += e_bytes;
  }
  double* d_om = (double*)base;
  base += om_bytes;
  double* d_w = (double*)base;
  base += w_bytes;
  void* d_split = s_bytes ? (void*)base : nullptr;

  const size_t out_host_bytes = sizeof(double) * 2 * (size_t)npack * nw;
  // pinned staging: the pageable slabs' gather, then the sums on their way back
  if ((rc = ensure_pinned(ctx, std::max(pinned ? (size_t)0 : nslab_buf * slab_bytes, out_host_bytes)))) return rc;
  double* stage = pinned ? nullptr : (double*)ctx->pinned;
  cudaStream_t cs = ctx->stream, xs = ctx->copy_stream;
  int64_t h2d = 0, d2h = 0;
  int launches = 0;
  // The device sums this call's contribution from zero; the host adds it to the
  // caller's susceph at the end (no upload of the output, a pinned download).
  if ((rc = check_cuda(ctx, cudaMemsetAsync(d_out, 0, out_host_bytes, cs), "zero output")))
    return rc;
  if ((rc = check_cuda(ctx, cudaMemcpyAsync(d_om, omega, sizeof(double) * nw,
                                            cudaMemcpyHostToDevice, cs),
                       "copy omega")))
    return rc;
  h2d += sizeof(double) * nw;
  cudaEvent_t ev_copied[nslab_buf] = {ctx->ev[2], ctx->ev[3], ctx->ev[4]};
  cudaEvent_t ev_free[nslab_buf] = {ctx->ev[5], ctx->ev[6], ctx->ev[7]};
  for (int b = 0; b < nslab_buf; ++b) cudaEventRecord(ev_free[b], cs);
  // device time of the accumulation and preparation (marks on the compute stream); the
  // rest of the call waits for the host copies
  ctx->timing = stats != nullptr;
  ctx->nmarks = 0;
  const int nthr = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
  int64_t k = 0;
  int64_t len = 0;
  for (int64_t p0 = 0; p0 < npair; p0 += len, ++k) {
    const int b = (int)(k % nslab_buf);
    int64_t want =
        k == 0 ? first
               : (ramp ? std::min<int64_t>(slab, (int64_t)align_up((size_t)(len + len / 8), (size_t)align))
                       : slab);
    // near the end the chunks halve: the accumulation left after the last copy lands
    // is that of a short chunk (the copies are the slower stream over PCIe)
    const int64_t left = npair - p0;
    if (ramp && k > 0 && left <= 2 * want)
      want = std::max<int64_t>(align, (int64_t)align_up((size_t)((left + 1) / 2), (size_t)align));
    len = std::min<int64_t>(want, left);
    cudaStreamWaitEvent(xs, ev_free[b], 0);
    const size_t bytes = sizeof(double) * 2 * (size_t)len;
    if (pinned) {
      rc = check_cuda(ctx, cudaMemcpy2DAsync(d_slab[b], bytes, cprod + 2 * p0, sizeof(double) * 2 * ldc,
                                             bytes, nbas, cudaMemcpyHostToDevice, xs),
                      "copy cprod slab");
    } else {
      // the staging part `b` is free once the previous copy out of it finished
      cudaEventSynchronize(ev_free[b]);
      double* st = stage + (size_t)b * (slab_bytes / sizeof(double));
      gather_slab(cprod, ldc, p0, len, nbas, st, nthr);
      rc = check_cuda(ctx, cudaMemcpyAsync(d_slab[b], st, bytes * nbas, cudaMemcpyHostToDevice, xs),
                      "copy cprod slab");
    }
    if (rc) {
      ctx->timing = false;
      return rc;
    }
    h2d += (int64_t)bytes * nbas;
    cudaMemcpyAsync(d_e[b], ediff + p0, sizeof(double) * len, cudaMemcpyHostToDevice, xs);
    h2d += sizeof(double) * len;
    if (wscale) {
      cudaMemcpyAsync(d_ws[b], wscale + p0, sizeof(double) * len, cudaMemcpyHostToDevice, xs);
      h2d += sizeof(double) * len;
    }
    cudaEventRecord(ev_copied[b], xs);
    cudaStreamWaitEvent(cs, ev_copied[b], 0);
    rc = chi0_slab(ctx, d_slab[b], len, len, nbas, d_e[b], wscale ? d_ws[b] : nullptr, scale_all,
                   nw, d_om, precision, d_out, d_w, d_split, s_bytes, cs, &launches,
                   precision == SPX_SPLIT ? plan : nullptr);
    if (rc) {
      ctx->timing = false;
      return rc;
    }
    cudaEventRecord(ev_free[b], cs);
  }
  ctx->timing = false;
  double* sums = (double*)ctx->pinned;
  if ((rc = check_cuda(ctx, cudaMemcpyAsync(sums, d_out, out_host_bytes, cudaMemcpyDeviceToHost, cs),
                       "copy the sums back")))
    return rc;
  d2h += out_host_bytes;
  rc = collect_status(ctx, cs, "chi0_accumulate");
  if (rc) return rc;
  {
    // susceph += sums, on the host threads
    const int64_t n = 2 * npack * nw;
    auto add = [&](int t) {
      const int64_t a = n * t / nthr, e = n * (t + 1) / nthr;
      for (int64_t i = a; i < e; ++i) susceph[i] += sums[i];
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nthr; ++t) th.emplace_back(add, t);
    add(0);
    for (auto& x : th) x.join();
  }
  if (stats) {
    timing_collect(ctx, &stats->ms_prep, &stats->ms_gram);
    stats->h2d_bytes = h2d;
    stats->d2h_bytes = d2h;
    stats->kernel_launches = launches;
    stats->ms_total =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  return SPX_OK;
}

// ---------------------------------------------------------------------------
// products and polarisation in one call (K4 -> K6 -> K1/K2), M stays on the device

namespace spx {
int wfprod_mt_run(spx_ctx*, const spx_mt_desc*, int, int, int, const double2*, const double2*,
                  double2*, int64_t, void*, size_t, cudaStream_t, int*);
int wfprod_pw_run(spx_ctx*, const spx_pw_desc*, int, int, int, const double2*, const double2*,
                  double2*, int64_t, int, void*, size_t, cudaStream_t, int*, bool, bool);
size_t wfprod_mt_workspace(const spx_mt_desc*, int, int);
size_t wfprod_pw_workspace(const spx_pw_desc*, int, int, int, bool);
}  // namespace spx

extern "C" int spx_chi0_from_coeffs_dev(spx_ctx* ctx, const spx_mt_desc* mt,
                                        const spx_pw_desc* pw, int32_t nk, int32_t nocc,
                                        int32_t nunocc, const double* cmt_occ,
                                        const double* cmt_unocc, const double* cpw_occ,
                                        const double* cpw_unocc, const double* ediff,
                                        const double* wscale, double scale_all, int32_t nw,
                                        const double* omega, int32_t precision, double* susceph,
                                        void* stream, spx_chi0_stats* stats) {
  if (!ctx) return SPX_EINVAL;
  if (!mt || !pw || !mt->gaunt || !mt->integral || !mt->cexp)
    return set_error(ctx, SPX_EINVAL, "null descriptor");
  if (nk < 0 || nocc < 0 || nunocc < 0 || nw < 0) return set_error(ctx, SPX_EINVAL, "negative size");
  const int64_t npair = (int64_t)nk * nocc * nunocc;
  const int maxllm = (mt->lcutm + 1) * (mt->lcutm + 1) * mt->nradm;
  const int64_t nbas64 = (int64_t)mt->natom * maxllm + pw->ngptm;
  if (nbas64 > 46340) return set_error(ctx, SPX_EINVAL, "nbas too large for packed indexing");
  const int nbas = (int)nbas64;
  // cprod is produced here: pass a non-null stand-in for the shared argument check
  int rc = check_chi0_args(ctx, ediff, npair, npair, nbas, ediff, nw, omega, precision, susceph);
  if (rc) return rc;
  if (npair > 0 && (!cmt_occ || !cmt_unocc || !cpw_occ || !cpw_unocc))
    return set_error(ctx, SPX_EINVAL, "null coefficient array");
  cudaSetDevice(ctx->device);
  auto t0 = std::chrono::steady_clock::now();
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->precision = precision;
    stats->flops = 8.0 * (double)nbas * nbas * (double)npair * nw;
  }
  if (npair == 0 || nbas == 0 || nw == 0) return SPX_OK;
  cudaStream_t s = pick_stream(ctx, stream);
  const int64_t ldc = (int64_t)align_up((size_t)npair, 16);
  const size_t m_bytes = align_up(sizeof(double2) * (size_t)ldc * nbas, 256);
  // interstitial products on int8 slices when the accumulation is split anyway
  const bool split_products = ctx->opt.products == SPX_PRODUCTS_SPLIT ||
                              (ctx->opt.products == SPX_PRODUCTS_AUTO && precision == SPX_SPLIT);
  const size_t prod_bytes = std::max(wfprod_mt_workspace(mt, nk, nocc),
                                     wfprod_pw_workspace(pw, nk, nocc, nunocc, split_products));
  const int64_t ldw = ldc;
  const size_t w_bytes = align_up(sizeof(double) * (size_t)ldw * nw, 256);
  const size_t s_bytes = precision == SPX_SPLIT ? split_scratch_bytes(ctx, npair, nbas, nw) : 0;
  const size_t scratch = std::max(prod_bytes, w_bytes + s_bytes);
  if ((rc = ensure_workspace(ctx, m_bytes + scratch))) return rc;
  double2* M = (double2*)ctx->ws;
  char* sc = (char*)ctx->ws + m_bytes;
  int launches = 0;
  ctx->timing = stats != nullptr;
  ctx->nmarks = 0;
  timing_mark(ctx, s, 0);
  if ((rc = check_cuda(ctx, cudaMemsetAsync(M, 0, m_bytes, s), "zero cprod"))) return rc;
  rc = wfprod_mt_run(ctx, mt, nk, nocc, nunocc, reinterpret_cast<const double2*>(cmt_occ),
                     reinterpret_cast<const double2*>(cmt_unocc), M, ldc, sc, scratch, s, &launches);
  if (!rc)
    rc = wfprod_pw_run(ctx, pw, nk, nocc, nunocc, reinterpret_cast<const double2*>(cpw_occ),
                       reinterpret_cast<const double2*>(cpw_unocc), M, ldc, mt->natom * maxllm,
                       sc, scratch, s, &launches, split_products, /*overwrite: M was zeroed*/ true);
  if (rc) {
    ctx->timing = false;
    return rc;
  }
  double* W = (double*)sc;
  void* sws = s_bytes ? (void*)(sc + w_bytes) : nullptr;
  rc = chi0_slab(ctx, M, ldc, npair, nbas, ediff, wscale, scale_all, nw, omega, precision,
                 reinterpret_cast<double2*>(susceph), W, sws, s_bytes, s, &launches);
  ctx->timing = false;
  if (rc) return rc;
  if (stats) {
    rc = collect_status(ctx, s, "chi0_from_coeffs_dev");
    if (rc) return rc;
    // the products count as preparation: everything before the first accumulation mark
    timing_collect(ctx, &stats->ms_prep, &stats->ms_gram);
    stats->kernel_launches = launches;
    stats->ms_total =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  return SPX_OK;
}

// ---------------------------------------------------------------------------
// Hilbert-mesh weights and the accumulation with caller-given weights

extern "C" int spx_weights_hilbert_dev(spx_ctx* ctx, int64_t npair, int32_t nfrqs,
                                       const double* wtetra, int64_t ldt, double thr, int32_t nw,
                                       const double* wghtSr, double scale_all, double* w,
                                       int64_t ldw, void* stream) {
  if (!ctx) return SPX_EINVAL;
  if (npair < 0 || nfrqs < 0 || nw < 0) return set_error(ctx, SPX_EINVAL, "negative size");
  if (npair == 0 || nw == 0) return SPX_OK;
  if (!w || (nfrqs > 0 && (!wtetra || !wghtSr))) return set_error(ctx, SPX_EINVAL, "null array argument");
  if (ldw < npair || (nfrqs > 0 && ldt < npair)) return set_error(ctx, SPX_EINVAL, "leading dimension too small");
  cudaSetDevice(ctx->device);
  return launch_hilbert_weights(ctx, npair, nfrqs, nw, wtetra, ldt, wghtSr, thr, scale_all, w, ldw,
                                pick_stream(ctx, stream));
}

// Adds sum_p M(p,i) conj(M(p,j)) w(p,f) with caller weights (any sign) into the
// packed `out`, using `scratch` (accumulate_w_scratch bytes) for the padded weight
// copy and the split path's planes.
static size_t accumulate_w_scratch(int64_t npair, int nbas, int nw, int precision) {
  const int64_t ldi = (int64_t)align_up((size_t)npair, 16);
  return align_up(sizeof(double) * (size_t)ldi * nw, 256) +
         (precision == SPX_SPLIT ? split_workspace_bytes(npair, nbas, nw) : 0);
}

static int accumulate_w_into(spx_ctx* ctx, const double* cprod, int64_t ldc, int64_t npair,
                             int nbas, const double* w, int64_t ldw, int nw, int precision,
                             double* out, char* scratch, cudaStream_t s, int* launches) {
  // the kernels read the weights with 16-pair bulk copies: an aligned, padded copy
  const int64_t ldi = (int64_t)align_up((size_t)npair, 16);
  const size_t wbytes = align_up(sizeof(double) * (size_t)ldi * nw, 256);
  const size_t sbytes = precision == SPX_SPLIT ? split_workspace_bytes(npair, nbas, nw) : 0;
  double* W = (double*)scratch;
  void* sws = scratch + wbytes;
  int rc;
  if ((rc = check_cuda(ctx, cudaMemsetAsync(W, 0, wbytes, s), "zero weights")) ||
      (rc = check_cuda(ctx, cudaMemcpy2DAsync(W, sizeof(double) * ldi, w, sizeof(double) * ldw,
                                              sizeof(double) * npair, nw, cudaMemcpyDeviceToDevice, s),
                       "copy weights")))
    return rc;
  if (precision == SPX_FP64) {
    timing_mark(ctx, s, 1);
    rc = launch_chi0_fp64(ctx, reinterpret_cast<const double2*>(cprod), ldc, npair, nbas, W, ldi, nw,
                          reinterpret_cast<double2*>(out), s, 8);
    ++*launches;
    return rc;
  }
  return split_chi0_slab(ctx, reinterpret_cast<const double2*>(cprod), ldc, npair, nbas, W, ldi, nw,
                         reinterpret_cast<double2*>(out), sws, sbytes, s, launches, 0, 0);
}

extern "C" int spx_chi0_accumulate_w_dev(spx_ctx* ctx, const double* cprod, int64_t ldc,
                                         int64_t npair, int32_t nbas, const double* w, int64_t ldw,
                                         int32_t nw, int32_t precision, double* susceph,
                                         void* stream, spx_chi0_stats* stats) {
  // the shared argument check, with w standing in for ediff and omega
  int rc = check_chi0_args(ctx, cprod, ldc, npair, nbas, w, nw, w, precision, susceph);
  if (rc) return rc;
  if (npair > 0 && nw > 0 && ldw < npair) return set_error(ctx, SPX_EINVAL, "ldw < npair");
  cudaSetDevice(ctx->device);
  auto t0 = std::chrono::steady_clock::now();
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->precision = precision;
    stats->flops = 8.0 * (double)nbas * nbas * (double)npair * nw;
  }
  if (npair == 0 || nbas == 0 || nw == 0) return SPX_OK;
  cudaStream_t s = pick_stream(ctx, stream);
  if ((rc = ensure_workspace(ctx, accumulate_w_scratch(npair, nbas, nw, precision)))) return rc;
  int launches = 0;
  ctx->timing = stats != nullptr;
  ctx->nmarks = 0;
  rc = accumulate_w_into(ctx, cprod, ldc, npair, nbas, w, ldw, nw, precision, susceph,
                         (char*)ctx->ws, s, &launches);
  timing_mark(ctx, s, 2);
  ctx->timing = false;
  if (rc) return rc;
  if (stats) {
    rc = collect_status(ctx, s, "chi0_accumulate_w_dev");
    if (rc) return rc;
    timing_collect(ctx, &stats->ms_prep, &stats->ms_gram);
    stats->kernel_launches = launches;
    stats->ms_total =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  return SPX_OK;
}

namespace spx {
int launch_suscepc_combine(spx_ctx*, int, int, const double2*, const double2*, double2*, int64_t,
                           cudaStream_t);
}

extern "C" int spx_chi0_accumulate_c_dev(spx_ctx* ctx, const double* cprod, int64_t ldc,
                                         int64_t npair, int32_t nbas, const double* wr,
                                         const double* wi, int64_t ldw, int32_t nw,
                                         int32_t precision, double* suscepc, int64_t ldo,
                                         void* stream, spx_chi0_stats* stats) {
  int rc = check_chi0_args(ctx, cprod, ldc, npair, nbas, wr, nw, wr, precision, suscepc);
  if (rc) return rc;
  if (npair > 0 && nw > 0 && (!wi || ldw < npair)) return set_error(ctx, SPX_EINVAL, "wi NULL or ldw < npair");
  if (nbas > 0 && ldo < nbas) return set_error(ctx, SPX_EINVAL, "ldo < nbas");
  cudaSetDevice(ctx->device);
  auto t0 = std::chrono::steady_clock::now();
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->precision = precision;
    stats->flops = 2 * 8.0 * (double)nbas * nbas * (double)npair * nw;
  }
  if (npair == 0 || nbas == 0 || nw == 0) return SPX_OK;
  cudaStream_t s = pick_stream(ctx, stream);
  // two packed Hermitian sums S1 (weights wr) and S2 (weights wi), then the full matrix
  const int64_t npack = (int64_t)nbas * (nbas + 1) / 2;
  const size_t pbytes = align_up(sizeof(double2) * (size_t)npack * nw, 256);
  const size_t sc = accumulate_w_scratch(npair, nbas, nw, precision);
  if ((rc = ensure_workspace(ctx, 2 * pbytes + sc))) return rc;
  double* S1 = (double*)ctx->ws;
  double* S2 = (double*)((char*)ctx->ws + pbytes);
  char* scratch = (char*)ctx->ws + 2 * pbytes;
  int launches = 0;
  ctx->timing = stats != nullptr;
  ctx->nmarks = 0;
  if ((rc = check_cuda(ctx, cudaMemsetAsync(S1, 0, 2 * pbytes, s), "zero partial sums"))) return rc;
  rc = accumulate_w_into(ctx, cprod, ldc, npair, nbas, wr, ldw, nw, precision, S1, scratch, s, &launches);
  if (!rc) rc = accumulate_w_into(ctx, cprod, ldc, npair, nbas, wi, ldw, nw, precision, S2, scratch, s, &launches);
  if (!rc) {
    timing_mark(ctx, s, 0);
    rc = launch_suscepc_combine(ctx, nbas, nw, (const double2*)S1, (const double2*)S2,
                                reinterpret_cast<double2*>(suscepc), ldo, s);
    ++launches;
  }
  timing_mark(ctx, s, 2);
  ctx->timing = false;
  if (rc) return rc;
  if (stats) {
    rc = collect_status(ctx, s, "chi0_accumulate_c_dev");
    if (rc) return rc;
    timing_collect(ctx, &stats->ms_prep, &stats->ms_gram);
    stats->kernel_launches = launches;
    stats->ms_total =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  return SPX_OK;
}
