// Allocation-free form of the FP64 band-pair accumulation.
//
// Some callers cannot call cudaMalloc: a Fortran host program whose device heap
// is owned by its OpenMP/OpenACC offload runtime or by a pool allocator, or
// code running under a process-level device-memory cap where every allocation is
// accounted elsewhere. For them this entry point uses no context and allocates
// nothing. Its only scratch (the FP64 frequency weights of one slab of band
// pairs, plus a status word) lives in the file-scope arrays below. They take
// SPX_NOALLOC_SCRATCH_BYTES (32 MiB) plus 256 bytes on every GPU that loads this
// part of the library, and they stay there until the process exits.
//
// The first call on a device looks up the arrays' device addresses with
// cudaGetSymbolAddress while that device is current, and looks them up again
// whenever the device's current context has changed since (after a
// cudaDeviceReset or a runtime that destroys and recreates the primary context,
// the module and its arrays are loaded anew). Every call ends by reading a status
// word back and synchronizing its stream, so no call may be made while that
// stream is being captured into a graph. Every call shares the same arrays, so
// calls that overlap on the GPU (two streams, two host threads) race on them: a
// caller must order such calls itself.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "spx_common.cuh"

#define SPX_NOALLOC_SCRATCH_BYTES (32u << 20)

namespace spx {
int launch_weights_noctx(int, int64_t, int64_t, const double*, const double*, double, int,
                         const double*, double*, cudaStream_t);
int launch_chi0_fp64_noctx(int, int*, uint64_t, const double2*, int64_t, int64_t, int,
                           const double*, int64_t, int, double2*, cudaStream_t);
}  // namespace spx

static __device__ __align__(256) double g_noalloc_weights[SPX_NOALLOC_SCRATCH_BYTES / 8];
static __device__ __align__(256) int g_noalloc_status[64];

namespace {

struct NoallocDevice {
  bool ready = false;
  unsigned long long ctx_id = 0;  // context the addresses below belong to
  double* weights = nullptr;  // device address of g_noalloc_weights on this device
  int* status = nullptr;      // device address of g_noalloc_status on this device
  int num_sms = 0;
};

constexpr int kMaxDevices = 64;
NoallocDevice g_dev[kMaxDevices];
std::mutex g_mu;

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

// Unique id of the calling thread's current context (0 if it cannot be read).
unsigned long long current_ctx_id() {
  static CtxGetCurrentFn get_cur = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool looked = false;
  if (!looked) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_cur = (CtxGetCurrentFn)p;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = (CtxGetIdFn)p;
    looked = true;
  }
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (get_cur && get_id && get_cur(&c) == CUDA_SUCCESS && c && get_id(c, &id) == CUDA_SUCCESS)
    return id;
  return 0;
}

// With the device current: resolve the static arrays for its current context
// (once, and again after that context has been replaced).
int noalloc_setup(int dev, NoallocDevice** out) {
  std::lock_guard<std::mutex> lock(g_mu);
  NoallocDevice& d = g_dev[dev];
  // No current context yet (first use, or just after a device reset) reads as 0:
  // the symbol lookup below makes the runtime bind the device's primary context,
  // and the id is read again after it.
  const unsigned long long before = current_ctx_id();
  if (d.ready && (before == 0 || before != d.ctx_id)) d.ready = false;
  if (!d.ready) {
    if (cudaGetSymbolAddress((void**)&d.weights, g_noalloc_weights) != cudaSuccess ||
        cudaGetSymbolAddress((void**)&d.status, g_noalloc_status) != cudaSuccess) {
      cudaGetLastError();
      return SPX_ECUDA;
    }
    if (cudaDeviceGetAttribute(&d.num_sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
      cudaGetLastError();
      return SPX_ECUDA;
    }
    d.ctx_id = current_ctx_id();
    d.ready = d.ctx_id != 0;
  }
  *out = &d;
  return SPX_OK;
}

}  // namespace

// Same result as spx_chi0_accumulate_dev(..., SPX_FP64, ...) on the device current
// to the calling thread, with every array a device pointer and no allocation.
// The weights of one slab of band pairs must fit the static scratch:
// 16 * nw * 8 bytes <= SPX_NOALLOC_SCRATCH_BYTES, i.e. nw <= 262144; larger nw is
// rejected with SPX_EINVAL, and so is nbas > 46340 (the packed index of the last
// element must fit 31 bits). Returns after the work on `stream` has completed.
extern "C" int spx_chi0_accumulate_dev_noalloc(const double* cprod, int64_t ldc, int64_t npair,
                                               int32_t nbas, const double* ediff,
                                               const double* wscale, double scale_all,
                                               int32_t nw, const double* omega, double* susceph,
                                               void* stream) {
  if (npair < 0 || nbas < 0 || nw < 0) return SPX_EINVAL;
  if (npair == 0 || nbas == 0 || nw == 0) return SPX_OK;
  if (!cprod || !ediff || !omega || !susceph || ldc < npair) return SPX_EINVAL;
  if (nbas > 46340) return SPX_EINVAL;
  const int64_t cap = SPX_NOALLOC_SCRATCH_BYTES / 8;  // doubles
  int64_t slab = (cap / nw) / 16 * 16;               // pairs whose weights fit
  if (slab < 16) return SPX_EINVAL;                  // nw beyond the scratch maximum
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return SPX_ENODEV;
  }
  NoallocDevice* d = nullptr;
  int rc = noalloc_setup(dev, &d);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  // the status word keeps the previous call's value: clear it
  if (cudaMemsetAsync(d->status, 0, sizeof(int), s) != cudaSuccess) return SPX_ECUDA;
  const uint64_t timeout_ns = 4000ull * 1000000ull;
  slab = std::min<int64_t>(slab, (npair + 15) / 16 * 16);
  for (int64_t p0 = 0; p0 < npair; p0 += slab) {
    const int64_t len = std::min<int64_t>(slab, npair - p0);
    const int64_t ldw = (len + 15) / 16 * 16;
    rc = spx::launch_weights_noctx(d->num_sms, len, ldw, ediff + p0, wscale ? wscale + p0 : nullptr,
                                   scale_all, nw, omega, d->weights, s);
    if (rc) return rc;
    rc = spx::launch_chi0_fp64_noctx(d->num_sms, d->status, timeout_ns,
                                     reinterpret_cast<const double2*>(cprod) + p0, ldc, len, nbas,
                                     d->weights, ldw, nw, reinterpret_cast<double2*>(susceph), s);
    if (rc) return rc;
  }
  int h = 0;
  if (cudaMemcpyAsync(&h, d->status, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    cudaGetLastError();
    return SPX_ECUDA;
  }
  return h == 0 ? SPX_OK : SPX_ETIMEOUT;
}
