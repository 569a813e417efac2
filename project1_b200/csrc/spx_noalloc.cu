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
// cudaGetSymbolAddress while that device is current. Make this first call
// before any stream capture begins. Every call shares the same arrays, so calls
// that overlap on the GPU (two streams, two host threads) race on them: a
// caller must order such calls itself.
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
  double* weights = nullptr;  // device address of g_noalloc_weights on this device
  int* status = nullptr;      // device address of g_noalloc_status on this device
  int num_sms = 0;
};

constexpr int kMaxDevices = 64;
NoallocDevice g_dev[kMaxDevices];
std::mutex g_mu;

// Once per device, with that device current: resolve the static arrays.
int noalloc_setup(int dev, NoallocDevice** out) {
  std::lock_guard<std::mutex> lock(g_mu);
  NoallocDevice& d = g_dev[dev];
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
    d.ready = true;
  }
  *out = &d;
  return SPX_OK;
}

}  // namespace

// Same result as spx_chi0_accumulate_dev(..., SPX_FP64, ...) on the device current
// to the calling thread, with every array a device pointer and no allocation.
// The weights of one slab of band pairs must fit the static scratch:
// 16 * nw * 8 bytes <= SPX_NOALLOC_SCRATCH_BYTES, i.e. nw <= 262144; larger nw is
// rejected with SPX_EINVAL. Returns after the work on `stream` has completed.
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
