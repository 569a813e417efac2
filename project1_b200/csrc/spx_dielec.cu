// Dielectric matrix and its inverse in FP64 (src/correlation.f:614-636, :703-745).
//
// For every imaginary frequency the reference turns the packed polarisation into
//   eps_ij = delta_ij - sqrt(v_i) chi_ij sqrt(v_j)          (p_diagmatdiag, p_plusdiag)
// with v the Coulomb eigenvalues of the basis (the Coulomb-eigenbasis transform has
// made v diagonal), and inverts it as a packed Hermitian matrix (LAPACK zpptrf/zpptri
// on one process, ScaLAPACK with MPI). On the imaginary axis chi is negative
// semi-definite, so eps = 1 + (positive semi-definite) is positive definite and the
// Cholesky route is the natural one. At Gamma the 3x3 head becomes 1 - 4 pi head and
// the wings -sqrt(4 pi) sqrt(v_i) wing.
//
// The build, unpack and pack steps are kernels of this file; the factorisation and
// the inverse from it (potrf, potri on the unpacked upper triangle) are cuSOLVER's,
// loaded at the first call, the way a plain GEMM may come from cuBLAS. Status of
// every frequency's factorisation is collected and reported after the batch.
#include <cuda_runtime.h>
#include <cusolverDn.h>
#include <dlfcn.h>

#include <mutex>
#include <string>
#include <vector>

#include "spx_common.cuh"

namespace spx {

__global__ void dielec_unpack_kernel(const double2* __restrict__ chi, const double* __restrict__ sq,
                                     int n, double2* __restrict__ full) {
  const int64_t total = (int64_t)n * n;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % n), j = (int)(t / n);
    double2 v;
    if (i <= j) {
      v = chi[(int64_t)j * (j + 1) / 2 + i];
    } else {
      v = chi[(int64_t)i * (i + 1) / 2 + j];
      v.y = -v.y;
    }
    const double s = -sq[i] * sq[j];
    double2 e = make_double2(s * v.x, s * v.y);
    if (i == j) e.x += 1.0;
    full[t] = e;
  }
}

__global__ void dielec_build_packed_kernel(double2* __restrict__ p, const double* __restrict__ sq,
                                           int n, int64_t npack, int nw) {
  const int64_t total = npack * nw;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t ij = t % npack;
    int j = (int)((sqrt(8.0 * (double)ij + 1.0) - 1.0) * 0.5);
    while ((int64_t)j * (j + 1) / 2 > ij) --j;
    while ((int64_t)(j + 1) * (j + 2) / 2 <= ij) ++j;
    const int i = (int)(ij - (int64_t)j * (j + 1) / 2);
    const double s = -sq[i] * sq[j];
    double2 v = p[t];
    v.x *= s;
    v.y *= s;
    if (i == j) v.x += 1.0;
    p[t] = v;
  }
}

__global__ void pack_upper_kernel(const double2* __restrict__ full, int n, double2* __restrict__ packed) {
  const int64_t npack = (int64_t)n * (n + 1) / 2;
  for (int64_t ij = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; ij < npack;
       ij += (int64_t)gridDim.x * blockDim.x) {
    int j = (int)((sqrt(8.0 * (double)ij + 1.0) - 1.0) * 0.5);
    while ((int64_t)j * (j + 1) / 2 > ij) --j;
    while ((int64_t)(j + 1) * (j + 2) / 2 <= ij) ++j;
    const int i = (int)(ij - (int64_t)j * (j + 1) / 2);
    packed[ij] = full[i + (int64_t)n * j];
  }
}

// head(:, f) = I3 - 4 pi head(:, f) (packed 3x3), wing(:, i, f) = -sqrt(4 pi) sqrt(v_i) wing
__global__ void dielec_headwing_kernel(double2* head, double2* wing, const double* __restrict__ sq,
                                       int n, int nw) {
  const double fourpi = 4.0 * 3.14159265358979323846;
  const double sfp = sqrt(fourpi);
  const int64_t nh = 6LL * nw, ng = wing ? 3LL * n * nw : 0;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nh + ng;
       t += (int64_t)gridDim.x * blockDim.x) {
    if (t < nh) {
      if (!head) continue;
      const int ij = (int)(t % 6);
      double2 v = head[t];
      v.x = -fourpi * v.x;
      v.y = -fourpi * v.y;
      if (ij == 0 || ij == 2 || ij == 5) v.x += 1.0;
      head[t] = v;
    } else {
      const int64_t u = t - nh;
      const int i = (int)((u / 3) % n);
      const double f = -sfp * sq[i];
      double2 v = wing[u];
      wing[u] = make_double2(f * v.x, f * v.y);
    }
  }
}

__global__ void sqrt_kernel(const double* __restrict__ v, double* __restrict__ s, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    s[i] = sqrt(v[i]);
}

// cuSOLVER entry points, resolved once
struct DnApi {
  bool ok = false;
  std::string err;
  cusolverStatus_t (*create)(cusolverDnHandle_t*);
  cusolverStatus_t (*destroy)(cusolverDnHandle_t);
  cusolverStatus_t (*set_stream)(cusolverDnHandle_t, cudaStream_t);
  cusolverStatus_t (*potrf_bs)(cusolverDnHandle_t, cublasFillMode_t, int, cuDoubleComplex*, int, int*);
  cusolverStatus_t (*potrf)(cusolverDnHandle_t, cublasFillMode_t, int, cuDoubleComplex*, int,
                            cuDoubleComplex*, int, int*);
  cusolverStatus_t (*potri_bs)(cusolverDnHandle_t, cublasFillMode_t, int, cuDoubleComplex*, int, int*);
  cusolverStatus_t (*potri)(cusolverDnHandle_t, cublasFillMode_t, int, cuDoubleComplex*, int,
                            cuDoubleComplex*, int, int*);
};

static DnApi& dn_api() {
  static DnApi api;
  static std::once_flag once;
  std::call_once(once, [] {
    void* h = dlopen("libcusolver.so.11", RTLD_NOW | RTLD_LOCAL);
    if (!h) h = dlopen("libcusolver.so", RTLD_NOW | RTLD_LOCAL);
    if (!h) {
      api.err = "cannot load libcusolver";
      return;
    }
    auto sym = [&](const char* name) { return dlsym(h, name); };
    api.create = (decltype(api.create))sym("cusolverDnCreate");
    api.destroy = (decltype(api.destroy))sym("cusolverDnDestroy");
    api.set_stream = (decltype(api.set_stream))sym("cusolverDnSetStream");
    api.potrf_bs = (decltype(api.potrf_bs))sym("cusolverDnZpotrf_bufferSize");
    api.potrf = (decltype(api.potrf))sym("cusolverDnZpotrf");
    api.potri_bs = (decltype(api.potri_bs))sym("cusolverDnZpotri_bufferSize");
    api.potri = (decltype(api.potri))sym("cusolverDnZpotri");
    api.ok = api.create && api.destroy && api.set_stream && api.potrf_bs && api.potrf &&
             api.potri_bs && api.potri;
    if (!api.ok) api.err = "libcusolver lacks an entry point";
  });
  return api;
}

void dielec_release(spx_ctx* ctx) {
  if (ctx->dn) {
    DnApi& api = dn_api();
    if (api.ok) api.destroy((cusolverDnHandle_t)ctx->dn);
    ctx->dn = nullptr;
  }
}

}  // namespace spx

using namespace spx;

extern "C" int spx_dielec_dev(spx_ctx* ctx, int32_t nbas, int32_t nw, double* susceph,
                              const double* coul, int32_t invert, double* head, double* wing,
                              void* stream) {
  if (!ctx) return SPX_EINVAL;
  if (nbas < 0 || nw < 0) return set_error(ctx, SPX_EINVAL, "negative size");
  if (nbas == 0 || nw == 0) return SPX_OK;
  if (!susceph || !coul) return set_error(ctx, SPX_EINVAL, "null array argument");
  if (nbas > 46340) return set_error(ctx, SPX_EINVAL, "nbas too large for packed indexing");
  cudaSetDevice(ctx->device);
  cudaStream_t s = pick_stream(ctx, stream);
  const int n = nbas;
  const int64_t npack = (int64_t)n * (n + 1) / 2;
  const int grid = ctx->num_sms * 8;
  int rc;
  // scratch: sqrt(v), infos, and for the inversion one full matrix and the solver buffer
  size_t need = align_up(sizeof(double) * n, 256) + align_up(sizeof(int) * 2 * nw, 256);
  int lwork = 0;
  DnApi* api = nullptr;
  if (invert) {
    api = &dn_api();
    if (!api->ok) return set_error(ctx, SPX_ENOTSUP, api->err);
    if (!ctx->dn) {
      cusolverDnHandle_t hdl;
      if (api->create(&hdl) != CUSOLVER_STATUS_SUCCESS)
        return set_error(ctx, SPX_ECUDA, "cusolverDnCreate failed");
      ctx->dn = hdl;
    }
    cusolverDnHandle_t hdl = (cusolverDnHandle_t)ctx->dn;
    int l1 = 0, l2 = 0;
    if (api->potrf_bs(hdl, CUBLAS_FILL_MODE_UPPER, n, nullptr, n, &l1) != CUSOLVER_STATUS_SUCCESS ||
        api->potri_bs(hdl, CUBLAS_FILL_MODE_UPPER, n, nullptr, n, &l2) != CUSOLVER_STATUS_SUCCESS)
      return set_error(ctx, SPX_ECUDA, "cuSOLVER buffer size query failed");
    lwork = std::max(std::max(l1, l2), 1);
    need += align_up(sizeof(double2) * (size_t)n * n, 256) + align_up(sizeof(double2) * (size_t)lwork, 256);
  }
  if ((rc = ensure_workspace(ctx, need + 1024))) return rc;
  char* b = (char*)ctx->ws;
  double* sq = (double*)b;
  b += align_up(sizeof(double) * n, 256);
  int* info = (int*)b;
  b += align_up(sizeof(int) * 2 * nw, 256);
  sqrt_kernel<<<(n + 255) / 256, 256, 0, s>>>(coul, sq, n);
  if ((rc = check_cuda(ctx, cudaGetLastError(), "sqrt_kernel launch"))) return rc;
  double2* P = reinterpret_cast<double2*>(susceph);
  if (head || wing) {
    dielec_headwing_kernel<<<grid, 256, 0, s>>>(reinterpret_cast<double2*>(head),
                                                reinterpret_cast<double2*>(wing), sq, n, nw);
    if ((rc = check_cuda(ctx, cudaGetLastError(), "dielec_headwing_kernel launch"))) return rc;
  }
  if (!invert) {
    dielec_build_packed_kernel<<<grid, 256, 0, s>>>(P, sq, n, npack, nw);
    return check_cuda(ctx, cudaGetLastError(), "dielec_build_packed_kernel launch");
  }
  double2* full = reinterpret_cast<double2*>(b);
  b += align_up(sizeof(double2) * (size_t)n * n, 256);
  double2* work = reinterpret_cast<double2*>(b);
  cusolverDnHandle_t hdl = (cusolverDnHandle_t)ctx->dn;
  if (api->set_stream(hdl, s) != CUSOLVER_STATUS_SUCCESS)
    return set_error(ctx, SPX_ECUDA, "cusolverDnSetStream failed");
  if ((rc = check_cuda(ctx, cudaMemsetAsync(info, 0, sizeof(int) * 2 * nw, s), "zero info"))) return rc;
  for (int f = 0; f < nw; ++f) {
    dielec_unpack_kernel<<<grid, 256, 0, s>>>(P + (int64_t)f * npack, sq, n, full);
    if ((rc = check_cuda(ctx, cudaGetLastError(), "dielec_unpack_kernel launch"))) return rc;
    if (api->potrf(hdl, CUBLAS_FILL_MODE_UPPER, n, reinterpret_cast<cuDoubleComplex*>(full), n,
                   reinterpret_cast<cuDoubleComplex*>(work), lwork, info + 2 * f) != CUSOLVER_STATUS_SUCCESS ||
        api->potri(hdl, CUBLAS_FILL_MODE_UPPER, n, reinterpret_cast<cuDoubleComplex*>(full), n,
                   reinterpret_cast<cuDoubleComplex*>(work), lwork, info + 2 * f + 1) != CUSOLVER_STATUS_SUCCESS)
      return set_error(ctx, SPX_ECUDA, "cuSOLVER potrf/potri launch failed");
    pack_upper_kernel<<<grid, 256, 0, s>>>(full, n, P + (int64_t)f * npack);
    if ((rc = check_cuda(ctx, cudaGetLastError(), "pack_upper_kernel launch"))) return rc;
  }
  std::vector<int> h(2 * nw);
  if ((rc = check_cuda(ctx, cudaMemcpyAsync(h.data(), info, sizeof(int) * 2 * nw, cudaMemcpyDeviceToHost, s),
                       "copy info")) ||
      (rc = check_cuda(ctx, cudaStreamSynchronize(s), "dielectric inversion")))
    return rc;
  for (int f = 0; f < nw; ++f)
    if (h[2 * f] != 0 || h[2 * f + 1] != 0)
      return set_error(ctx, SPX_EINVAL,
                       "dielectric matrix of frequency " + std::to_string(f) +
                           " is not positive definite (Cholesky info " + std::to_string(h[2 * f]) + ")");
  return SPX_OK;
}
