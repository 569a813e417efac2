// K6: FP64 frequency weights, spin factor, and the seeded input generator (K8).
#include <cuda_runtime.h>

#include "spx_common.cuh"
#include "spx_philox.h"
#include "spx_split.cuh"

namespace spx {

// HILBERT NONE weights of src/susceptibility.f:950-975,
//   wghtSr(p, f) = -2*rdum / ((frqh(f)/img)**2 + rdum**2) / nkpt / nsym1 * nkpts(k),
// rdum = ediff[p], frqh(f)/img = omega[f], nkpts(k)/nkpt/nsym1 = wscale[p]*scale_all.
// Always FP64: near-degenerate pairs (|rdum| ~ 1e-6 eV) keep full relative
// accuracy because rdum is taken as given, never recomputed from energies in a
// narrower type. Rows [P, ldw) of every column are zeroed.
__global__ void weights_kernel(int64_t P, int64_t ldw, const double* __restrict__ ediff,
                               const double* __restrict__ wscale, double scale_all, int nw,
                               const double* __restrict__ omega, double* __restrict__ w) {
  const int64_t total = ldw * nw;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = t % ldw;
    const int f = (int)(t / ldw);
    double v = 0.0;
    if (p < P) {
      const double s = (wscale ? wscale[p] : 1.0) * scale_all;
      v = hilbert_none_weight(ediff[p], omega[f], s);
    }
    w[t] = v;
  }
}

int launch_weights(spx_ctx* ctx, int64_t P, int64_t ldw, const double* ediff,
                   const double* wscale, double scale_all, int nw, const double* omega,
                   double* w, cudaStream_t stream) {
  const int64_t total = ldw * nw;
  if (total <= 0) return SPX_OK;
  int grid = (int)std::min<int64_t>((total + 255) / 256, (int64_t)ctx->num_sms * 16);
  weights_kernel<<<grid, 256, 0, stream>>>(P, ldw, ediff, wscale, scale_all, nw, omega, w);
  return check_cuda(ctx, cudaGetLastError(), "weights_kernel launch");
}

// suscepc(i, j, f) += S1 + i S2 and suscepc(j, i, f) += conj(S1) + i conj(S2) for the
// packed Hermitian sums S1 (weights wr) and S2 (weights wi) of element (i <= j): the
// non-Hermitian real-frequency polarisation of src/susceptibility.f:1229-1235 (one
// thread per packed element and frequency; each output element has one writer).
__global__ void suscepc_combine_kernel(int N, int nw, const double2* __restrict__ S1,
                                       const double2* __restrict__ S2, double2* __restrict__ out,
                                       int64_t ldo) {
  const int64_t npack = (int64_t)N * (N + 1) / 2;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < npack * nw;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int f = (int)(t / npack);
    const int64_t p = t - (int64_t)f * npack;
    int j = (int)((sqrt(8.0 * (double)p + 1.0) - 1.0) * 0.5);
    while ((int64_t)j * (j + 1) / 2 > p) --j;
    while ((int64_t)(j + 1) * (j + 2) / 2 <= p) ++j;
    const int i = (int)(p - (int64_t)j * (j + 1) / 2);
    const double2 a = S1[t], b = S2[t];
    double2* of = out + (int64_t)f * ldo * N;
    double2 v = of[(int64_t)j * ldo + i];
    v.x += a.x - b.y;
    v.y += a.y + b.x;
    of[(int64_t)j * ldo + i] = v;
    if (i != j) {
      double2 u = of[(int64_t)i * ldo + j];
      u.x += a.x + b.y;
      u.y += b.x - a.y;
      of[(int64_t)i * ldo + j] = u;
    }
  }
}

int launch_suscepc_combine(spx_ctx* ctx, int N, int nw, const double2* S1, const double2* S2,
                           double2* out, int64_t ldo, cudaStream_t stream) {
  const int64_t total = (int64_t)N * (N + 1) / 2 * nw;
  if (total <= 0) return SPX_OK;
  const int grid = (int)std::min<int64_t>((total + 255) / 256, (int64_t)ctx->num_sms * 16);
  suscepc_combine_kernel<<<grid, 256, 0, stream>>>(N, nw, S1, S2, out, ldo);
  return check_cuda(ctx, cudaGetLastError(), "suscepc_combine_kernel launch");
}

__global__ void scale_kernel(double* z, int64_t n2, double factor) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n2;
       t += (int64_t)gridDim.x * blockDim.x)
    z[t] *= factor;
}

int launch_scale(spx_ctx* ctx, double* z, int64_t n, double factor, cudaStream_t stream) {
  if (n <= 0) return SPX_OK;
  int grid = (int)std::min<int64_t>((2 * n + 255) / 256, (int64_t)ctx->num_sms * 16);
  scale_kernel<<<grid, 256, 0, stream>>>(z, 2 * n, factor);
  return check_cuda(ctx, cudaGetLastError(), "scale_kernel launch");
}

// out[t] = scale * normal(offset + t)
__global__ void gen_normal_kernel(uint64_t seed, uint32_t sid, int64_t offset, int64_t n,
                                  double scale, double* out) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x)
    out[t] = __dmul_rn(scale, normal_at(seed, sid, (uint64_t)(offset + t)));
}

// Complex matrix: element (p, c) re/im = stream elements 2*rows*(col0+c) + 2p + {0,1}.
// One thread per complex element; a Philox block yields exactly that pair.
// out[c*ld + p] = element (p0 + p, col0 + c) of a (rows_total x ...) stream matrix,
// p < rows: rows [p0, p0+rows) of its columns [col0, col0+cols).
__global__ void gen_cmatrix_kernel(uint64_t seed, uint32_t sid, int64_t rows_total, int64_t p0,
                                   int64_t rows, int64_t cols, int64_t ld, int64_t col0,
                                   double scale, double2* out) {
  const int64_t total = rows * cols;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = t / rows, p = t - c * rows;
    const uint64_t e = (uint64_t)(2 * rows_total * (col0 + c) + 2 * (p0 + p));
    double z0, z1;
    normal_pair(seed, sid, e >> 1, &z0, &z1);  // e is even: (z0, z1) = elements e, e+1
    out[c * ld + p] = make_double2(__dmul_rn(scale, z0), __dmul_rn(scale, z1));
  }
}

int launch_gen_normal(spx_ctx* ctx, uint64_t seed, uint32_t sid, int64_t offset, int64_t n,
                      double scale, double* out, cudaStream_t stream) {
  if (n <= 0) return SPX_OK;
  int grid = (int)std::min<int64_t>((n + 255) / 256, (int64_t)ctx->num_sms * 32);
  gen_normal_kernel<<<grid, 256, 0, stream>>>(seed, sid, offset, n, scale, out);
  return check_cuda(ctx, cudaGetLastError(), "gen_normal_kernel launch");
}

__global__ void abs_kernel(int64_t n, double* __restrict__ x) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x)
    x[t] = fabs(x[t]);
}

// x = |x| in place (the autotuners' probe energies: positive transition energies
// give one-signed imaginary-axis weights, as in the calls they tune for).
int launch_abs(spx_ctx* ctx, int64_t n, double* x, cudaStream_t stream) {
  if (n <= 0) return SPX_OK;
  int grid = (int)std::min<int64_t>((n + 255) / 256, (int64_t)ctx->num_sms * 32);
  abs_kernel<<<grid, 256, 0, stream>>>(n, x);
  return check_cuda(ctx, cudaGetLastError(), "abs_kernel launch");
}

int launch_gen_cmatrix(spx_ctx* ctx, uint64_t seed, uint32_t sid, int64_t rows, int64_t cols,
                       int64_t ld, int64_t col0, double scale, double* out,
                       cudaStream_t stream) {
  if (rows <= 0 || cols <= 0) return SPX_OK;
  int grid = (int)std::min<int64_t>((rows * cols + 255) / 256, (int64_t)ctx->num_sms * 32);
  gen_cmatrix_kernel<<<grid, 256, 0, stream>>>(seed, sid, rows, 0, rows, cols, ld, col0, scale,
                                               reinterpret_cast<double2*>(out));
  return check_cuda(ctx, cudaGetLastError(), "gen_cmatrix_kernel launch");
}

// Rows [p0, p0+rows) of the generated (rows_total x cols) matrix, into out (ld >= rows).
int launch_gen_cmatrix_rows(spx_ctx* ctx, uint64_t seed, uint32_t sid, int64_t rows_total,
                            int64_t p0, int64_t rows, int64_t cols, int64_t ld, double scale,
                            double2* out, cudaStream_t stream) {
  if (rows <= 0 || cols <= 0) return SPX_OK;
  int grid = (int)std::min<int64_t>((rows * cols + 255) / 256, (int64_t)ctx->num_sms * 32);
  gen_cmatrix_kernel<<<grid, 256, 0, stream>>>(seed, sid, rows_total, p0, rows, cols, ld, 0,
                                               scale, out);
  return check_cuda(ctx, cudaGetLastError(), "gen_cmatrix_kernel launch");
}

}  // namespace spx

// host generators (same arithmetic as the kernels above)
extern "C" void spx_gen_normal_host(uint64_t seed, uint32_t stream_id, int64_t offset,
                                    int64_t n, double scale, double* out) {
  for (int64_t t = 0; t < n; ++t) out[t] = scale * spx::normal_at(seed, stream_id, offset + t);
}

extern "C" void spx_gen_cmatrix_host(uint64_t seed, uint32_t stream_id, int64_t rows,
                                     int64_t cols, int64_t ld, int64_t col0, double scale,
                                     double* out) {
  for (int64_t c = 0; c < cols; ++c)
    for (int64_t p = 0; p < rows; ++p) {
      const uint64_t e = (uint64_t)(2 * rows * (col0 + c) + 2 * p);
      double z0, z1;
      spx::normal_pair(seed, stream_id, e >> 1, &z0, &z1);
      out[2 * (c * ld + p)] = scale * z0;
      out[2 * (c * ld + p) + 1] = scale * z1;
    }
}

namespace spx {

// Weights launch with explicit resources (no context): see launch_chi0_fp64_noctx.
int launch_weights_noctx(int num_sms, int64_t P, int64_t ldw, const double* ediff,
                         const double* wscale, double scale_all, int nw, const double* omega,
                         double* w, cudaStream_t stream) {
  const int64_t total = ldw * nw;
  if (total <= 0) return SPX_OK;
  const int grid = (int)std::min<int64_t>((total + 255) / 256, (int64_t)num_sms * 16);
  weights_kernel<<<grid, 256, 0, stream>>>(P, ldw, ediff, wscale, scale_all, nw, omega, w);
  return cudaGetLastError() == cudaSuccess ? SPX_OK : SPX_ECUDA;
}


// Effective imaginary-axis weights of the Hilbert-mesh path:
//   w(p, f) = scale * sum_s [wtetra(p, s) > thr] wtetra(p, s) * wghtSr(s, f)
// (the spectral function on the mesh, src/susceptibility.f:996-1078, followed by the
// Hilbert weights of src/hilbert.f:193-300). One thread per pair, the weight table
// in shared memory, frequencies in groups of 8 accumulators.
__global__ void hilbert_weights_kernel(int64_t P, int S, int nw, const double* __restrict__ wt,
                                       int64_t ldt, const double* __restrict__ ws, double thr,
                                       double scale, double* __restrict__ W, int64_t ldw) {
  extern __shared__ double sws[];
  for (int i = threadIdx.x; i < S * nw; i += blockDim.x) sws[i] = ws[i];
  __syncthreads();
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < P;
       p += (int64_t)gridDim.x * blockDim.x) {
    for (int f0 = 0; f0 < nw; f0 += 8) {
      double acc[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) acc[k] = 0.0;
      for (int s = 0; s < S; ++s) {
        const double v = wt[p + ldt * s];
        if (!(v > thr)) continue;
#pragma unroll
        for (int k = 0; k < 8; ++k)
          if (f0 + k < nw) acc[k] = fma(v, sws[s + S * (f0 + k)], acc[k]);
      }
#pragma unroll
      for (int k = 0; k < 8; ++k)
        if (f0 + k < nw) W[p + ldw * (f0 + k)] = scale * acc[k];
    }
  }
}

int launch_hilbert_weights(spx_ctx* ctx, int64_t P, int S, int nw, const double* wt, int64_t ldt,
                           const double* ws, double thr, double scale, double* W, int64_t ldw,
                           cudaStream_t stream) {
  if (P <= 0 || nw <= 0) return SPX_OK;
  const size_t smem = sizeof(double) * (size_t)S * nw;
  if (smem > 200 * 1024)
    return set_error(ctx, SPX_EINVAL, "nfrqs * nw too large (at most 25600 weights)");
  cudaFuncSetAttribute(hilbert_weights_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const int grid = (int)std::min<int64_t>((P + 255) / 256, (int64_t)ctx->num_sms * 8);
  hilbert_weights_kernel<<<grid, 256, smem, stream>>>(P, S, nw, wt, ldt, ws, thr, scale, W, ldw);
  return check_cuda(ctx, cudaGetLastError(), "hilbert_weights_kernel launch");
}


// One bounded wait on an mbarrier phase that nothing completes: the failure path of
// every device-side wait in this library (status word set, kernel returns).
__global__ void wait_selftest_kernel(int* status, uint64_t timeout_ns) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  mbar_wait(&bar, 0u, timeout_ns, status);  // no thread ever arrives
  __syncthreads();
}

}  // namespace spx

extern "C" int spx_selftest_wait_dev(spx_ctx* ctx, int32_t timeout_ms) {
  if (!ctx) return SPX_EINVAL;
  if (timeout_ms <= 0 || timeout_ms > 10000) return spx::set_error(ctx, SPX_EINVAL, "timeout_ms must be 1..10000");
  cudaSetDevice(ctx->device);
  spx::wait_selftest_kernel<<<1, 32, 0, ctx->stream>>>(ctx->d_status, (uint64_t)timeout_ms * 1000000ull);
  int rc = spx::check_cuda(ctx, cudaGetLastError(), "wait_selftest_kernel launch");
  if (rc) return rc;
  return spx::collect_status(ctx, ctx->stream, "selftest_wait");
}
