// Dielectric matrix and its inverse in FP64 (src/correlation.f:614-636, :703-745).
//
// For every imaginary frequency the reference turns the packed polarisation into
//   eps_ij = delta_ij - sqrt(v_i) chi_ij sqrt(v_j)          (p_diagmatdiag, p_plusdiag)
// with v the Coulomb eigenvalues of the basis (the Coulomb-eigenbasis transform has
// made v diagonal), and inverts it as a packed Hermitian matrix (LAPACK zpptrf/zpptri
// on one process, ScaLAPACK with MPI). On the imaginary axis chi is negative
// semi-definite, so eps = 1 + (positive semi-definite) is positive definite. At
// Gamma the 3x3 head becomes 1 - 4 pi head and the wings -sqrt(4 pi) sqrt(v_i) wing.
//
// The inverse is computed here, for all frequencies at once, by the block sweep
// (Gauss-Jordan elimination without pivoting, which is stable for Hermitian positive
// definite matrices): for each 64-column pivot block k with P = inv(A_kk),
//   A_ij -= A_ik P A_kj,  A_ik <- A_ik P,  A_kj <- P A_kj,  A_kk <- -P   (i, j not in k),
// and after the last block A holds -inv(A). The pivot block is inverted by the same
// sweep one column at a time in shared memory; its pivots are the squares of the
// Cholesky pivots of A, so a pivot <= 0 marks a matrix that is not positive definite,
// reported with its frequency as zpptrf's info would be. The rank-64 updates run on
// the complex FP64 DMMA GEMM (K4c).
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "spx_common.cuh"
#include "spx_zgemm.h"

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

// packed(ij) = factor * full(i, j), i <= j, for every frequency (grid.y).
__global__ void pack_upper_kernel(const double2* __restrict__ full, int n, double factor,
                                  double2* __restrict__ packed) {
  const int64_t npack = (int64_t)n * (n + 1) / 2;
  const double2* fw = full + (int64_t)blockIdx.y * n * n;
  double2* pw = packed + (int64_t)blockIdx.y * npack;
  for (int64_t ij = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; ij < npack;
       ij += (int64_t)gridDim.x * blockDim.x) {
    int j = (int)((sqrt(8.0 * (double)ij + 1.0) - 1.0) * 0.5);
    while ((int64_t)j * (j + 1) / 2 > ij) --j;
    while ((int64_t)(j + 1) * (j + 2) / 2 <= ij) ++j;
    const int i = (int)(ij - (int64_t)j * (j + 1) / 2);
    const double2 v = fw[i + (int64_t)n * j];
    pw[ij] = make_double2(factor * v.x, factor * v.y);
  }
}

constexpr int DI_B = 64;  // pivot block of the sweep

// For every frequency (grid.y): CpT[j][t] = A(j, kb + t) for all rows j (the pivot
// block's column panel, stored row by row), and Pb[t][u] = A(kb + t, kb + u).
__global__ void sweep_extract_kernel(const double2* __restrict__ A, int n, int kb, int bk,
                                     double2* __restrict__ CpT, double2* __restrict__ Pb) {
  const double2* Aw = A + (int64_t)blockIdx.y * n * n;
  double2* Cw = CpT + (int64_t)blockIdx.y * n * DI_B;
  double2* Pw = Pb + (int64_t)blockIdx.y * DI_B * DI_B;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)n * bk;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int t = (int)(e / n), j = (int)(e - (int64_t)t * n);
    const double2 v = Aw[(int64_t)(kb + t) * n + j];
    Cw[(int64_t)j * DI_B + t] = v;
    if (j >= kb && j < kb + bk) Pw[(j - kb) * DI_B + t] = v;
  }
}

// In place: Pb <- inv(Pb) for the bk x bk Hermitian positive-definite block of every
// frequency (one CTA each), by the sweep of its columns in shared memory. A pivot
// that is not positive records (block row + 1) in info[frequency].
__global__ void __launch_bounds__(256) sweep_block_inverse_kernel(double2* __restrict__ Pb, int bk,
                                                                  int kb, int* __restrict__ info) {
  extern __shared__ double2 m[];              // [DI_B][DI_B + 1]
  __shared__ double2 col[DI_B], row[DI_B];
  __shared__ double pinv;
  constexpr int LD = DI_B + 1;
  double2* Pw = Pb + (int64_t)blockIdx.x * DI_B * DI_B;
  for (int e = threadIdx.x; e < bk * bk; e += blockDim.x) m[(e / bk) * LD + e % bk] = Pw[(e / bk) * DI_B + e % bk];
  __syncthreads();
  for (int p = 0; p < bk; ++p) {
    if (threadIdx.x == 0) {
      const double piv = m[p * LD + p].x;
      if (!(piv > 0.0)) {
        if (info[blockIdx.x] == 0) info[blockIdx.x] = kb + p + 1;
        pinv = 0.0;
      } else {
        pinv = 1.0 / piv;
      }
    }
    for (int i = threadIdx.x; i < bk; i += blockDim.x) {
      col[i] = m[i * LD + p];
      row[i] = m[p * LD + i];
    }
    __syncthreads();
    const double d = pinv;
    for (int e = threadIdx.x; e < bk * bk; e += blockDim.x) {
      const int i = e / bk, j = e % bk;
      const double2 ci = col[i], rj = row[j];
      double2 v;
      if (i == p && j == p) {
        v = make_double2(-d, 0.0);
      } else if (j == p) {
        v = make_double2(ci.x * d, ci.y * d);
      } else if (i == p) {
        v = make_double2(rj.x * d, rj.y * d);
      } else {
        // m_ij - m_ip m_pj / m_pp
        const double re = ci.x * rj.x - ci.y * rj.y, im = ci.x * rj.y + ci.y * rj.x;
        v = m[i * LD + j];
        v.x -= re * d;
        v.y -= im * d;
      }
      m[i * LD + j] = v;
    }
    __syncthreads();
  }
  // the sweep of every column leaves -inv
  for (int e = threadIdx.x; e < bk * bk; e += blockDim.x) {
    const double2 v = m[(e / bk) * LD + e % bk];
    Pw[(e / bk) * DI_B + e % bk] = make_double2(-v.x, -v.y);
  }
}

// After the trailing update: A(i, kb+t) = U(i, t), A(kb+t, i) = conj U(i, t) for rows i
// outside the block, and A(kb+t, kb+u) = -P(t, u).
__global__ void sweep_panels_kernel(double2* __restrict__ A, int n, int kb, int bk,
                                    const double2* __restrict__ U, const double2* __restrict__ Pb) {
  double2* Aw = A + (int64_t)blockIdx.y * n * n;
  const double2* Uw = U + (int64_t)blockIdx.y * n * DI_B;
  const double2* Pw = Pb + (int64_t)blockIdx.y * DI_B * DI_B;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)n * bk;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int t = (int)(e / n), i = (int)(e - (int64_t)t * n);
    if (i >= kb && i < kb + bk) {
      const double2 v = Pw[(i - kb) * DI_B + t];   // P(i - kb, t)
      Aw[(int64_t)(kb + t) * n + i] = make_double2(-v.x, -v.y);
    } else {
      const double2 u = Uw[(int64_t)t * n + i];
      Aw[(int64_t)(kb + t) * n + i] = u;
      Aw[(int64_t)i * n + (kb + t)] = make_double2(u.x, -u.y);
    }
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

void dielec_release(spx_ctx* ctx) { ctx->dn = nullptr; }

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
  // scratch: sqrt(v), infos, and for the inversion the full matrices of every
  // frequency, the pivot blocks, the column panels and their products
  size_t need = align_up(sizeof(double) * n, 256) + align_up(sizeof(int) * nw, 256);
  const size_t full_b = align_up(sizeof(double2) * (size_t)n * n * nw, 256);
  const size_t pan_b = align_up(sizeof(double2) * (size_t)n * DI_B * nw, 256);
  const size_t blk_b = align_up(sizeof(double2) * (size_t)DI_B * DI_B * nw, 256);
  if (invert) need += full_b + 2 * pan_b + blk_b;
  if ((rc = ensure_workspace(ctx, need + 1024))) return rc;
  char* b = (char*)ctx->ws;
  double* sq = (double*)b;
  b += align_up(sizeof(double) * n, 256);
  int* info = (int*)b;
  b += align_up(sizeof(int) * nw, 256);
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
  b += full_b;
  double2* CpT = reinterpret_cast<double2*>(b);
  b += pan_b;
  double2* U = reinterpret_cast<double2*>(b);
  b += pan_b;
  double2* Pb = reinterpret_cast<double2*>(b);
  if ((rc = check_cuda(ctx, cudaMemsetAsync(info, 0, sizeof(int) * nw, s), "zero info"))) return rc;
  for (int f = 0; f < nw; ++f) {
    dielec_unpack_kernel<<<grid, 256, 0, s>>>(P + (int64_t)f * npack, sq, n, full + (int64_t)f * n * n);
    if ((rc = check_cuda(ctx, cudaGetLastError(), "dielec_unpack_kernel launch"))) return rc;
  }
  const size_t bsmem = sizeof(double2) * DI_B * (DI_B + 1);
  cudaFuncSetAttribute(sweep_block_inverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bsmem);
  const dim3 pgrid((unsigned)std::min<int64_t>(((int64_t)n * DI_B + 255) / 256, 4096), (unsigned)nw);
  for (int kb = 0; kb < n; kb += DI_B) {
    const int bk = std::min(DI_B, n - kb);
    sweep_extract_kernel<<<pgrid, 256, 0, s>>>(full, n, kb, bk, CpT, Pb);
    sweep_block_inverse_kernel<<<nw, 256, bsmem, s>>>(Pb, bk, kb, info);
    if ((rc = check_cuda(ctx, cudaGetLastError(), "sweep pivot block")) ||
        (rc = check_cuda(ctx, cudaMemsetAsync(U, 0, pan_b, s), "zero panel")))
      return rc;
    // U = Cp P: U(i, c) = sum_t Cp(i, t) conj(P(c, t))   (P Hermitian)
    ZgParams g{};
    g.A = CpT;
    g.lda = DI_B;
    g.sA1 = (int64_t)n * DI_B;
    g.B = Pb;
    g.sB1 = (int64_t)DI_B * DI_B;
    g.sBc = DI_B;
    g.O = U;
    g.sO1 = (int64_t)n * DI_B;
    g.sOc = n;
    g.alpha_v = make_double2(1.0, 0.0);
    g.M = n;
    g.ncol = bk;
    g.ncin = bk;
    g.K = bk;
    g.nb1 = nw;
    if ((rc = launch_zgemm(ctx, g, nw, s))) return rc;
    // A(i, j) -= sum_t U(i, t) conj(Cp(j, t))   (= U_i A_kj, A Hermitian)
    ZgParams h{};
    h.A = U;
    h.a_mcontig = 1;
    h.lda = n;
    h.sA1 = (int64_t)n * DI_B;
    h.B = CpT;
    h.sB1 = (int64_t)n * DI_B;
    h.sBc = DI_B;
    h.O = full;
    h.sO1 = (int64_t)n * n;
    h.sOc = n;
    h.alpha_v = make_double2(-1.0, 0.0);
    h.M = n;
    h.ncol = n;
    h.ncin = n;
    h.K = bk;
    h.nb1 = nw;
    if ((rc = launch_zgemm(ctx, h, nw, s))) return rc;
    sweep_panels_kernel<<<pgrid, 256, 0, s>>>(full, n, kb, bk, U, Pb);
    if ((rc = check_cuda(ctx, cudaGetLastError(), "sweep panels"))) return rc;
  }
  // the sweep leaves -inv(eps)
  pack_upper_kernel<<<dim3(grid, nw), 256, 0, s>>>(full, n, -1.0, P);
  if ((rc = check_cuda(ctx, cudaGetLastError(), "pack_upper_kernel launch"))) return rc;
  std::vector<int> hinfo(nw);
  if ((rc = check_cuda(ctx, cudaMemcpyAsync(hinfo.data(), info, sizeof(int) * nw, cudaMemcpyDeviceToHost, s),
                       "copy info")) ||
      (rc = check_cuda(ctx, cudaStreamSynchronize(s), "dielectric inversion")))
    return rc;
  for (int f = 0; f < nw; ++f)
    if (hinfo[f] != 0)
      return set_error(ctx, SPX_EINVAL,
                       "dielectric matrix of frequency " + std::to_string(f) +
                           " is not positive definite (pivot " + std::to_string(hinfo[f]) + ")");
  return SPX_OK;
}
