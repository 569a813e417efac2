// K4c, the batched complex FP64 GEMM on the DMMA path (spx_wfprod.cu), as used by
// other parts of the library: C(m, col) += alpha * sum_k A(m, k) * conj(B(col, k)).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "spx_common.cuh"

namespace spx {

struct ZgParams {
  // A_b(m, k) = A[b1*sA1 + b2*sA2 + m*lda + k], or with a_mcontig
  // A[b1*sA1 + b2*sA2 + m + k*lda] (a Fortran column-major panel)
  const double2* A;
  int64_t lda, sA1, sA2;
  int a_mcontig;
  // B_b(col, k) = B[b1*sB1 + b2*sB2 + colOff(col) + kOff(k)], col = n*ncin + c,
  // colOff = n*sBn + (cOff ? cOff[c] : c*sBc), kOff = kOff ? kOff[k] : k
  const double2* B;
  int64_t sB1, sB2, sBn, sBc;
  const int64_t* cOff;
  const int* kOff;
  // O_b(m, col) = O[b1*sO1 + b2*sO2 + m + n*sOn + c*sOc]
  double2* O;
  int64_t sO1, sO2, sOn, sOc;
  const double2* alpha;  // per b1, or null: alpha_v
  double2 alpha_v;
  int M, ncol, ncin, K, nb1;
  int K_last;  // K of the last batch when > 0 (split-K over batches)
  int mtiles, ntiles;
};

// Batch b = b1 + nb1 * b2 runs on grid.y; tiles of 64 x 64 on grid.x.
int launch_zgemm(spx_ctx* ctx, ZgParams prm, int nbatch, cudaStream_t s);

}  // namespace spx
