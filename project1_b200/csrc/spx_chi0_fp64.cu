// K1: complex FP64 band-pair accumulation on the DMMA tensor path (the drop-in).
//
// Computes, for every upper-triangle 64x64 tile (I, J) of the mixed-basis
// matrix and every frequency f,
//   chi_f(i, j) += sum_p M(p, i) * conj(M(p, j)) * w(p, f),      i <= j,
// which is the body loop of src/susceptibility.f:1182-1240 with the HILBERT
// NONE spectral_function (:1766-1789) folded in: the reference forms
// re/im(k) = cprod(k,i)*conjg(cprod(k,j)) for one (i,j) at a time and takes a
// ddot per frequency; here the same sum is a weighted complex Gram evaluated
// tile by tile, so every loaded band-pair value feeds 64 outputs instead of one.
//
// Layout and pipeline:
//   * one work item = (frequency, upper tile); persistent CTAs stride over items;
//   * warp 0 streams 16-pair slabs of the two 64-column panels of M
//     (p-contiguous columns, exactly the Fortran cprod layout) into shared
//     memory with 1-D bulk TMA copies, one per column, plus the 16 weights,
//     one stage ahead of the math; each warp releases a stage on an mbarrier
//     when it is done with it, and only warp 0 waits for that before refilling;
//   * four warps each own a 32x32 complex sub-tile and run
//     mma.sync m16n8kKI f64 on re/im planes: re += ar*(w br) + ai*(w bi),
//     im += ai*(w br) - ar*(w bi);
//   * shared rows are padded to 20 complex (320 B) so the 16-byte fragment
//     loads of a quarter-warp hit eight distinct bank groups;
//   * the epilogue adds the tile into the packed upper triangle
//     susceph(j*(j+1)/2 + i, f) (src/susceptibility.f:1210).
#include <cuda_runtime.h>

#include "spx_common.cuh"

namespace spx {

constexpr int F64_B = 64;                 // tile edge in complex rows / columns
constexpr int F64_KC = 16;                // band pairs per pipeline stage
constexpr int F64_ROW = F64_KC + 4;       // padded shared row, double2 units
constexpr int F64_ST = 2;                 // pipeline stages
constexpr int F64_WARPS = 4;              // each owns a 32x32 complex sub-tile
constexpr int F64_THREADS = 32 * F64_WARPS;

struct F64Params {
  const double2* M;
  int64_t ldc;
  int64_t P;
  int N;
  const double* W;
  int64_t ldw;
  int nw;
  double2* out;
  int64_t npack;
  int ntile;
  int64_t nitems;
  int* status;
  uint64_t timeout_ns;
};

struct __align__(16) F64Smem {
  double2 a[F64_ST][F64_B][F64_ROW];
  double2 b[F64_ST][F64_B][F64_ROW];
  double w[F64_ST][F64_KC];
  uint64_t full[F64_ST];
  uint64_t empty[F64_ST];  // every warp has finished with the stage
};

// Upper-triangle tile t -> (bi, bj), bi <= bj, column-major over the triangle.
__device__ __forceinline__ void decode_tile(int t, int* bi, int* bj) {
  int j = (int)((sqrtf(8.0f * (float)t + 1.0f) - 1.0f) * 0.5f);
  while (j * (j + 1) / 2 > t) --j;
  while ((j + 1) * (j + 2) / 2 <= t) ++j;
  *bj = j;
  *bi = t - j * (j + 1) / 2;
}

// D(16x8) += A(16xKI) * B(KIx8), f64. Fragment order: a[2q+h] = A(g+8h, t+4q),
// b[q] = B(t+4q, g), d[r] = D(g + 8*(r>>1), 2t + (r&1)); g = lane/4, t = lane%4.
template <int KI>
__device__ __forceinline__ void dmma(double (&d)[4], const double* a, const double* b);

template <>
__device__ __forceinline__ void dmma<4>(double (&d)[4], const double* a, const double* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(b[0]));
}
template <>
__device__ __forceinline__ void dmma<8>(double (&d)[4], const double* a, const double* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}
template <>
__device__ __forceinline__ void dmma<16>(double (&d)[4], const double* a, const double* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
      "{%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]),
        "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

// Issues the bulk copies of chunk `c` (item, p0) into stage `st`: one copy per
// panel column plus the weights. Called by all lanes of warp 0.
__device__ __forceinline__ void f64_issue(F64Smem& sm, const F64Params& prm, int st,
                                          int64_t item, int64_t p0, int lane) {
  const int f = (int)(item / prm.ntile);
  int bi, bj;
  decode_tile((int)(item % prm.ntile), &bi, &bj);
  const int i0 = bi * F64_B, j0 = bj * F64_B;
  const int ni = min(F64_B, prm.N - i0), nj = min(F64_B, prm.N - j0);
  const int len = (int)min((int64_t)F64_KC, prm.P - p0);
  const int wlen = (len + 1) & ~1;
  if (lane == 0) mbar_arrive_expect_tx(&sm.full[st], (uint32_t)((ni + nj) * len * 16 + wlen * 8));
  __syncwarp();
  for (int c = lane; c < ni; c += 32)
    bulk_g2s(&sm.a[st][c][0], prm.M + (int64_t)(i0 + c) * prm.ldc + p0, len * 16, &sm.full[st]);
  for (int c = lane; c < nj; c += 32)
    bulk_g2s(&sm.b[st][c][0], prm.M + (int64_t)(j0 + c) * prm.ldc + p0, len * 16, &sm.full[st]);
  if (lane == 0)
    bulk_g2s(&sm.w[st][0], prm.W + (int64_t)f * prm.ldw + p0, wlen * 8, &sm.full[st]);
}

template <int KI>
__global__ void __launch_bounds__(F64_THREADS, 2) chi0_fp64_kernel(F64Params prm) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  F64Smem& sm = *reinterpret_cast<F64Smem*>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  // zero the stages once so that masked lanes never read uninitialised bits
  for (int t = threadIdx.x; t < 2 * F64_ST * F64_B * F64_ROW; t += blockDim.x)
    reinterpret_cast<double2*>(smem_raw)[t] = make_double2(0.0, 0.0);
  if (threadIdx.x == 0) {
    for (int s = 0; s < F64_ST; ++s) {
      mbar_init(&sm.full[s], 1);
      mbar_init(&sm.empty[s], F64_WARPS);
    }
    fence_barrier_init();
  }
  __syncthreads();

  // The chunk sequence of this CTA: items blockIdx.x, +gridDim.x, ...; each item
  // is nchunk slabs of F64_KC band pairs. Chunk c lives in stage c % F64_ST.
  const int64_t nchunk = (prm.P + F64_KC - 1) / F64_KC;
  const int64_t my_items = prm.nitems > blockIdx.x
                               ? (prm.nitems - blockIdx.x + gridDim.x - 1) / gridDim.x
                               : 0;
  const int64_t total = my_items * nchunk;
  auto chunk_item = [&](int64_t c) { return blockIdx.x + (c / nchunk) * (int64_t)gridDim.x; };
  auto chunk_p0 = [&](int64_t c) { return (c % nchunk) * (int64_t)F64_KC; };
  // chunks [0, issued) have their copies issued (tracked by warp 0)
  int64_t issued = total < F64_ST - 1 ? total : (int64_t)(F64_ST - 1);
  if (warp == 0)
    for (int64_t c = 0; c < issued; ++c)
      f64_issue(sm, prm, (int)(c % F64_ST), chunk_item(c), chunk_p0(c), lane);

  const int wi = warp & 1, wj = warp >> 1;
  const int g = lane >> 2, t = lane & 3;
  constexpr int NQ = KI / 4;
  double accR[2][4][4], accI[2][4][4];
  bool failed = false;
  int64_t c = 0;
  for (; c < total; ++c) {
    const int st = (int)(c % F64_ST);
    const uint32_t ph = (uint32_t)((c / F64_ST) & 1);
    const int64_t p0 = chunk_p0(c);
    if (p0 == 0) {
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
          for (int r = 0; r < 4; ++r) accR[mt][nt][r] = accI[mt][nt][r] = 0.0;
    }
    // chunk c + F64_ST - 1 goes into the stage of chunk c - 1, once all four warps
    // have released that one (its release completes phase (c-1)/F64_ST of empty)
    if (warp == 0 && c + F64_ST - 1 < total) {
      const int64_t prev = c - 1;
      int ok = 1;
      if (prev >= 0 && lane == 0)
        ok = mbar_wait(&sm.empty[(int)(prev % F64_ST)], (uint32_t)((prev / F64_ST) & 1),
                       prm.timeout_ns, prm.status);
      if (!__shfl_sync(0xffffffffu, ok, 0)) {
        failed = true;
        break;
      }
      f64_issue(sm, prm, (int)((c + F64_ST - 1) % F64_ST), chunk_item(c + F64_ST - 1),
                chunk_p0(c + F64_ST - 1), lane);
      issued = c + F64_ST;
    }
    if (!mbar_wait(&sm.full[st], ph, prm.timeout_ns, prm.status)) {
      failed = true;
      break;
    }
    const int len = (int)min((int64_t)F64_KC, prm.P - p0);
#pragma unroll
    for (int ks = 0; ks < F64_KC / KI; ++ks) {
      double wq[NQ];
      bool valid[NQ];
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        const int p = ks * KI + t + 4 * q;
        valid[q] = p < len;
        wq[q] = valid[q] ? sm.w[st][p] : 0.0;
      }
      // one 16-row slice of A at a time keeps the live set small; B slices are
      // re-read from shared memory for the second slice
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        double ar[2 * NQ], ai[2 * NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const double2 v = sm.a[st][32 * wi + 16 * mt + g + 8 * h][ks * KI + t + 4 * q];
            ar[2 * q + h] = valid[q] ? v.x : 0.0;
            ai[2 * q + h] = valid[q] ? v.y : 0.0;
          }
        // two column slices at a time: the two MMAs that share an accumulator are
        // three independent MMAs apart, hiding the DMMA latency
#pragma unroll
        for (int np = 0; np < 2; ++np) {
          double br[2][NQ], bim[2][NQ], bneg[2][NQ];
#pragma unroll
          for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
              const double2 v = sm.b[st][32 * wj + 8 * (2 * np + h) + g][ks * KI + t + 4 * q];
              br[h][q] = wq[q] * v.x;
              bim[h][q] = wq[q] * v.y;
              bneg[h][q] = -bim[h][q];
            }
          dmma<KI>(accR[mt][2 * np], ar, br[0]);
          dmma<KI>(accR[mt][2 * np + 1], ar, br[1]);
          dmma<KI>(accI[mt][2 * np], ai, br[0]);
          dmma<KI>(accI[mt][2 * np + 1], ai, br[1]);
          dmma<KI>(accR[mt][2 * np], ai, bim[0]);
          dmma<KI>(accR[mt][2 * np + 1], ai, bim[1]);
          dmma<KI>(accI[mt][2 * np], ar, bneg[0]);
          dmma<KI>(accI[mt][2 * np + 1], ar, bneg[1]);
        }
      }
    }
    // this warp is done with stage st; only the issuing warp waits for all four
    __syncwarp();
    if (lane == 0) mbar_arrive(&sm.empty[st]);

    if (p0 + F64_KC >= prm.P) {
      // last slab of this item: add the tile into the packed upper triangle
      const int64_t item = chunk_item(c);
      const int f = (int)(item / prm.ntile);
      int bi, bj;
      decode_tile((int)(item % prm.ntile), &bi, &bj);
      double2* outf = prm.out + (int64_t)f * prm.npack;
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            const int i = bi * F64_B + 32 * wi + 16 * mt + g + 8 * (r >> 1);
            const int j = bj * F64_B + 32 * wj + 8 * nt + 2 * t + (r & 1);
            if (i <= j && j < prm.N) {
              double2* o = outf + (int64_t)j * (j + 1) / 2 + i;
              double2 v = *o;
              v.x += accR[mt][nt][r];
              v.y += accI[mt][nt][r];
              *o = v;
            }
          }
    }
  }
  if (failed && warp == 0) {
    // never leave with bulk copies still landing in this CTA's shared memory
    for (int64_t k = c; k < issued; ++k)
      mbar_drain(&sm.full[(int)(k % F64_ST)], (uint32_t)((k / F64_ST) & 1), prm.timeout_ns);
  }
}

// Enqueues K1 over one slab of band pairs. W holds the weights of exactly these
// pairs (leading dimension ldw, padding zeroed).
int launch_chi0_fp64(spx_ctx* ctx, const double2* M, int64_t ldc, int64_t P, int N,
                     const double* W, int64_t ldw, int nw, double2* out, cudaStream_t stream,
                     int ki) {
  if (P <= 0 || N <= 0 || nw <= 0) return SPX_OK;
  const int nblk = (N + F64_B - 1) / F64_B;
  F64Params prm;
  prm.M = M;
  prm.ldc = ldc;
  prm.P = P;
  prm.N = N;
  prm.W = W;
  prm.ldw = ldw;
  prm.nw = nw;
  prm.out = out;
  prm.npack = (int64_t)N * (N + 1) / 2;
  prm.ntile = nblk * (nblk + 1) / 2;
  prm.nitems = (int64_t)prm.ntile * nw;
  prm.status = ctx->d_status;
  prm.timeout_ns = (uint64_t)(ctx->opt.timeout_ms > 0 ? ctx->opt.timeout_ms : 4000) * 1000000ull;
  const size_t smem = sizeof(F64Smem);
  int grid = (int)std::min<int64_t>(prm.nitems, (int64_t)2 * ctx->num_sms);
  cudaError_t e;
  switch (ki) {
    case 4:
      cudaFuncSetAttribute(chi0_fp64_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem);
      chi0_fp64_kernel<4><<<grid, F64_THREADS, smem, stream>>>(prm);
      break;
    case 16:
      cudaFuncSetAttribute(chi0_fp64_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem);
      chi0_fp64_kernel<16><<<grid, F64_THREADS, smem, stream>>>(prm);
      break;
    default:
      cudaFuncSetAttribute(chi0_fp64_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem);
      chi0_fp64_kernel<8><<<grid, F64_THREADS, smem, stream>>>(prm);
      break;
  }
  e = cudaGetLastError();
  return check_cuda(ctx, e, "chi0_fp64_kernel launch");
}

}  // namespace spx

namespace spx {

// Launches K1 with explicit device resources instead of a context: used by the
// allocation-free entry point, whose status word and weights live in static
// device memory.
int launch_chi0_fp64_noctx(int num_sms, int* status, uint64_t timeout_ns, const double2* M,
                           int64_t ldc, int64_t P, int N, const double* W, int64_t ldw, int nw,
                           double2* out, cudaStream_t stream) {
  if (P <= 0 || N <= 0 || nw <= 0) return SPX_OK;
  const int nblk = (N + F64_B - 1) / F64_B;
  F64Params prm;
  prm.M = M;
  prm.ldc = ldc;
  prm.P = P;
  prm.N = N;
  prm.W = W;
  prm.ldw = ldw;
  prm.nw = nw;
  prm.out = out;
  prm.npack = (int64_t)N * (N + 1) / 2;
  prm.ntile = nblk * (nblk + 1) / 2;
  prm.nitems = (int64_t)prm.ntile * nw;
  prm.status = status;
  prm.timeout_ns = timeout_ns;
  const size_t smem = sizeof(F64Smem);
  if (cudaFuncSetAttribute(chi0_fp64_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return SPX_ECUDA;
  const int grid = (int)std::min<int64_t>(prm.nitems, (int64_t)2 * num_sms);
  chi0_fp64_kernel<8><<<grid, F64_THREADS, smem, stream>>>(prm);
  return cudaGetLastError() == cudaSuccess ? SPX_OK : SPX_ECUDA;
}

}  // namespace spx
