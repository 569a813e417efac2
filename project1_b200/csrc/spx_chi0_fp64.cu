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
//     (p-contiguous columns, exactly the Fortran cprod layout) into shared memory
//     with 2-D TMA boxes of 8 pairs x 64 columns (128-byte rows, SWIZZLE_128B, so
//     fragment loads of eight rows hit eight different bank groups), three stages
//     ahead (five copy instructions per stage); pairs and columns past the slab's
//     end arrive as zeros, and a diagonal tile loads its one panel once;
//   * four warps each own a 32x32 complex sub-tile and run
//     mma.sync m16n8k8 f64 on re/im parts: re += ar*(w br) + ai*(w bi),
//     im += ai*(w br) - ar*(w bi); each warp releases a stage on an mbarrier;
//   * the epilogue adds the tile into the packed upper triangle
//     susceph(j*(j+1)/2 + i, f) (src/susceptibility.f:1210).
#include <cuda.h>
#include <cuda_runtime.h>

#include "spx_common.cuh"
#include "spx_tcgen05.cuh"

namespace spx {

constexpr int F64_B = 64;                 // tile edge in complex rows / columns
constexpr int F64_KC = 16;                // band pairs per pipeline stage
constexpr int F64_KBOX = 8;               // pairs per TMA box: one 128-byte swizzled row
constexpr int F64_ST = 3;                 // pipeline stages
constexpr int F64_WARPS = 4;              // each owns a 32x32 complex sub-tile
constexpr int F64_THREADS = 32 * F64_WARPS;

struct F64Params {
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

// one panel half: 64 columns x 8 pairs, row r's 16-byte chunk c stored at c ^ (r & 7)
typedef double2 F64Box[F64_B][F64_KBOX];

struct __align__(1024) F64Smem {
  F64Box a[F64_ST][2];
  F64Box b[F64_ST][2];
  double w[F64_ST][F64_KC];
  uint64_t full[F64_ST];
  uint64_t empty[F64_ST];  // every compute warp has finished with the stage
};

// Upper-triangle tile t -> (bi, bj), bi <= bj, column-major over the triangle.
__device__ __forceinline__ void decode_tile(int t, int* bi, int* bj) {
  int j = (int)((sqrtf(8.0f * (float)t + 1.0f) - 1.0f) * 0.5f);
  while (j * (j + 1) / 2 > t) --j;
  while ((j + 1) * (j + 2) / 2 <= t) ++j;
  *bj = j;
  *bi = t - j * (j + 1) / 2;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
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

__global__ void __launch_bounds__(F64_THREADS, 2)
    chi0_fp64_kernel(const __grid_constant__ CUtensorMap mapM, F64Params prm) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  F64Smem& sm = *reinterpret_cast<F64Smem*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                            ~(uintptr_t)1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
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

  // chunk c's copies (one thread): 2 or 4 boxes of M and the 16 weights
  auto issue = [&](int64_t c) {
    const int st = (int)(c % F64_ST);
    const int64_t item = chunk_item(c), p0 = chunk_p0(c);
    const int f = (int)(item / prm.ntile);
    int bi, bj;
    decode_tile((int)(item % prm.ntile), &bi, &bj);
    const bool same = bi == bj;
    mbar_arrive_expect_tx(&sm.full[st], (uint32_t)((same ? 2 : 4) * sizeof(F64Box) + F64_KC * 8));
    const int x = (int)(2 * p0);
    tma_load_2d(&sm.a[st][0][0][0], &mapM, x, bi * F64_B, &sm.full[st]);
    tma_load_2d(&sm.a[st][1][0][0], &mapM, x + 2 * F64_KBOX, bi * F64_B, &sm.full[st]);
    if (!same) {
      tma_load_2d(&sm.b[st][0][0][0], &mapM, x, bj * F64_B, &sm.full[st]);
      tma_load_2d(&sm.b[st][1][0][0], &mapM, x + 2 * F64_KBOX, bj * F64_B, &sm.full[st]);
    }
    bulk_g2s(&sm.w[st][0], prm.W + (int64_t)f * prm.ldw + p0, F64_KC * 8, &sm.full[st]);
  };
  // chunks [0, issued) have their copies issued (tracked by warp 0, lane 0)
  int64_t issued = total < F64_ST - 1 ? total : (int64_t)(F64_ST - 1);
  if (warp == 0 && lane == 0)
    for (int64_t c = 0; c < issued; ++c) issue(c);

  // ---------------- compute warps ----------------
  const int wi = warp & 1, wj = warp >> 1;
  const int g = lane >> 2, t = lane & 3;
  double accR[2][4][4], accI[2][4][4];
  bool failed = false;
  int64_t c = 0;
  for (; c < total; ++c) {
    const int st = (int)(c % F64_ST);
    const uint32_t ph = (uint32_t)((c / F64_ST) & 1);
    const int64_t item = chunk_item(c), p0 = chunk_p0(c);
    int bi, bj;
    decode_tile((int)(item % prm.ntile), &bi, &bj);
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
      if (lane == 0) {
        if (prev >= 0)
          ok = mbar_wait(&sm.empty[(int)(prev % F64_ST)], (uint32_t)((prev / F64_ST) & 1),
                         prm.timeout_ns, prm.status);
        if (ok) issue(c + F64_ST - 1);
      }
      if (!__shfl_sync(0xffffffffu, ok, 0)) {
        failed = true;
        break;
      }
      issued = c + F64_ST;
    }
    if (!mbar_wait(&sm.full[st], ph, prm.timeout_ns, prm.status)) {
      failed = true;
      break;
    }
    const F64Box* Ab = sm.a[st];
    const F64Box* Bb = bi == bj ? sm.a[st] : sm.b[st];
#pragma unroll
    for (int ks = 0; ks < F64_KC / F64_KBOX; ++ks) {
      const double w0 = sm.w[st][ks * F64_KBOX + t], w1 = sm.w[st][ks * F64_KBOX + t + 4];
      // one 16-row slice of A at a time keeps the live set small
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        double ar[4], ai[4];
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int r = 32 * wi + 16 * mt + g + 8 * h;
            const double2 v = Ab[ks][r][(t + 4 * q) ^ (r & 7)];
            ar[2 * q + h] = v.x;
            ai[2 * q + h] = v.y;
          }
        // two column slices at a time: the two MMAs that share an accumulator are
        // three independent MMAs apart, hiding the DMMA latency
#pragma unroll
        for (int np = 0; np < 2; ++np) {
          double br[2][2], bim[2][2], bneg[2][2];
#pragma unroll
          for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int q = 0; q < 2; ++q) {
              const int r = 32 * wj + 8 * (2 * np + h) + g;
              const double2 v = Bb[ks][r][(t + 4 * q) ^ (r & 7)];
              const double wq = q ? w1 : w0;
              br[h][q] = wq * v.x;
              bim[h][q] = wq * v.y;
              bneg[h][q] = -bim[h][q];
            }
          dmma<8>(accR[mt][2 * np], ar, br[0]);
          dmma<8>(accR[mt][2 * np + 1], ar, br[1]);
          dmma<8>(accI[mt][2 * np], ai, br[0]);
          dmma<8>(accI[mt][2 * np + 1], ai, br[1]);
          dmma<8>(accR[mt][2 * np], ai, bim[0]);
          dmma<8>(accR[mt][2 * np + 1], ai, bim[1]);
          dmma<8>(accI[mt][2 * np], ar, bneg[0]);
          dmma<8>(accI[mt][2 * np + 1], ar, bneg[1]);
        }
      }
    }
    // this warp is done with stage st
    __syncwarp();
    if (lane == 0) mbar_arrive(&sm.empty[st]);

    if (p0 + F64_KC >= prm.P) {
      // last slab of this item: add the tile into the packed upper triangle
      const int f = (int)(item / prm.ntile);
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
  if (failed && warp == 0 && lane == 0) {
    // never leave with copies still landing in this CTA's shared memory
    for (int64_t k = c; k < issued; ++k)
      mbar_drain(&sm.full[(int)(k % F64_ST)], (uint32_t)((k / F64_ST) & 1), prm.timeout_ns);
  }
}

// Tensor map of M as a 2-D FP64 array: pairs (re, im interleaved) contiguous,
// columns ldc complex apart; boxes of 8 pairs x 64 columns, SWIZZLE_128B.
static int f64_map(CUtensorMap* map, const double2* M, int64_t ldc, int64_t P, int N) {
  const uint64_t dims[2] = {(uint64_t)(2 * P), (uint64_t)N};
  const uint64_t strides[1] = {(uint64_t)ldc * 16};
  const uint32_t box[2] = {2 * F64_KBOX, F64_B};
  return encode_tmap(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, M, dims, strides, box,
                     CU_TENSOR_MAP_SWIZZLE_128B);
}

static int f64_launch(int num_sms, const double2* M, int64_t ldc, int64_t P, int N, const double* W,
                      int64_t ldw, int nw, double2* out, int* status, uint64_t timeout_ns,
                      cudaStream_t stream) {
  const int nblk = (N + F64_B - 1) / F64_B;
  F64Params prm;
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
  CUtensorMap map;
  const int e = f64_map(&map, M, ldc, P, N);
  if (e) return e;
  const size_t smem = sizeof(F64Smem) + 1024;
  if (cudaFuncSetAttribute(chi0_fp64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return -2;
  const int grid = (int)std::min<int64_t>(prm.nitems, (int64_t)2 * num_sms);
  chi0_fp64_kernel<<<grid, F64_THREADS, smem, stream>>>(map, prm);
  return 0;
}

// Enqueues K1 over one slab of band pairs. W holds the weights of exactly these
// pairs (leading dimension ldw, a multiple of 16, padding zeroed).
int launch_chi0_fp64(spx_ctx* ctx, const double2* M, int64_t ldc, int64_t P, int N,
                     const double* W, int64_t ldw, int nw, double2* out, cudaStream_t stream,
                     int ki) {
  (void)ki;
  if (P <= 0 || N <= 0 || nw <= 0) return SPX_OK;
  const uint64_t timeout_ns =
      (uint64_t)(ctx->opt.timeout_ms > 0 ? ctx->opt.timeout_ms : 4000) * 1000000ull;
  const int e = f64_launch(ctx->num_sms, M, ldc, P, N, W, ldw, nw, out, ctx->d_status, timeout_ns, stream);
  if (e) return set_error(ctx, SPX_ECUDA, "chi0_fp64_kernel: tensor map or attribute failed (" +
                                              std::to_string(e) + ")");
  return check_cuda(ctx, cudaGetLastError(), "chi0_fp64_kernel launch");
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
  if (f64_launch(num_sms, M, ldc, P, N, W, ldw, nw, out, status, timeout_ns, stream)) return SPX_ECUDA;
  return cudaGetLastError() == cudaSuccess ? SPX_OK : SPX_ECUDA;
}

}  // namespace spx

namespace spx {

// ---------------------------------------------------------------------------
// K1r: the -DINV build (MCOMPLEX_dp = real_dp, src/cppmacro.h:53-64), where
// re(k) = cprod(k,i) * cprod(k,j) (src/susceptibility.f:1197) and chi is real:
//   chi_f(i, j) += sum_p M(p, i) M(p, j) w(p, f),  i <= j,
// on the same pipeline as K1 with one 2-D TMA box of 16 pairs x 64 columns per
// panel and stage (128-byte rows, SWIZZLE_128B: pair k of row r sits in 16-byte
// chunk (k/2) ^ (r & 7)), and one DMMA per 8 x 8 real product.
typedef double F64RBox[F64_B][F64_KC];

struct __align__(1024) F64RSmem {
  F64RBox a[F64_ST];
  F64RBox b[F64_ST];
  double w[F64_ST][F64_KC];
  uint64_t full[F64_ST];
  uint64_t empty[F64_ST];
};

__device__ __forceinline__ double f64r_at(const F64RBox& box, int r, int k) {
  return box[r][(((k >> 1) ^ (r & 7)) << 1) | (k & 1)];
}

__global__ void __launch_bounds__(F64_THREADS, 2)
    chi0_fp64_real_kernel(const __grid_constant__ CUtensorMap mapM, F64Params prm, double* outr) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  F64RSmem& sm = *reinterpret_cast<F64RSmem*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                              ~(uintptr_t)1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < F64_ST; ++s) {
      mbar_init(&sm.full[s], 1);
      mbar_init(&sm.empty[s], F64_WARPS);
    }
    fence_barrier_init();
  }
  __syncthreads();
  const int64_t nchunk = (prm.P + F64_KC - 1) / F64_KC;
  const int64_t my_items = prm.nitems > blockIdx.x
                               ? (prm.nitems - blockIdx.x + gridDim.x - 1) / gridDim.x
                               : 0;
  const int64_t total = my_items * nchunk;
  auto chunk_item = [&](int64_t c) { return blockIdx.x + (c / nchunk) * (int64_t)gridDim.x; };
  auto chunk_p0 = [&](int64_t c) { return (c % nchunk) * (int64_t)F64_KC; };
  auto issue = [&](int64_t c) {
    const int st = (int)(c % F64_ST);
    const int64_t item = chunk_item(c), p0 = chunk_p0(c);
    const int f = (int)(item / prm.ntile);
    int bi, bj;
    decode_tile((int)(item % prm.ntile), &bi, &bj);
    const bool same = bi == bj;
    mbar_arrive_expect_tx(&sm.full[st], (uint32_t)((same ? 1 : 2) * sizeof(F64RBox) + F64_KC * 8));
    tma_load_2d(&sm.a[st][0][0], &mapM, (int)p0, bi * F64_B, &sm.full[st]);
    if (!same) tma_load_2d(&sm.b[st][0][0], &mapM, (int)p0, bj * F64_B, &sm.full[st]);
    bulk_g2s(&sm.w[st][0], prm.W + (int64_t)f * prm.ldw + p0, F64_KC * 8, &sm.full[st]);
  };
  int64_t issued = total < F64_ST - 1 ? total : (int64_t)(F64_ST - 1);
  if (warp == 0 && lane == 0)
    for (int64_t c = 0; c < issued; ++c) issue(c);

  const int wi = warp & 1, wj = warp >> 1;
  const int g = lane >> 2, t = lane & 3;
  double acc[2][4][4];
  bool failed = false;
  int64_t c = 0;
  for (; c < total; ++c) {
    const int st = (int)(c % F64_ST);
    const uint32_t ph = (uint32_t)((c / F64_ST) & 1);
    const int64_t item = chunk_item(c), p0 = chunk_p0(c);
    int bi, bj;
    decode_tile((int)(item % prm.ntile), &bi, &bj);
    if (p0 == 0) {
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
          for (int r = 0; r < 4; ++r) acc[mt][nt][r] = 0.0;
    }
    if (warp == 0 && c + F64_ST - 1 < total) {
      const int64_t prev = c - 1;
      int ok = 1;
      if (lane == 0) {
        if (prev >= 0)
          ok = mbar_wait(&sm.empty[(int)(prev % F64_ST)], (uint32_t)((prev / F64_ST) & 1),
                         prm.timeout_ns, prm.status);
        if (ok) issue(c + F64_ST - 1);
      }
      if (!__shfl_sync(0xffffffffu, ok, 0)) {
        failed = true;
        break;
      }
      issued = c + F64_ST;
    }
    if (!mbar_wait(&sm.full[st], ph, prm.timeout_ns, prm.status)) {
      failed = true;
      break;
    }
    const F64RBox& A = sm.a[st];
    const F64RBox& B = bi == bj ? sm.a[st] : sm.b[st];
#pragma unroll
    for (int ks = 0; ks < F64_KC / 8; ++ks) {
      const double w0 = sm.w[st][8 * ks + t], w1 = sm.w[st][8 * ks + t + 4];
      double bq[4][2];
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const int r = 32 * wj + 8 * nt + g;
        bq[nt][0] = w0 * f64r_at(B, r, 8 * ks + t);
        bq[nt][1] = w1 * f64r_at(B, r, 8 * ks + t + 4);
      }
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        double a[4];
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
          for (int h = 0; h < 2; ++h)
            a[2 * q + h] = f64r_at(A, 32 * wi + 16 * mt + g + 8 * h, 8 * ks + t + 4 * q);
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) dmma<8>(acc[mt][nt], a, bq[nt]);
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&sm.empty[st]);
    if (p0 + F64_KC >= prm.P) {
      const int f = (int)(item / prm.ntile);
      double* of = outr + (int64_t)f * prm.npack;
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            const int i = bi * F64_B + 32 * wi + 16 * mt + g + 8 * (r >> 1);
            const int j = bj * F64_B + 32 * wj + 8 * nt + 2 * t + (r & 1);
            if (i <= j && j < prm.N) of[(int64_t)j * (j + 1) / 2 + i] += acc[mt][nt][r];
          }
    }
  }
  if (failed && warp == 0 && lane == 0) {
    for (int64_t k = c; k < issued; ++k)
      mbar_drain(&sm.full[(int)(k % F64_ST)], (uint32_t)((k / F64_ST) & 1), prm.timeout_ns);
  }
}

// Enqueues K1r over one slab of real band-pair products M (ldc, N).
int launch_chi0_fp64_real(spx_ctx* ctx, const double* M, int64_t ldc, int64_t P, int N,
                          const double* W, int64_t ldw, int nw, double* out, cudaStream_t stream) {
  if (P <= 0 || N <= 0 || nw <= 0) return SPX_OK;
  const int nblk = (N + F64_B - 1) / F64_B;
  F64Params prm;
  prm.P = P;
  prm.N = N;
  prm.W = W;
  prm.ldw = ldw;
  prm.nw = nw;
  prm.out = nullptr;
  prm.npack = (int64_t)N * (N + 1) / 2;
  prm.ntile = nblk * (nblk + 1) / 2;
  prm.nitems = (int64_t)prm.ntile * nw;
  prm.status = ctx->d_status;
  prm.timeout_ns = (uint64_t)(ctx->opt.timeout_ms > 0 ? ctx->opt.timeout_ms : 4000) * 1000000ull;
  CUtensorMap map;
  const uint64_t dims[2] = {(uint64_t)P, (uint64_t)N};
  const uint64_t strides[1] = {(uint64_t)ldc * 8};
  const uint32_t box[2] = {F64_KC, F64_B};
  const int e = encode_tmap(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, M, dims, strides, box,
                            CU_TENSOR_MAP_SWIZZLE_128B);
  if (e) return set_error(ctx, SPX_ECUDA, "chi0_fp64_real_kernel: tensor map (" + std::to_string(e) + ")");
  const size_t smem = sizeof(F64RSmem) + 1024;
  cudaFuncSetAttribute(chi0_fp64_real_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const int grid = (int)std::min<int64_t>(prm.nitems, (int64_t)2 * ctx->num_sms);
  chi0_fp64_real_kernel<<<grid, F64_THREADS, smem, stream>>>(map, prm, out);
  return check_cuda(ctx, cudaGetLastError(), "chi0_fp64_real_kernel launch");
}

// FP64 tensor-pipe peak: every warp issues back-to-back m16n8k8 DMMAs on register
// operands into eight independent accumulators (no memory traffic in the loop),
// so the rate is the DMMA pipe's own. The sums go to `sink` so nothing is elided.
__global__ void __launch_bounds__(128) dmma_peak_kernel(int iters, double* sink) {
  const int lane = threadIdx.x & 31;
  double a[4], b[2];
#pragma unroll
  for (int k = 0; k < 4; ++k) a[k] = 1.0 + 1e-3 * (lane + k);
  b[0] = 0.5 - 1e-3 * lane;
  b[1] = 0.25 + 1e-3 * lane;
  double d[8][4];
#pragma unroll
  for (int k = 0; k < 8; ++k)
#pragma unroll
    for (int r = 0; r < 4; ++r) d[k][r] = 0.0;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int k = 0; k < 8; ++k) dmma<8>(d[k], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 8; ++k)
#pragma unroll
    for (int r = 0; r < 4; ++r) s += d[k][r];
  sink[blockIdx.x * (int64_t)blockDim.x + threadIdx.x] = s;
}

}  // namespace spx

// Measured FP64 tensor (DMMA) peak of the context's device in TFLOP/s (2 flops
// per MAC), timed with CUDA events on the context stream: one warm-up launch, then
// one launch of 4 CTAs x 4 warps per SM. No counterpart in the reference.
extern "C" int spx_measure_dmma_peak(spx_ctx* ctx, double* tflops) {
  if (!ctx || !tflops) return SPX_EINVAL;
  cudaSetDevice(ctx->device);
  const int blocks = 4 * ctx->num_sms, threads = 128, iters = 20000;
  int rc = spx::ensure_workspace(ctx, sizeof(double) * (size_t)blocks * threads);
  if (rc) return rc;
  double* sink = reinterpret_cast<double*>(ctx->ws);
  cudaEvent_t e0, e1;
  if ((rc = spx::check_cuda(ctx, cudaEventCreate(&e0), "event")) ||
      (rc = spx::check_cuda(ctx, cudaEventCreate(&e1), "event")))
    return rc;
  spx::dmma_peak_kernel<<<blocks, threads, 0, ctx->stream>>>(iters / 10, sink);
  cudaEventRecord(e0, ctx->stream);
  spx::dmma_peak_kernel<<<blocks, threads, 0, ctx->stream>>>(iters, sink);
  cudaEventRecord(e1, ctx->stream);
  rc = spx::check_cuda(ctx, cudaGetLastError(), "dmma_peak_kernel launch");
  if (!rc) rc = spx::check_cuda(ctx, cudaEventSynchronize(e1), "dmma_peak_kernel");
  float ms = 0.f;
  if (!rc) rc = spx::check_cuda(ctx, cudaEventElapsedTime(&ms, e0, e1), "event time");
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  const double macs = 16.0 * 8 * 8 * 8 * (double)iters * (blocks * threads / 32);
  *tflops = 2.0 * macs / (ms * 1e-3) / 1e12;
  return SPX_OK;
}
