// K2: split-precision band-pair accumulation on the 5th-generation tensor cores.
//
// The sum chi_f(i, j) = sum_p M(p, i) conj(M(p, j)) w(p, f) (src/susceptibility.f:
// 1182-1240 with the HILBERT NONE weights of :950-975) is evaluated as an exact
// integer contraction of 8-bit digit slices (an Ozaki-type error-free split):
//
//   x = s/127 * (d0 + d1/256 + d2/256^2 + d3/256^3 + r/256^3),  |d0| <= 127,
//   d1..d3 in [-128, 127], |r| <= 1/2,
//
// with s the largest |Re|, |Im| of the column over a slab of band pairs. The
// digits are the balanced base-256 bytes of one integer, round(x*127/s * 2^24),
// so a single FP64 -> int32 rounding per value produces all of them. The
// unweighted operand A = M keeps 3 slices, the weighted operand B = w_f M keeps 4
// (its column scale is s_j * max_p |w(p,f)|, so its relative resolution must
// absorb the spread of the weights). Digit products with t + u <= 3 are summed on
// tcgen05.mma kind::i8 into four int32 accumulators in tensor memory, one per
// order g = t + u, which is exact: no rounding happens inside the contraction.
// Once per slab of 32768 pairs (the int32 headroom: 3 * 128^2 * 32768 < 2^31) the
// epilogue forms ((D0*256 + D1)*256 + D2)*256 + D3 exactly in int64 and adds
// s_i s_j wmax_f / (127^2 2^24) times it to the FP64 output. The weights and
// the scale factors stay FP64 throughout; near-degenerate pairs therefore keep
// their FP64 weights.
//
// Error (per element, relative to sqrt|chi_ii chi_jj|): slicing of A (half a unit of
// its third digit, 2^-17/127 of the column scale per value) <= 2^-17/127 times the
// column crest factor max|x| sqrt(P)/||x||, slicing of B <= 2^-25/127 times the
// weighted crest factor, dropped orders g >= 4 below that; see the accuracy tests.
//
// Tile layout: a 64 x 64 complex tile is a 128 x 128 real-stacked product: A rows
// are (Re M_i | Im M_i) for 64 mixed-basis functions, B rows likewise for the
// 64 columns j; D[(c,i)][(c',j)] holds the four real products, combined in the
// epilogue as re = D[re_i][re_j] + D[im_i][im_j], im = D[im_i][re_j] - D[re_i][im_j]
// (the two halves live in different TMEM lane quarters and meet in shared memory).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "spx_common.cuh"
#include "spx_tcgen05.cuh"

namespace spx {

constexpr int SP_TILE = 64;            // complex rows / columns per tile
constexpr int SP_ROWS = 128;           // real-stacked rows per tile (re | im)
constexpr int SP_KB = 64;              // band pairs (bytes) per pipeline stage: two MMA K steps
constexpr int SP_KSTEP = 32;           // int8 MMA K
constexpr int SP_NKS = SP_KB / SP_KSTEP;
constexpr int SP_SA = 3;               // digit slices of the unweighted operand
constexpr int SP_SB = 4;               // digit slices of the weighted operand
constexpr int SP_ST = 3;               // pipeline stages
constexpr int SP_SLAB = 32768;         // band pairs per exact int32 accumulation
constexpr int SP_THREADS = 192;        // warp 0 TMA, warp 1 MMA + TMEM, warps 2-5 epilogue
constexpr int SP_PLANE = SP_ROWS * SP_KB;  // bytes of one slice of one stage
constexpr int SP_TMEM_COLS = 512;      // 4 orders x 128 columns of int32


// idesc for kind::i8: D s32 (bits 4-5 = 2), A/B signed int8 (bits 7-9, 10-12 = 1),
// K-major A and B, N = 128 (bits 17-22 = N/8), M = 128 (bits 24-28 = M/16).
constexpr uint32_t SP_IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(SP_ROWS / 8) << 17) |
                              ((uint32_t)(SP_ROWS / 16) << 24);

struct __align__(1024) SplitSmem {
  uint8_t a[SP_ST][SP_SA][SP_PLANE];
  uint8_t b[SP_ST][SP_SB][SP_PLANE];
  long long xchg[2][SP_TILE][33];      // epilogue exchange of the (row, Im col) halves
  uint64_t full[SP_ST];
  uint64_t empty[SP_ST];
  uint64_t tfull, tempty, xfull, xfree, mdone;
  uint32_t tmem_base;
};

struct SplitParams {
  int N;
  int ntile;
  int nw;
  int nitems;
  int nk;                 // pipeline stages per item (pairs of the slab / 32)
  const double* sA;       // column scales of the slab
  const double* wmax;     // max |w(p, f)| of the slab
  double* out;            // packed complex output, as doubles
  int64_t npack;
  int* status;
  uint64_t timeout_ns;
};

__device__ __forceinline__ void split_decode_tile(int t, int* bi, int* bj) {
  int j = (int)((sqrtf(8.0f * (float)t + 1.0f) - 1.0f) * 0.5f);
  while (j * (j + 1) / 2 > t) --j;
  while ((j + 1) * (j + 2) / 2 <= t) ++j;
  *bj = j;
  *bi = t - j * (j + 1) / 2;
}

// T = ((D0*256 + D1)*256 + D2)*256 + D3 for 32 columns starting at `taddr`, where
// D_g sits 128 g columns further: the exact integer value of the slab's sum.
__device__ __forceinline__ void load_orders(uint32_t taddr, long long (&T)[32]) {
  int32_t r[32];
  tmem_ld32(taddr, r);
  tmem_wait_ld();
#pragma unroll
  for (int k = 0; k < 32; ++k) T[k] = r[k];
#pragma unroll
  for (int g = 1; g < 4; ++g) {
    tmem_ld32(taddr + (uint32_t)(g * 128), r);
    tmem_wait_ld();
#pragma unroll
    for (int k = 0; k < 32; ++k) T[k] = T[k] * 256 + r[k];
  }
}

__global__ void __launch_bounds__(SP_THREADS, 1)
    split_gram_kernel(const __grid_constant__ CUtensorMap mapA,
                      const __grid_constant__ CUtensorMap mapB, SplitParams prm) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  SplitSmem& sm = *reinterpret_cast<SplitSmem*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < SP_ST; ++s) {
      mbar_init(&sm.full[s], 1);
      mbar_init(&sm.empty[s], 1);
    }
    mbar_init(&sm.tfull, 1);
    mbar_init(&sm.tempty, 4);
    mbar_init(&sm.xfull, 4);
    mbar_init(&sm.xfree, 4);
    mbar_init(&sm.mdone, 1);
    fence_barrier_init();
  }
  if (warp == 1) tmem_alloc(&sm.tmem_base, SP_TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sm.tmem_base;

  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      int st = 0;
      uint32_t ph = 0;
      bool issued[SP_ST];
      uint32_t last_ph[SP_ST];
      for (int s = 0; s < SP_ST; ++s) issued[s] = false, last_ph[s] = 0;
      bool ok = true;
      for (int item = blockIdx.x; item < prm.nitems && ok; item += gridDim.x) {
        const int f = item / prm.ntile;
        int bi, bj;
        split_decode_tile(item % prm.ntile, &bi, &bj);
        for (int ks = 0; ks < prm.nk; ++ks) {
          if (!mbar_wait(&sm.empty[st], ph ^ 1u, prm.timeout_ns, prm.status)) {
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(&sm.full[st], (uint32_t)((SP_SA + SP_SB) * SP_PLANE));
          tma_load_4d(&sm.a[st][0][0], &mapA, 0, bi * SP_ROWS, ks, 0, &sm.full[st]);
          tma_load_4d(&sm.b[st][0][0], &mapB, 0, bj * SP_ROWS, ks, f * SP_SB, &sm.full[st]);
          issued[st] = true;
          last_ph[st] = ph;
          if (++st == SP_ST) st = 0, ph ^= 1u;
        }
      }
      // copies still landing must finish before this CTA's shared memory goes away
      for (int s = 0; s < SP_ST; ++s)
        if (issued[s]) mbar_drain(&sm.full[s], last_ph[s], prm.timeout_ns);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      int st = 0;
      uint32_t ph = 0;
      int j = 0;
      bool committed = false;
      for (int item = blockIdx.x; item < prm.nitems; item += gridDim.x, ++j) {
        // accumulators free (first item: immediately)
        if (!mbar_wait(&sm.tempty, (uint32_t)(j & 1) ^ 1u, prm.timeout_ns, prm.status)) break;
        tc_fence_after();
        bool ok = true;
        for (int ks = 0; ks < prm.nk; ++ks) {
          if (!mbar_wait(&sm.full[st], ph, prm.timeout_ns, prm.status)) {
            ok = false;
            break;
          }
          tc_fence_after();
          // order g = t + u lives at TMEM columns [128 g, 128 g + 128); the first
          // product of every order in a slab (t == 0, first K step) overwrites it
#pragma unroll
          for (int kk = 0; kk < SP_NKS; ++kk) {
            uint64_t da[SP_SA], db[SP_SB];
#pragma unroll
            for (int t = 0; t < SP_SA; ++t) da[t] = desc_sw64(&sm.a[st][t][0]) + (uint64_t)(kk * 2);
#pragma unroll
            for (int u = 0; u < SP_SB; ++u) db[u] = desc_sw64(&sm.b[st][u][0]) + (uint64_t)(kk * 2);
            const uint32_t k0 = (ks > 0 || kk > 0);
            mma_i8<1>(tmem + 0 * 128, da[0], db[0], SP_IDESC, k0);
            mma_i8<2>(tmem + 1 * 128, da[0], db[1], SP_IDESC, k0);
            mma_i8<2>(tmem + 2 * 128, da[0], db[2], SP_IDESC, k0);
            mma_i8<3>(tmem + 3 * 128, da[0], db[3], SP_IDESC, k0);
            mma_i8<1>(tmem + 1 * 128, da[1], db[0], SP_IDESC, 1u);
            mma_i8<2>(tmem + 2 * 128, da[1], db[1], SP_IDESC, 1u);
            mma_i8<3>(tmem + 3 * 128, da[1], db[2], SP_IDESC, 1u);
            mma_i8<1>(tmem + 2 * 128, da[2], db[0], SP_IDESC, 1u);
            mma_i8<3>(tmem + 3 * 128, da[2], db[1], SP_IDESC, 1u);
          }
          tc_commit(&sm.empty[st]);  // stage free once these MMAs have read it
          committed = true;
          if (++st == SP_ST) st = 0, ph ^= 1u;
        }
        if (!ok) break;
        tc_commit(&sm.tfull);  // accumulators complete
      }
      // every MMA issued by this thread must retire before TMEM is released: a
      // commit issued now arrives once all of them are done
      if (committed) {
        tc_commit(&sm.mdone);
        mbar_drain(&sm.mdone, 0u, prm.timeout_ns);
      }
    }
  } else {
    // ---------------- epilogue: 4 warps, one TMEM lane quarter each ----------------
    const int q = warp & 3;                 // lane quarter
    const bool is_re = q < 2;               // lanes 0-63: Re rows, 64-127: Im rows
    const int ii = (q & 1) * 32 + lane;     // complex row within the tile
    const uint32_t tl = tmem + ((uint32_t)(32 * q) << 16);
    int j = 0;
    uint32_t xseq = 0;
    for (int item = blockIdx.x; item < prm.nitems; item += gridDim.x, ++j) {
      if (!mbar_wait_idle(&sm.tfull, (uint32_t)(j & 1), prm.timeout_ns, prm.status)) break;
      tc_fence_after();
      const int f = item / prm.ntile;
      int bi, bj;
      split_decode_tile(item % prm.ntile, &bi, &bj);
      const int gi = bi * SP_TILE + ii;
      const double si = gi < prm.N ? prm.sA[gi] : 0.0;
      const double fac =
          si * prm.wmax[f] * (1.0 / (127.0 * 127.0 * 16777216.0));
      double* outf = prm.out + 2 * (int64_t)f * prm.npack;
      bool ok = true;
      for (int js = 0; js < 2 && ok; ++js, ++xseq) {
        long long tre[32], tim[32];  // T[row][Re col], T[row][Im col] for 32 columns j
        load_orders(tl + (uint32_t)(js * 32), tre);
        load_orders(tl + (uint32_t)(64 + js * 32), tim);
        // exchange the Im-column halves between the Re and Im rows of each i
        if (!mbar_wait(&sm.xfree, (xseq & 1u) ^ 1u, prm.timeout_ns, prm.status)) {
          ok = false;
          break;
        }
#pragma unroll
        for (int k = 0; k < 32; ++k) sm.xchg[is_re ? 0 : 1][ii][k] = tim[k];
        __syncwarp();
        if (lane == 0) mbar_arrive(&sm.xfull);
        if (!mbar_wait(&sm.xfull, xseq & 1u, prm.timeout_ns, prm.status)) {
          ok = false;
          break;
        }
        // Re rows: chi_re = T[re_i][re_j] + T[im_i][im_j]; Im rows: chi_im = T[im_i][re_j] - T[re_i][im_j]
#pragma unroll
        for (int k = 0; k < 32; ++k) {
          const int gj = bj * SP_TILE + js * 32 + k;
          const long long partner = sm.xchg[is_re ? 1 : 0][ii][k];
          const long long v = is_re ? tre[k] + partner : tre[k] - partner;
          if (gi <= gj && gj < prm.N) {
            // one add per element per launch: launches are ordered, so the sum is
            // deterministic, and the reduction needs no read round trip
            double* o = outf + 2 * ((int64_t)gj * (gj + 1) / 2 + gi) + (is_re ? 0 : 1);
            atomicAdd(o, fac * prm.sA[gj] * (double)v);
          }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&sm.xfree);
      }
      if (!ok) break;
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&sm.tempty);
    }
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1) tmem_dealloc(tmem, SP_TMEM_COLS);
}

// ---------------------------------------------------------------------------
// CTA-pair form: one tcgen05.mma.cta_group::2 (M = 256) covers two 64 x 64 complex
// tiles stacked in i. Each CTA of the cluster stages its own A tile (128 rows) and
// half of the shared B tile (64 rows: CTA 0 the Re rows, CTA 1 the Im rows of the
// 64 columns j); the leader CTA issues the MMAs, which read both CTAs' shared
// memory and write each CTA's own TMEM. Per SM and stage this moves 20 KB instead
// of 28 KB from L2 for the same tensor work. Every completion that crosses the
// pair is an explicit remote arrive or commit (no multicast).

constexpr int SP2_ST = 5;
constexpr int SP2_XC = 16;                      // columns per epilogue exchange
constexpr int SP2_BROWS = SP_ROWS / 2;          // B rows staged per CTA
constexpr int SP2_BPLANE = SP2_BROWS * SP_KB;   // 2048 bytes
constexpr uint32_t SP2_IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(SP_ROWS / 8) << 17) |
                               ((uint32_t)(2 * SP_ROWS / 16) << 24);   // M = 256, N = 128

struct __align__(1024) Split2Smem {
  uint8_t a[SP2_ST][SP_SA][SP_PLANE];
  uint8_t b[SP2_ST][SP_SB][SP2_BPLANE];
  long long xchg[2][SP_TILE][SP2_XC + 1];
  uint64_t full[SP2_ST];   // leader: both CTAs' bytes of a stage have landed
  uint64_t empty[SP2_ST];  // each CTA: the MMAs have read the stage
  uint64_t tfull;          // each CTA: accumulators ready
  uint64_t tempty;         // leader: both CTAs' epilogues have drained TMEM (8 warps)
  uint64_t xfull, xfree, mdone;
  uint32_t tmem_base;
};

// Pair tile t -> (bI, bJ): i-blocks of 128 (two 64-blocks), j-blocks of 64, with
// 2 bI <= bJ; column-major over bJ.
__device__ __forceinline__ void pair_decode_tile(int t, int* bI, int* bJ) {
  int j = 0, c = 0;
  while (c + j / 2 + 1 <= t) {
    c += j / 2 + 1;
    ++j;
  }
  *bJ = j;
  *bI = t - c;
}

// T = ((D0*256 + D1)*256 + D2)*256 + D3 for 16 columns starting at `taddr`.
__device__ __forceinline__ void load_orders16(uint32_t taddr, long long (&T)[16]) {
  int32_t r[16];
  tmem_ld16(taddr, r);
  tmem_wait_ld();
#pragma unroll
  for (int k = 0; k < 16; ++k) T[k] = r[k];
#pragma unroll
  for (int g = 1; g < 4; ++g) {
    tmem_ld16(taddr + (uint32_t)(g * 128), r);
    tmem_wait_ld();
#pragma unroll
    for (int k = 0; k < 16; ++k) T[k] = T[k] * 256 + r[k];
  }
}

__global__ void __launch_bounds__(SP_THREADS, 1)
    split_gram2_kernel(const __grid_constant__ CUtensorMap mapA,
                       const __grid_constant__ CUtensorMap mapB, SplitParams prm) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  Split2Smem& sm = *reinterpret_cast<Split2Smem*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_ctarank();
  const int cid = (int)cluster_id_x(), ncl = (int)nclusters_x();

  if (threadIdx.x == 0) {
    for (int s = 0; s < SP2_ST; ++s) {
      mbar_init(&sm.full[s], 1);
      mbar_init(&sm.empty[s], 1);
    }
    mbar_init(&sm.tfull, 1);
    mbar_init(&sm.tempty, 8);
    mbar_init(&sm.xfull, 4);
    mbar_init(&sm.xfree, 4);
    mbar_init(&sm.mdone, 1);
    fence_barrier_init();
  }
  if (warp == 1) tmem_alloc2(&sm.tmem_base, SP_TMEM_COLS);
  tc_fence_before();
  cluster_sync();  // both CTAs' barriers initialised and TMEM allocated
  tc_fence_after();
  const uint32_t tmem = sm.tmem_base;

  if (warp == 0) {
    // ---------------- TMA producer (both CTAs) ----------------
    if (lane == 0) {
      int st = 0;
      uint32_t ph = 0;
      bool issued[SP2_ST];
      uint32_t last_ph[SP2_ST];
      for (int q = 0; q < SP2_ST; ++q) issued[q] = false, last_ph[q] = 0;
      bool ok = true;
      // Cursor over this cluster's (item, stage) sequence; it advances by increments
      // and decodes a tile only when it enters a new item.
      struct Cursor {
        int item, ks, ya, yb, zf;
      };
      auto enter = [&](Cursor& u) {
        int bI, bJ;
        pair_decode_tile(u.item % prm.ntile, &bI, &bJ);
        u.ya = (2 * bI + (int)rank) * SP_ROWS;
        u.yb = bJ * SP_ROWS + (int)rank * SP2_BROWS;
        u.zf = (u.item / prm.ntile) * SP_SB;
      };
      auto advance = [&](Cursor& u) {
        if (++u.ks == prm.nk) {
          u.ks = 0;
          u.item += ncl;
          if (u.item < prm.nitems) enter(u);
        }
      };
      Cursor ld{cid, 0, 0, 0, 0};
      if (cid < prm.nitems) enter(ld);
      while (ld.item < prm.nitems) {
        if (!mbar_wait(&sm.empty[st], ph ^ 1u, prm.timeout_ns, prm.status)) {
          ok = false;
          break;
        }
        const uint32_t lead_full = mapa_shared(smem_u32(&sm.full[st]), 0);
        if (rank == 0)
          mbar_arrive_expect_tx(&sm.full[st],
                                (uint32_t)(2 * (SP_SA * SP_PLANE + SP_SB * SP2_BPLANE)));
        tma_load_4d_pair(&sm.a[st][0][0], &mapA, 0, ld.ya, ld.ks, 0, lead_full);
        tma_load_4d_pair(&sm.b[st][0][0], &mapB, 0, ld.yb, ld.ks, ld.zf, lead_full);
        advance(ld);
        issued[st] = true;
        last_ph[st] = ph;
        if (++st == SP2_ST) st = 0, ph ^= 1u;
      }
      if (rank == 0) {
        // the leader's stage barriers count both CTAs' bytes
        for (int q = 0; q < SP2_ST; ++q)
          if (issued[q]) mbar_drain(&sm.full[q], last_ph[q], prm.timeout_ns);
      } else {
        // the peer cannot poll the leader's barrier: give its last copies a bounded
        // grace period to land (they complete in microseconds)
        const uint64_t t0 = global_ns();
        while (global_ns() - t0 < 200000ull) {
        }
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer (leader CTA only) ----------------
    if (rank == 0 && lane == 0) {
      int st = 0;
      uint32_t ph = 0;
      int j = 0;
      bool committed = false;
      const uint32_t peer_tfull = mapa_shared(smem_u32(&sm.tfull), 1);
      for (int item = cid; item < prm.nitems; item += ncl, ++j) {
        if (!mbar_wait(&sm.tempty, (uint32_t)(j & 1) ^ 1u, prm.timeout_ns, prm.status)) break;
        tc_fence_after();
        bool ok = true;
        for (int ks = 0; ks < prm.nk; ++ks) {
          if (!mbar_wait(&sm.full[st], ph, prm.timeout_ns, prm.status)) {
            ok = false;
            break;
          }
          tc_fence_after();
#pragma unroll
          for (int kk = 0; kk < SP_NKS; ++kk) {
            uint64_t da[SP_SA], db[SP_SB];
#pragma unroll
            for (int t = 0; t < SP_SA; ++t) da[t] = desc_sw64(&sm.a[st][t][0]) + (uint64_t)(kk * 2);
#pragma unroll
            for (int u = 0; u < SP_SB; ++u) db[u] = desc_sw64(&sm.b[st][u][0]) + (uint64_t)(kk * 2);
            const uint32_t k0 = (ks > 0 || kk > 0);
            mma2_i8<1>(tmem + 0 * 128, da[0], db[0], SP2_IDESC, k0);
            mma2_i8<2>(tmem + 1 * 128, da[0], db[1], SP2_IDESC, k0);
            mma2_i8<2>(tmem + 2 * 128, da[0], db[2], SP2_IDESC, k0);
            mma2_i8<3>(tmem + 3 * 128, da[0], db[3], SP2_IDESC, k0);
            mma2_i8<1>(tmem + 1 * 128, da[1], db[0], SP2_IDESC, 1u);
            mma2_i8<2>(tmem + 2 * 128, da[1], db[1], SP2_IDESC, 1u);
            mma2_i8<3>(tmem + 3 * 128, da[1], db[2], SP2_IDESC, 1u);
            mma2_i8<1>(tmem + 2 * 128, da[2], db[0], SP2_IDESC, 1u);
            mma2_i8<3>(tmem + 3 * 128, da[2], db[1], SP2_IDESC, 1u);
          }
          // the stage is free in both CTAs once these MMAs have read it
          tc_commit2(smem_u32(&sm.empty[st]));
          tc_commit2(mapa_shared(smem_u32(&sm.empty[st]), 1));
          committed = true;
          if (++st == SP2_ST) st = 0, ph ^= 1u;
        }
        if (!ok) break;
        tc_commit2(smem_u32(&sm.tfull));
        tc_commit2(peer_tfull);
      }
      if (committed) {
        tc_commit2(smem_u32(&sm.mdone));
        mbar_drain(&sm.mdone, 0u, prm.timeout_ns);
      }
    }
  } else {
    // ---------------- epilogue (both CTAs): this CTA's 64 x 64 tile ----------------
    const int q = warp & 3;
    const bool is_re = q < 2;
    const int ii = (q & 1) * 32 + lane;
    const uint32_t tl = tmem + ((uint32_t)(32 * q) << 16);
    const uint32_t lead_tempty = mapa_shared(smem_u32(&sm.tempty), 0);
    int j = 0;
    uint32_t xseq = 0;
    for (int item = cid; item < prm.nitems; item += ncl, ++j) {
      if (!mbar_wait_idle(&sm.tfull, (uint32_t)(j & 1), prm.timeout_ns, prm.status)) break;
      tc_fence_after();
      const int f = item / prm.ntile;
      int bI, bJ;
      pair_decode_tile(item % prm.ntile, &bI, &bJ);
      const int bi = 2 * bI + (int)rank;
      bool ok = true;
      // a tile wholly below the diagonal or past N has nothing to store
      if (bi <= bJ && bi * SP_TILE < prm.N) {
        const int gi = bi * SP_TILE + ii;
        const double si = gi < prm.N ? prm.sA[gi] : 0.0;
        const double fac = si * prm.wmax[f] * (1.0 / (127.0 * 127.0 * 16777216.0));
        double* outf = prm.out + 2 * (int64_t)f * prm.npack;
        for (int js = 0; js < SP_TILE / SP2_XC && ok; ++js, ++xseq) {
          long long tre[SP2_XC], tim[SP2_XC];
          load_orders16(tl + (uint32_t)(js * SP2_XC), tre);
          load_orders16(tl + (uint32_t)(64 + js * SP2_XC), tim);
          if (!mbar_wait(&sm.xfree, (xseq & 1u) ^ 1u, prm.timeout_ns, prm.status)) {
            ok = false;
            break;
          }
#pragma unroll
          for (int k = 0; k < SP2_XC; ++k) sm.xchg[is_re ? 0 : 1][ii][k] = tim[k];
          __syncwarp();
          if (lane == 0) mbar_arrive(&sm.xfull);
          if (!mbar_wait(&sm.xfull, xseq & 1u, prm.timeout_ns, prm.status)) {
            ok = false;
            break;
          }
#pragma unroll
          for (int k = 0; k < SP2_XC; ++k) {
            const int gj = bJ * SP_TILE + js * SP2_XC + k;
            const long long partner = sm.xchg[is_re ? 1 : 0][ii][k];
            const long long v = is_re ? tre[k] + partner : tre[k] - partner;
            if (gi <= gj && gj < prm.N) {
              double* o = outf + 2 * ((int64_t)gj * (gj + 1) / 2 + gi) + (is_re ? 0 : 1);
              atomicAdd(o, fac * prm.sA[gj] * (double)v);
            }
          }
          __syncwarp();
          if (lane == 0) mbar_arrive(&sm.xfree);
        }
      }
      if (!ok) break;
      tc_fence_before();
      __syncwarp();
      if (lane == 0) {
        if (rank == 0) mbar_arrive(&sm.tempty);
        else mbar_arrive_cluster(lead_tempty);
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  cluster_sync();  // neither CTA leaves while the pair's MMAs may read its shared memory
  tc_fence_after();
  if (warp == 1) tmem_dealloc2(tmem, SP_TMEM_COLS);
}

// ---------------------------------------------------------------------------
// operand preparation

// Column scales of one slab: sA[i] = max_p max(|Re M(p,i)|, |Im M(p,i)|).
__global__ void split_colmax_kernel(const double2* __restrict__ M, int64_t ldc, int64_t p0,
                                    int len, double* __restrict__ sA) {
  const int i = blockIdx.x;
  const double2* col = M + (int64_t)i * ldc + p0;
  double m = 0.0;
  for (int p = threadIdx.x; p < len; p += blockDim.x) {
    const double2 v = col[p];
    m = fmax(m, fmax(fabs(v.x), fabs(v.y)));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) sA[i] = m;
  }
}

// wmax[f] = max_p |w(p, f)| over the slab.
__global__ void split_wmax_kernel(const double* __restrict__ W, int64_t ldw, int64_t p0, int len,
                                  double* __restrict__ wmax) {
  const int f = blockIdx.x;
  const double* wf = W + (int64_t)f * ldw + p0;
  double m = 0.0;
  for (int p = threadIdx.x; p < len; p += blockDim.x) m = fmax(m, fabs(wf[p]));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) wmax[f] = m;
  }
}

// Round-to-nearest integer of a*b (|a*b| < 2^31) through the FP64 magic constant
// 1.5*2^52: one fused multiply-add, the low word of the sum is the integer.
__device__ __forceinline__ uint32_t round_mul(double a, double b) {
  return (uint32_t)__double2loint(__fma_rn(a, b, 6755399441055744.0));
}

// Four values Y (two's complement words) -> their balanced base-256 digit planes.
// With U = Y + 0x808080, bytes 0..2 of U are the lower digits plus 128 and byte 3
// is the top digit (|top| <= 127 because |Y| <= 127 * 2^24). out[t] holds digit t
// (t = 0 most significant) of the four values, one per byte.
template <int S>
__device__ __forceinline__ void digit_planes(const uint32_t (&Y)[4], uint32_t (&out)[S]) {
  const uint32_t bias = S == 4 ? 0x00808080u : 0x00008080u;
  const uint32_t u0 = Y[0] + bias, u1 = Y[1] + bias, u2 = Y[2] + bias, u3 = Y[3] + bias;
  const uint32_t lo01 = __byte_perm(u0, u1, 0x5140), lo23 = __byte_perm(u2, u3, 0x5140);
  const uint32_t hi01 = __byte_perm(u0, u1, 0x7362), hi23 = __byte_perm(u2, u3, 0x7362);
  const uint32_t b0 = __byte_perm(lo01, lo23, 0x5410) ^ 0x80808080u;  // byte 0 of each
  const uint32_t b1 = __byte_perm(lo01, lo23, 0x7632) ^ 0x80808080u;  // byte 1
  const uint32_t b2 = __byte_perm(hi01, hi23, 0x5410);                // byte 2
  if constexpr (S == 4) {
    out[0] = __byte_perm(hi01, hi23, 0x7632);  // byte 3: top digit
    out[1] = b2 ^ 0x80808080u;
    out[2] = b1;
    out[3] = b0;
  } else {
    out[0] = b2;  // byte 2: top digit of a 3-digit value
    out[1] = b1;
    out[2] = b0;
  }
}

// One thread = one complex column i and 16 consecutive pairs of the slab. Digit
// planes are stored [plane][k-block of 64 pairs][row][64 bytes]; a warp holds 8
// consecutive columns x the four quarters of one k-block, so every store
// instruction writes 8 adjacent rows x 64 bytes = 512 contiguous bytes, and the TMA
// box (64 B, rows, 1 k-block, planes) lands as [plane][row][64 B] in shared memory.
// Rows are real-stacked: block b of 64 columns -> rows 128 b + {0..63 Re, 64..127 Im}.
__global__ void __launch_bounds__(128)
    split_quantize_kernel(const double2* __restrict__ M, int64_t ldc, int64_t p0, int len,
                          int nchunk, int N, int npad, int64_t R, int64_t Ps,
                          const double* __restrict__ W, int64_t ldw, int nw,
                          const double* __restrict__ sA, const double* __restrict__ wmax,
                          int8_t* __restrict__ A, int8_t* __restrict__ B) {
  const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (tid >= (int64_t)npad * nchunk) return;
  // tid -> (k-block, column group of 8, quarter of the k-block, column in group)
  const int ngroup = npad / 8;
  const int lane8 = (int)(tid & 7), quarter = (int)((tid >> 3) & 3);
  const int64_t rest = tid >> 5;
  const int i = (int)(rest % ngroup) * 8 + lane8;
  const int64_t kb = rest / ngroup;
  const int p = (int)(kb * SP_KB) + quarter * 16;
  const int64_t r_re = (int64_t)(i / SP_TILE) * SP_ROWS + (i % SP_TILE);
  const int64_t r_im = r_re + SP_TILE;
  const int64_t nkb = Ps / SP_KB;
  // byte offsets of (plane 0, k-block, row) for this thread's 16 pairs; planes are
  // nkb * R * 32 bytes apart
  const int64_t pstride = nkb * R * SP_KB;
  const int64_t a_re = (kb * R + r_re) * SP_KB + quarter * 16;
  const int64_t a_im = (kb * R + r_im) * SP_KB + quarter * 16;
  const int64_t b_re = a_re, b_im = a_im;
  double xr[16], xi[16];
  const bool col_ok = i < N;
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    double2 v = make_double2(0.0, 0.0);
    if (col_ok && p + k < len) v = M[(int64_t)i * ldc + p0 + p + k];
    xr[k] = v.x;
    xi[k] = v.y;
  }
  const double s = col_ok ? sA[i] : 0.0;
  // unweighted operand: 3 digits of round(x * 127/s * 2^16)
  {
    const double inv = s > 0.0 ? 127.0 * 65536.0 / s : 0.0;
    uint32_t wr[SP_SA][4], wi[SP_SA][4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      uint32_t yr[4], yi[4], pr[SP_SA], pi[SP_SA];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        yr[k] = round_mul(xr[4 * q + k], inv);
        yi[k] = round_mul(xi[4 * q + k], inv);
      }
      digit_planes<SP_SA>(yr, pr);
      digit_planes<SP_SA>(yi, pi);
#pragma unroll
      for (int t = 0; t < SP_SA; ++t) wr[t][q] = pr[t], wi[t][q] = pi[t];
    }
#pragma unroll
    for (int t = 0; t < SP_SA; ++t) {
      *reinterpret_cast<uint4*>(A + a_re + t * pstride) =
          make_uint4(wr[t][0], wr[t][1], wr[t][2], wr[t][3]);
      *reinterpret_cast<uint4*>(A + a_im + t * pstride) =
          make_uint4(wi[t][0], wi[t][1], wi[t][2], wi[t][3]);
    }
  }
  // weighted operand, one frequency at a time: 4 digits of round(x w 127/(wmax s) 2^24)
  for (int f = 0; f < nw; ++f) {
    const double wm = wmax[f];
    const double g = (s > 0.0 && wm > 0.0) ? 127.0 * 16777216.0 / (wm * s) : 0.0;
    const double* wf = W + (int64_t)f * ldw + p0 + p;
    uint32_t wr[SP_SB][4], wi[SP_SB][4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      uint32_t yr[4], yi[4], pr[SP_SB], pi[SP_SB];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int kk = 4 * q + k;
        const double wk = (p + kk < len) ? wf[kk] * g : 0.0;
        yr[k] = round_mul(xr[kk], wk);
        yi[k] = round_mul(xi[kk], wk);
      }
      digit_planes<SP_SB>(yr, pr);
      digit_planes<SP_SB>(yi, pi);
#pragma unroll
      for (int u = 0; u < SP_SB; ++u) wr[u][q] = pr[u], wi[u][q] = pi[u];
    }
#pragma unroll
    for (int u = 0; u < SP_SB; ++u) {
      const int64_t plane = (int64_t)f * SP_SB + u;
      *reinterpret_cast<uint4*>(B + b_re + plane * pstride) =
          make_uint4(wr[u][0], wr[u][1], wr[u][2], wr[u][3]);
      *reinterpret_cast<uint4*>(B + b_im + plane * pstride) =
          make_uint4(wi[u][0], wi[u][1], wi[u][2], wi[u][3]);
    }
  }
}

// ---------------------------------------------------------------------------
// host side

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn get_encode() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

int make_tmap_u8_3d(spx_ctx* ctx, CUtensorMap* map, const void* base, uint64_t d0, uint64_t d1,
                    uint64_t d2, uint64_t s1, uint64_t s2, uint32_t b0, uint32_t b1, uint32_t b2,
                    CUtensorMapSwizzle swz) {
  auto enc = get_encode();
  if (!enc) return set_error(ctx, SPX_ECUDA, "cuTensorMapEncodeTiled unavailable");
  cuuint64_t dims[3] = {d0, d1, d2};
  cuuint64_t strides[2] = {s1, s2};
  cuuint32_t box[3] = {b0, b1, b2};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(base), dims, strides,
                   box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, swz,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return set_error(ctx, SPX_ECUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
  return SPX_OK;
}

int make_tmap_u8_4d(spx_ctx* ctx, CUtensorMap* map, const void* base, const uint64_t dims[4],
                    const uint64_t strides[3], const uint32_t box[4], CUtensorMapSwizzle swz) {
  auto enc = get_encode();
  if (!enc) return set_error(ctx, SPX_ECUDA, "cuTensorMapEncodeTiled unavailable");
  cuuint64_t d[4] = {dims[0], dims[1], dims[2], dims[3]};
  cuuint64_t st[3] = {strides[0], strides[1], strides[2]};
  cuuint32_t b[4] = {box[0], box[1], box[2], box[3]};
  cuuint32_t es[4] = {1, 1, 1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 4, const_cast<void*>(base), d, st, b, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return set_error(ctx, SPX_ECUDA, "cuTensorMapEncodeTiled (4-D) failed: " + std::to_string((int)r));
  return SPX_OK;
}

struct SplitLayout {
  int64_t Ps, R;
  int nblk;
  size_t a_bytes, b_bytes, s_bytes, w_bytes;
};

// slab: band pairs per exact int32 slab, a multiple of SP_KB in [SP_KB, SP_SLAB]
static SplitLayout split_layout(int64_t P, int N, int nw, int slab = SP_SLAB) {
  SplitLayout L;
  L.Ps = std::min<int64_t>((int64_t)align_up((size_t)std::max<int64_t>(P, 1), SP_KB), slab);
  L.nblk = (N + SP_TILE - 1) / SP_TILE;
  // an even number of 64-blocks, so a CTA pair's second A tile always exists
  L.R = (int64_t)((L.nblk + 1) / 2 * 2) * SP_ROWS;
  L.a_bytes = align_up((size_t)SP_SA * L.R * L.Ps, 1024);
  L.b_bytes = align_up((size_t)SP_SB * nw * L.R * L.Ps, 1024);
  L.s_bytes = align_up(sizeof(double) * (size_t)std::max(N, 1), 256);
  L.w_bytes = align_up(sizeof(double) * (size_t)std::max(nw, 1), 256);
  return L;
}

// Two operand buffers when there is more than one slab: slab s+1 is quantized
// while slab s accumulates.
static int split_nbuf(int64_t P, int slab = SP_SLAB) { return P > slab ? 2 : 1; }

static int clamp_slab(int slab) {
  if (slab <= 0) return SP_SLAB;
  return (int)std::min<int64_t>(SP_SLAB, std::max<int64_t>(SP_KB, slab / SP_KB * SP_KB));
}

size_t split_workspace_bytes(int64_t P, int N, int nw, int slab) {
  slab = clamp_slab(slab);
  SplitLayout L = split_layout(P, N, nw, slab);
  return split_nbuf(P, slab) * (L.a_bytes + L.b_bytes + L.s_bytes + L.w_bytes) + 1024;
}
size_t split_workspace_bytes(int64_t P, int N, int nw) {
  return split_workspace_bytes(P, N, nw, SP_SLAB);
}

void timing_mark(spx_ctx* ctx, cudaStream_t s, int kind);

// variant: 1 one CTA per tile, 2 CTA pair, 0 the context's choice; slab: pairs per
// exact int32 slab (0 = 32768).
int split_chi0_slab(spx_ctx* ctx, const double2* M, int64_t ldc, int64_t P, int N, const double* W,
                    int64_t ldw, int nw, double2* out, void* ws, size_t ws_bytes,
                    cudaStream_t stream, int* launches, int variant, int slab) {
  if (P <= 0 || N <= 0 || nw <= 0) return SPX_OK;
  slab = clamp_slab(slab);
  SplitLayout L = split_layout(P, N, nw, slab);
  if (!ws || ws_bytes < split_workspace_bytes(P, N, nw, slab))
    return set_error(ctx, SPX_EINVAL, "split workspace too small");
  uint8_t* base = (uint8_t*)align_up((size_t)ws, 1024);
  const int nbuf = split_nbuf(P, slab);
  const size_t set_bytes = L.a_bytes + L.b_bytes + L.s_bytes + L.w_bytes;
  int8_t* A[2];
  int8_t* B[2];
  double* sA[2];
  double* wmax[2];
  for (int b = 0; b < 2; ++b) {
    uint8_t* s0 = base + (size_t)(b < nbuf ? b : 0) * set_bytes;
    A[b] = (int8_t*)s0;
    B[b] = (int8_t*)(s0 + L.a_bytes);
    sA[b] = (double*)(s0 + L.a_bytes + L.b_bytes);
    wmax[b] = (double*)(s0 + L.a_bytes + L.b_bytes + L.s_bytes);
  }

  // planes in HBM: [plane][k-block][row][K bytes]; TMA dims (K, row, k-block, plane)
  // with increasing strides; a box (K, rows, 1, planes) lands as [plane][row][K]
  const uint64_t nkb = (uint64_t)(L.Ps / SP_KB);
  if (variant == 0) variant = ctx->opt.split_variant;
  const bool pair = variant != 1;  // 0 (auto) and 2 select the CTA pair
  CUtensorMap mapA[2], mapB[2];
  for (int b = 0; b < nbuf; ++b) {
    const uint64_t sta[3] = {SP_KB, (uint64_t)L.R * SP_KB, nkb * L.R * SP_KB};
    const uint64_t da[4] = {SP_KB, (uint64_t)L.R, nkb, SP_SA};
    const uint32_t ba[4] = {SP_KB, SP_ROWS, 1, SP_SA};
    int rc0 = make_tmap_u8_4d(ctx, &mapA[b], A[b], da, sta, ba, CU_TENSOR_MAP_SWIZZLE_64B);
    if (rc0) return rc0;
    const uint64_t db[4] = {SP_KB, (uint64_t)L.R, nkb, (uint64_t)SP_SB * nw};
    const uint32_t bb[4] = {SP_KB, (uint32_t)(pair ? SP2_BROWS : SP_ROWS), 1, SP_SB};
    rc0 = make_tmap_u8_4d(ctx, &mapB[b], B[b], db, sta, bb, CU_TENSOR_MAP_SWIZZLE_64B);
    if (rc0) return rc0;
  }
  int rc = SPX_OK;

  const size_t smem = sizeof(SplitSmem) + 1024;
  const size_t smem2 = sizeof(Split2Smem) + 1024;
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(split_gram_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(split_gram2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem2);
    attr_set = true;
  }
  const int ntile = L.nblk * (L.nblk + 1) / 2;
  int ntile2 = 0;
  for (int bj = 0; bj < L.nblk; ++bj) ntile2 += bj / 2 + 1;
  const int nitems = (pair ? ntile2 : ntile) * nw;
  const int grid = std::min(nitems, ctx->num_sms);
  const int npad = (int)(L.R / 2);  // columns covered by the stacked rows
  // CTA-pair launch: as many clusters as can be resident at once (persistent)
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute cattr[1];
  int nclusters = 0;
  if (pair) {
    cattr[0].id = cudaLaunchAttributeClusterDimension;
    cattr[0].val.clusterDim.x = 2;
    cattr[0].val.clusterDim.y = 1;
    cattr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(SP_THREADS);
    cfg.dynamicSmemBytes = smem2;
    cfg.stream = stream;
    cfg.attrs = cattr;
    cfg.numAttrs = 1;
    cfg.gridDim = dim3(2 * (ctx->num_sms / 2));
    int maxc = 0;
    rc = check_cuda(ctx, cudaOccupancyMaxActiveClusters(&maxc, split_gram2_kernel, &cfg),
                    "cudaOccupancyMaxActiveClusters");
    if (rc) return rc;
    if (maxc <= 0) return set_error(ctx, SPX_ENOTSUP, "no CTA-pair cluster fits on this device");
    nclusters = std::min(nitems, maxc);
    cfg.gridDim = dim3(2 * nclusters);
  }

  // Preparation (column scales, weight maxima, digit planes) of slab s+1 runs on
  // the preparation stream while slab s accumulates on `stream`; buffer b = s % 2.
  const int64_t nslab = (P + L.Ps - 1) / L.Ps;
  cudaStream_t ps = ctx->prep_stream;
  cudaEvent_t ev_start = ctx->sev[0];
  cudaEvent_t prep_done[2] = {ctx->sev[1], ctx->sev[2]};
  cudaEvent_t gram_done[2] = {ctx->sev[3], ctx->sev[4]};
  auto prep = [&](int64_t s) -> int {
    const int b = (int)(s % nbuf);
    const int64_t p0 = s * L.Ps;
    const int len = (int)std::min<int64_t>(L.Ps, P - p0);
    const int lenp = (int)align_up((size_t)len, SP_KB);
    const int nchunk = lenp / 16;  // 16-pair chunks; npad is a multiple of 64
    split_colmax_kernel<<<N, 256, 0, ps>>>(M, ldc, p0, len, sA[b]);
    split_wmax_kernel<<<nw, 256, 0, ps>>>(W, ldw, p0, len, wmax[b]);
    const int64_t nthr = (int64_t)npad * nchunk;
    split_quantize_kernel<<<(unsigned)((nthr + 127) / 128), 128, 0, ps>>>(
        M, ldc, p0, len, nchunk, N, npad, L.R, L.Ps, W, ldw, nw, sA[b], wmax[b], A[b], B[b]);
    int r = check_cuda(ctx, cudaGetLastError(), "split operand preparation");
    if (r) return r;
    *launches += 3;
    return check_cuda(ctx, cudaEventRecord(prep_done[b], ps), "event");
  };
  // the preparation stream starts after everything already queued on `stream`
  // (the weights, and whatever produced cprod)
  if ((rc = check_cuda(ctx, cudaEventRecord(ev_start, stream), "event")) ||
      (rc = check_cuda(ctx, cudaStreamWaitEvent(ps, ev_start, 0), "event")))
    return rc;
  timing_mark(ctx, stream, 0);
  if ((rc = prep(0))) return rc;
  for (int64_t s = 0; s < nslab; ++s) {
    const int b = (int)(s % nbuf);
    const int len = (int)std::min<int64_t>(L.Ps, P - s * L.Ps);
    const int lenp = (int)align_up((size_t)len, SP_KB);
    if ((rc = check_cuda(ctx, cudaStreamWaitEvent(stream, prep_done[b], 0), "event"))) return rc;
    // with two buffers, slab s+1 goes into the buffer that slab s-1 accumulated from
    if (nbuf == 2 && s >= 1 && s + 1 < nslab &&
        (rc = check_cuda(ctx, cudaStreamWaitEvent(ps, gram_done[(s + 1) % 2], 0), "event")))
      return rc;
    timing_mark(ctx, stream, 1);
    SplitParams prm;
    prm.N = N;
    prm.ntile = pair ? ntile2 : ntile;
    prm.nw = nw;
    prm.nitems = nitems;
    prm.nk = lenp / SP_KB;
    prm.sA = sA[b];
    prm.wmax = wmax[b];
    prm.out = reinterpret_cast<double*>(out);
    prm.npack = (int64_t)N * (N + 1) / 2;
    prm.status = ctx->d_status;
    prm.timeout_ns =
        (uint64_t)(ctx->opt.timeout_ms > 0 ? ctx->opt.timeout_ms : 4000) * 1000000ull;
    if (pair) {
      rc = check_cuda(ctx, cudaLaunchKernelEx(&cfg, split_gram2_kernel, mapA[b], mapB[b], prm),
                      "split_gram2_kernel launch");
    } else {
      split_gram_kernel<<<grid, SP_THREADS, smem, stream>>>(mapA[b], mapB[b], prm);
      rc = check_cuda(ctx, cudaGetLastError(), "split_gram_kernel launch");
    }
    if (rc) return rc;
    *launches += 1;
    if ((rc = check_cuda(ctx, cudaEventRecord(gram_done[b], stream), "event"))) return rc;
    if (s + 1 < nslab) {
      // with one buffer, the next preparation waits for this accumulation
      if (nbuf == 1 &&
          (rc = check_cuda(ctx, cudaStreamWaitEvent(ps, gram_done[0], 0), "event")))
        return rc;
      if ((rc = prep(s + 1))) return rc;
    }
  }
  return SPX_OK;
}

}  // namespace spx

// ---------------------------------------------------------------------------
// K4s: the interstitial product GEMM of the explicit convolution
// (src/wavefproducts.f:945, cprod += conj(cpw2^H cpw3)/sqrt(vol)) on the same
// int8 digit slices as K2. C_b(m, col) = alpha * sum_k A_b(m, k) conj(B_b(col, k)):
// A = the unoccupied coefficients (rows n'), B = the gathered convolution
// cpw0(G2 - G_M + g) (rows (n, ig)), one batch per k point. Each row is scaled
// by its own largest |Re|, |Im| over k; A keeps 3 digits, B 4, and the nine
// products with t + u <= 3 are summed exactly in int32 (k <= 32768 per launch),
// so the only rounding is the slicing: 2^-17/127 of A's row scale per value, so
// |error of C(m, col)| <= 2^-17/127 * crest(A_m) * ||A_m|| ||B_col||.
// Items are rectangular (batch, column tile, row tile), row tiles fastest so that
// concurrent CTAs share the large B tile through L2. The epilogue adds alpha
// times the tile into cprod's columns: each double is written by one thread.

namespace spx {

struct SgParams {
  int nbatch, mtiles, ntiles, nitems, nk;
  int64_t RA, RB;          // real-stacked rows per batch of the A and B planes
  int M, ncol, ncin;       // valid rows of A, columns (= rows of B), col = n*ncin + c
  const double* sA;        // row scales [batch][mtiles*64]
  const double* sB;        // [batch][ntiles*64]
  double* out;             // cprod as doubles, at (row 0, column 0) of batch 0
  int64_t sO2, sOn, sOc;   // complex strides: batch, n, c
  double alpha;
  int* status;
  uint64_t timeout_ns;
};

// The same GEMM with 32-column tiles (N = 64 real rows of B, stacked in 32-blocks)
// and two TMEM buffers of 4 orders x 64 columns: the MMAs of item j+1 run while the
// epilogue drains item j, which the short K of the product GEMM needs (47 stages at
// 3000 plane waves, against 512 for K2).
constexpr int SG_TB = 32;                        // complex B rows per tile
constexpr int SG_ST = 4;
constexpr int SG_BPLANE = 2 * SG_TB * SP_KB;     // 4096 bytes
constexpr uint32_t SG_IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(2 * SG_TB / 8) << 17) |
                              ((uint32_t)(SP_ROWS / 16) << 24);

struct __align__(1024) SgSmem {
  uint8_t a[SG_ST][SP_SA][SP_PLANE];
  uint8_t b[SG_ST][SP_SB][SG_BPLANE];
  long long xchg[2][SP_TILE][33];
  uint64_t full[SG_ST];
  uint64_t empty[SG_ST];
  uint64_t tfull[2], tempty[2];
  uint64_t xfull, xfree, mdone;
  uint32_t tmem_base;
};

// T = ((D0*256 + D1)*256 + D2)*256 + D3 for 32 columns, orders 64 columns apart.
__device__ __forceinline__ void load_orders64(uint32_t taddr, long long (&T)[32]) {
  int32_t r[32];
  tmem_ld32(taddr, r);
  tmem_wait_ld();
#pragma unroll
  for (int k = 0; k < 32; ++k) T[k] = r[k];
#pragma unroll
  for (int g = 1; g < 4; ++g) {
    tmem_ld32(taddr + (uint32_t)(g * 64), r);
    tmem_wait_ld();
#pragma unroll
    for (int k = 0; k < 32; ++k) T[k] = T[k] * 256 + r[k];
  }
}

__global__ void __launch_bounds__(SP_THREADS, 1)
    split_gemm2_kernel(const __grid_constant__ CUtensorMap mapA,
                       const __grid_constant__ CUtensorMap mapB, SgParams prm) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  SgSmem& sm = *reinterpret_cast<SgSmem*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < SG_ST; ++s) {
      mbar_init(&sm.full[s], 1);
      mbar_init(&sm.empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&sm.tfull[b], 1);
      mbar_init(&sm.tempty[b], 4);
    }
    mbar_init(&sm.xfull, 4);
    mbar_init(&sm.xfree, 4);
    mbar_init(&sm.mdone, 1);
    fence_barrier_init();
  }
  if (warp == 1) tmem_alloc(&sm.tmem_base, SP_TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sm.tmem_base;
  const int mtiles = prm.mtiles, ntiles = prm.ntiles;

  if (warp == 0) {
    if (lane == 0) {
      int st = 0;
      uint32_t ph = 0;
      bool issued[SG_ST];
      uint32_t last_ph[SG_ST];
      for (int s = 0; s < SG_ST; ++s) issued[s] = false, last_ph[s] = 0;
      bool ok = true;
      for (int item = blockIdx.x; item < prm.nitems && ok; item += gridDim.x) {
        const int mt = item % mtiles, r = item / mtiles, ct = r % ntiles, b = r / ntiles;
        const int ra = (int)(b * prm.RA) + mt * SP_ROWS, rb = (int)(b * prm.RB) + ct * (2 * SG_TB);
        for (int ks = 0; ks < prm.nk; ++ks) {
          if (!mbar_wait(&sm.empty[st], ph ^ 1u, prm.timeout_ns, prm.status)) {
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(&sm.full[st], (uint32_t)(SP_SA * SP_PLANE + SP_SB * SG_BPLANE));
          tma_load_4d(&sm.a[st][0][0], &mapA, 0, ra, ks, 0, &sm.full[st]);
          tma_load_4d(&sm.b[st][0][0], &mapB, 0, rb, ks, 0, &sm.full[st]);
          issued[st] = true;
          last_ph[st] = ph;
          if (++st == SG_ST) st = 0, ph ^= 1u;
        }
      }
      for (int s = 0; s < SG_ST; ++s)
        if (issued[s]) mbar_drain(&sm.full[s], last_ph[s], prm.timeout_ns);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int st = 0;
      uint32_t ph = 0;
      int j = 0;
      bool committed = false;
      for (int item = blockIdx.x; item < prm.nitems; item += gridDim.x, ++j) {
        const int buf = j & 1;
        // this buffer's previous item (j - 2) has been drained (first use: immediately)
        if (!mbar_wait(&sm.tempty[buf], (uint32_t)((j >> 1) & 1) ^ 1u, prm.timeout_ns, prm.status)) break;
        tc_fence_after();
        const uint32_t tb = tmem + (uint32_t)(buf * 256);
        bool ok = true;
        for (int ks = 0; ks < prm.nk; ++ks) {
          if (!mbar_wait(&sm.full[st], ph, prm.timeout_ns, prm.status)) {
            ok = false;
            break;
          }
          tc_fence_after();
#pragma unroll
          for (int kk = 0; kk < SP_NKS; ++kk) {
            uint64_t da[SP_SA], db[SP_SB];
#pragma unroll
            for (int t = 0; t < SP_SA; ++t) da[t] = desc_sw64(&sm.a[st][t][0]) + (uint64_t)(kk * 2);
#pragma unroll
            for (int u = 0; u < SP_SB; ++u) db[u] = desc_sw64(&sm.b[st][u][0]) + (uint64_t)(kk * 2);
            const uint32_t k0 = (ks > 0 || kk > 0);
            mma_i8<1>(tb + 0 * 64, da[0], db[0], SG_IDESC, k0);
            mma_i8<2>(tb + 1 * 64, da[0], db[1], SG_IDESC, k0);
            mma_i8<2>(tb + 2 * 64, da[0], db[2], SG_IDESC, k0);
            mma_i8<3>(tb + 3 * 64, da[0], db[3], SG_IDESC, k0);
            mma_i8<1>(tb + 1 * 64, da[1], db[0], SG_IDESC, 1u);
            mma_i8<2>(tb + 2 * 64, da[1], db[1], SG_IDESC, 1u);
            mma_i8<3>(tb + 3 * 64, da[1], db[2], SG_IDESC, 1u);
            mma_i8<1>(tb + 2 * 64, da[2], db[0], SG_IDESC, 1u);
            mma_i8<3>(tb + 3 * 64, da[2], db[1], SG_IDESC, 1u);
          }
          tc_commit(&sm.empty[st]);
          committed = true;
          if (++st == SG_ST) st = 0, ph ^= 1u;
        }
        if (!ok) break;
        tc_commit(&sm.tfull[buf]);
      }
      if (committed) {
        tc_commit(&sm.mdone);
        mbar_drain(&sm.mdone, 0u, prm.timeout_ns);
      }
    }
  } else {
    const int q = warp & 3;
    const bool is_re = q < 2;
    const int ii = (q & 1) * 32 + lane;
    const uint32_t tl = tmem + ((uint32_t)(32 * q) << 16);
    int j = 0;
    uint32_t xseq = 0;
    for (int item = blockIdx.x; item < prm.nitems; item += gridDim.x, ++j, ++xseq) {
      const int buf = j & 1;
      if (!mbar_wait_idle(&sm.tfull[buf], (uint32_t)((j >> 1) & 1), prm.timeout_ns, prm.status)) break;
      tc_fence_after();
      const int mt = item % mtiles, r = item / mtiles, ct = r % ntiles, b = r / ntiles;
      long long tre[32], tim[32];
      load_orders64(tl + (uint32_t)(buf * 256), tre);
      load_orders64(tl + (uint32_t)(buf * 256 + SG_TB), tim);
      // the buffer is read: the MMAs of item j + 2 may overwrite it
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&sm.tempty[buf]);
      const int gm = mt * SP_TILE + ii;
      const double fac = prm.alpha * prm.sA[(int64_t)b * mtiles * SP_TILE + gm] *
                         (1.0 / (127.0 * 127.0 * 16777216.0));
      const double* sbb = prm.sB + (int64_t)b * ntiles * SG_TB;
      double* ob = prm.out + 2 * (b * prm.sO2 + gm) + (is_re ? 0 : 1);
      if (!mbar_wait(&sm.xfree, (xseq & 1u) ^ 1u, prm.timeout_ns, prm.status)) break;
#pragma unroll
      for (int k = 0; k < 32; ++k) sm.xchg[is_re ? 0 : 1][ii][k] = tim[k];
      __syncwarp();
      if (lane == 0) mbar_arrive(&sm.xfull);
      if (!mbar_wait(&sm.xfull, xseq & 1u, prm.timeout_ns, prm.status)) break;
#pragma unroll
      for (int k = 0; k < 32; ++k) {
        const int gc = ct * SG_TB + k;
        const long long partner = sm.xchg[is_re ? 1 : 0][ii][k];
        const long long v = is_re ? tre[k] + partner : tre[k] - partner;
        if (gm < prm.M && gc < prm.ncol) {
          const int n = gc / prm.ncin, c = gc - n * prm.ncin;
          // one add per element per launch: a reduction that nothing waits on
          atomicAdd(ob + 2 * (n * prm.sOn + c * prm.sOc), fac * sbb[gc] * (double)v);
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&sm.xfree);
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1) tmem_dealloc(tmem, SP_TMEM_COLS);
}

// Row sources of the two operands: A rows are contiguous in k, B rows are gathered.
struct SgSrcRows {
  const double2* base;
  int64_t ld, bstride;
  __device__ __forceinline__ double2 get(int b, int r, int k) const {
    return base[b * bstride + (int64_t)r * ld + k];
  }
};
struct SgSrcGather {
  const double2* grid;      // [batch][n][box]
  int64_t bstride, nstride;
  const int64_t* coff;      // per c
  const int* koff;          // per k
  int ncin;
  __device__ __forceinline__ double2 get(int b, int r, int k) const {
    const int n = r / ncin, c = r - n * ncin;
    return grid[b * bstride + n * nstride + coff[c] + koff[k]];
  }
};

// s[b*rows_pad + r] = max_k max(|Re|, |Im|) of row r of batch b (0 for padding rows).
template <class Src>
__global__ void sgemm_rowmax_kernel(Src src, int rows, int rows_pad, int K, double* s) {
  const int r = blockIdx.x, b = blockIdx.y;
  double m = 0.0;
  if (r < rows)
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
      const double2 v = src.get(b, r, k);
      m = fmax(m, fmax(fabs(v.x), fabs(v.y)));
    }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) s[(int64_t)b * rows_pad + r] = m;
  }
}

// S digits of round(x * 127/s * 2^(8(S-1))) into planes [t][k-block][row][64 B] with
// real-stacked rows b*R + 2 TB (r/TB) + {r%TB Re, TB + r%TB Im}. One thread = one row
// and 16 consecutive k; a warp = 8 consecutive rows x the 4 quarters of a k-block.
template <int S, int TB, class Src>
__global__ void __launch_bounds__(128)
    sgemm_quant_kernel(Src src, int rows, int rows_pad, int K, int nkb, int nbatch, int64_t R,
                       const double* __restrict__ s, int8_t* __restrict__ planes) {
  const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int ngroup = rows_pad / 8;
  if (tid >= (int64_t)ngroup * 32 * nkb * nbatch) return;
  const int lane8 = (int)(tid & 7), quarter = (int)((tid >> 3) & 3);
  const int64_t rest = tid >> 5;
  const int r = (int)(rest % ngroup) * 8 + lane8;
  const int64_t kbb = rest / ngroup;
  const int kb = (int)(kbb % nkb), b = (int)(kbb / nkb);
  const int k0 = kb * SP_KB + quarter * 16;
  const int64_t rows_total = (int64_t)nbatch * R;
  const int64_t rr = (int64_t)b * R + (r / TB) * (2 * TB) + (r % TB);
  const int64_t pstride = (int64_t)nkb * rows_total * SP_KB;
  const int64_t o_re = ((int64_t)kb * rows_total + rr) * SP_KB + quarter * 16;
  const int64_t o_im = o_re + (int64_t)TB * SP_KB;
  const double sc = r < rows ? s[(int64_t)b * rows_pad + r] : 0.0;
  const double inv = sc > 0.0 ? 127.0 * (S == 4 ? 16777216.0 : 65536.0) / sc : 0.0;
  uint32_t wr[S][4], wi[S][4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    uint32_t yr[4], yi[4], pr[S], pi[S];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int k = k0 + 4 * q + e;
      double2 v = make_double2(0.0, 0.0);
      if (r < rows && k < K) v = src.get(b, r, k);
      yr[e] = round_mul(v.x, inv);
      yi[e] = round_mul(v.y, inv);
    }
    digit_planes<S>(yr, pr);
    digit_planes<S>(yi, pi);
#pragma unroll
    for (int t = 0; t < S; ++t) wr[t][q] = pr[t], wi[t][q] = pi[t];
  }
#pragma unroll
  for (int t = 0; t < S; ++t) {
    *reinterpret_cast<uint4*>(planes + o_re + t * pstride) = make_uint4(wr[t][0], wr[t][1], wr[t][2], wr[t][3]);
    *reinterpret_cast<uint4*>(planes + o_im + t * pstride) = make_uint4(wi[t][0], wi[t][1], wi[t][2], wi[t][3]);
  }
}

// Bytes of scratch for one launch group of `nbatch` batches (planes and scales).
size_t sgemm_workspace_bytes(int nbatch, int M, int ncol, int K) {
  const int64_t mt = (M + SP_TILE - 1) / SP_TILE, nt2 = (ncol + SG_TB - 1) / SG_TB;
  const int64_t nt = (nt2 + 1) / 2;  // in 64-row units: B has 2 SG_TB rows per tile
  const int64_t kp = (int64_t)align_up((size_t)std::min(std::max(K, 1), SP_SLAB), SP_KB);
  return align_up((size_t)SP_SA * kp * nbatch * mt * SP_ROWS, 1024) +
         align_up((size_t)SP_SB * kp * nbatch * nt * SP_ROWS, 1024) +
         align_up(sizeof(double) * nbatch * mt * SP_TILE, 256) +
         align_up(sizeof(double) * nbatch * nt * SP_TILE, 256) + 2048;
}

// The interstitial product GEMM on int8 slices for `nbatch` k points: A rows from
// cpw_unocc (contiguous), B rows gathered from the convolved grids.
int sgemm_products(spx_ctx* ctx, int nbatch, int M, int ncol, int K, const double2* A,
                   int64_t lda, int64_t a_bstride, const double2* grid, int64_t g_bstride,
                   int64_t g_nstride, const int64_t* coff, const int* koff, int ncin,
                   double2* out, int64_t sO2, int64_t sOn, int64_t sOc, double alpha, void* ws,
                   size_t ws_bytes, cudaStream_t s, int* launches) {
  if (nbatch <= 0 || M <= 0 || ncol <= 0 || K <= 0) return SPX_OK;
  const int mt = (M + SP_TILE - 1) / SP_TILE, nt = (ncol + SG_TB - 1) / SG_TB;
  const int64_t RA = (int64_t)mt * SP_ROWS, RB = (int64_t)nt * 2 * SG_TB;
  if ((int64_t)nbatch * RB > 2147483647LL || (int64_t)nbatch * mt * nt > 2147483647LL)
    return set_error(ctx, SPX_EINVAL, "product GEMM too large for one launch group");
  uint8_t* base = (uint8_t*)align_up((size_t)ws, 1024);
  const size_t need = sgemm_workspace_bytes(nbatch, M, ncol, K);
  if (!ws || ws_bytes < need + 1024) return set_error(ctx, SPX_ENOMEM, "split product scratch too small");
  const size_t smem = sizeof(SgSmem) + 1024;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(split_gemm2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attr = true;
  }
  int rc;
  // k is cut into exact int32 slabs of at most 32768; each slab adds into the output
  for (int kbeg = 0; kbeg < K; kbeg += SP_SLAB) {
    const int Ks = std::min(SP_SLAB, K - kbeg);
    const int nkb = (int)(align_up((size_t)Ks, SP_KB) / SP_KB);
    const int64_t kp = (int64_t)nkb * SP_KB;
    int8_t* PA = (int8_t*)base;
    int8_t* PB = (int8_t*)(base + align_up((size_t)SP_SA * kp * nbatch * RA, 1024));
    double* sA = (double*)((uint8_t*)PB + align_up((size_t)SP_SB * kp * nbatch * RB, 1024));
    double* sB = (double*)((uint8_t*)sA + align_up(sizeof(double) * nbatch * mt * SP_TILE, 256));
    const int rows_b = nt * SG_TB;  // padded B rows (complex) per batch
    SgSrcRows sa{A + kbeg, lda, a_bstride};
    SgSrcGather sb{grid, g_bstride, g_nstride, coff, koff + kbeg, ncin};
    sgemm_rowmax_kernel<<<dim3(mt * SP_TILE, nbatch), 256, 0, s>>>(sa, M, mt * SP_TILE, Ks, sA);
    sgemm_rowmax_kernel<<<dim3(rows_b, nbatch), 256, 0, s>>>(sb, ncol, rows_b, Ks, sB);
    const int64_t ta = (int64_t)mt * SP_TILE / 8 * 32 * nkb * nbatch;
    const int64_t tb = (int64_t)rows_b / 8 * 32 * nkb * nbatch;
    sgemm_quant_kernel<SP_SA, SP_TILE><<<(unsigned)((ta + 127) / 128), 128, 0, s>>>(sa, M, mt * SP_TILE, Ks, nkb, nbatch, RA, sA, PA);
    sgemm_quant_kernel<SP_SB, SG_TB><<<(unsigned)((tb + 127) / 128), 128, 0, s>>>(sb, ncol, rows_b, Ks, nkb, nbatch, RB, sB, PB);
    if ((rc = check_cuda(ctx, cudaGetLastError(), "split product operand preparation"))) return rc;
    *launches += 4;
    CUtensorMap mapA, mapB;
    const uint64_t rta = (uint64_t)nbatch * RA, rtb = (uint64_t)nbatch * RB;
    const uint64_t da[4] = {SP_KB, rta, (uint64_t)nkb, SP_SA};
    const uint64_t sta[3] = {SP_KB, rta * SP_KB, (uint64_t)nkb * rta * SP_KB};
    const uint32_t ba[4] = {SP_KB, SP_ROWS, 1, SP_SA};
    if ((rc = make_tmap_u8_4d(ctx, &mapA, PA, da, sta, ba, CU_TENSOR_MAP_SWIZZLE_64B))) return rc;
    const uint64_t db[4] = {SP_KB, rtb, (uint64_t)nkb, SP_SB};
    const uint64_t stb[3] = {SP_KB, rtb * SP_KB, (uint64_t)nkb * rtb * SP_KB};
    const uint32_t bb[4] = {SP_KB, 2 * SG_TB, 1, SP_SB};
    if ((rc = make_tmap_u8_4d(ctx, &mapB, PB, db, stb, bb, CU_TENSOR_MAP_SWIZZLE_64B))) return rc;
    SgParams prm;
    prm.nbatch = nbatch;
    prm.mtiles = mt;
    prm.ntiles = nt;
    prm.nitems = nbatch * mt * nt;
    prm.nk = nkb;
    prm.RA = RA;
    prm.RB = RB;
    prm.M = M;
    prm.ncol = ncol;
    prm.ncin = ncin;
    prm.sA = sA;
    prm.sB = sB;
    prm.out = reinterpret_cast<double*>(out);
    prm.sO2 = sO2;
    prm.sOn = sOn;
    prm.sOc = sOc;
    prm.alpha = alpha;
    prm.status = ctx->d_status;
    prm.timeout_ns = (uint64_t)(ctx->opt.timeout_ms > 0 ? ctx->opt.timeout_ms : 4000) * 1000000ull;
    const int grid_n = std::min(prm.nitems, ctx->num_sms);
    split_gemm2_kernel<<<grid_n, SP_THREADS, smem, s>>>(mapA, mapB, prm);
    if ((rc = check_cuda(ctx, cudaGetLastError(), "split_gemm2_kernel launch"))) return rc;
    *launches += 1;
  }
  return SPX_OK;
}

}  // namespace spx
