// K2: split-precision band-pair accumulation on the 5th-generation tensor cores.
//
// The sum chi_f(i, j) = sum_p M(p, i) conj(M(p, j)) w(p, f) (src/susceptibility.f:
// 1182-1240 with the HILBERT NONE weights of :950-975) is evaluated as an exact
// integer contraction of 8-bit digit slices (an Ozaki-type error-free split) of
// the weight-folded operand
//
//   A(p, i) = sqrt(|w(p, f)|) M(p, i),   chi_f = A^T diag(sgn w) conj(A),
//
// one operand per frequency for both sides of the product. For every frequency
// whose weights have one sign over the slab (all imaginary-axis HILBERT NONE
// weights) the Gram is A^T conj(A) times that sign, a Hermitian rank-P update
// whose two operands are the same digit planes. Frequencies with weights of both
// signs take B(p, j) = sgn(w(p, f)) A(p, j) as the second operand (its own planes).
// Each value becomes three balanced base-256 digits of one rounded integer,
//
//   A = s sqrt(wmax)/127 * 2^-16 * (d0 2^16 + d1 2^8 + d2),  |d0| <= 127,
//
// with s the largest |Re|, |Im| of the column M(:, i) over the slab of band pairs
// and wmax = max_p |w(p, f)|. The six digit products with t + u <= 2 are summed on
// tcgen05.mma kind::i8 into three int32 accumulators in tensor memory, one per
// order g = t + u, exactly (3 * 128^2 * 32768 < 2^31). Once per slab the epilogue
// forms (D0*256 + D1)*256 + D2 exactly and adds s_i s_j wmax / (127^2 2^16) times
// it (times the sign) to the FP64 output. Weights and scales stay FP64 throughout,
// so near-degenerate pairs keep their FP64 weights.
//
// Error (per element, relative to sqrt(sum_p |w| |M_pi|^2 sum_p |w| |M_pj|^2), which
// is sqrt|chi_ii chi_jj| for one-signed weights): rounding of each operand is half a
// unit of its third digit, 2^-17/127 of its column scale, and the dropped orders
// g >= 3 are of the same size; both enter with the crest factor max|A| sqrt(P)/||A||
// of the folded columns.
//
// Tile layout: a 64 x 64 complex tile is a 128 x 128 real-stacked product whose rows
// interleave the parts of each mixed-basis function: row 2i holds Re A_i and row
// 2i+1 holds Im A_i (likewise the columns for j). D[2i+c][2j+c'] then holds the four
// real products of (i, j) in two adjacent TMEM lanes, and the epilogue combines
// re = D[2i][2j] + D[2i+1][2j+1], im = D[2i+1][2j] - D[2i][2j+1] by one warp shuffle.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "spx_split.cuh"

namespace spx {

constexpr int SP_ST = 4;               // pipeline stages (one CTA per tile)
constexpr int SP_THREADS = 192;        // warp 0 TMA, warp 1 MMA + TMEM, warps 2-5 epilogue
// The one-CTA kernel drains a tile with 8 epilogue warps (warps 2-9; two per TMEM lane
// quarter, each half of the columns): fewer registers per thread, so the operand
// quantizer of the next slab keeps more warps resident beside it on every SM.
constexpr int SP1_EPI = 8;
constexpr int SP_WIDE_BN = 80;  // complex columns of the wide tile (variant 5): N = 160
constexpr int SP1_THREADS = 64 + 32 * SP1_EPI;
constexpr int SP1_REGS = 128;  // 40960 registers: two 96-register quantizer blocks fit beside

// BROWS: real rows of the B tile (the MMA's N): 128 for 64 x 64 complex tiles, 160
// for 64 x 80 (three orders x 160 TMEM columns still fit in 512).
template <int BROWS>
struct __align__(1024) SplitSmemT {
  uint8_t a[SP_ST][SP_SF][SP_PLANE];
  uint8_t b[SP_ST][SP_SF][BROWS * SP_KB];
  uint64_t full[SP_ST];
  uint64_t empty[SP_ST];
  uint64_t tfull, tempty, mdone;
  uint32_t tmem_base;
};
using SplitSmem = SplitSmemT<SP_ROWS>;

struct SplitParams {
  int N;
  int nbr;                // 64-row blocks covering N
  int ntile;
  int nw;
  int nitems;
  int nk;                 // pipeline stages per item (pairs of the slab / 64)
  const double* sA;       // column scales of the slab
  const double* wmax;     // max |w(p, f)| of the slab
  const int* wsgn;        // per frequency: +1 / -1 one-signed weights, 0 both signs
  double* out;            // packed complex output, as doubles
  int64_t npack;
  int* status;
  uint64_t timeout_ns;
};

// The epilogue of one tile (or of NC of its 64 complex columns, from column j0), run
// by the epilogue warps (warp q reads TMEM lanes 32q..32q+31, i.e. rows
// i = 16q + lane/2, part c = lane & 1). The warp's part of the accumulator is read
// into registers first and released to the MMA warp, so the next item's MMAs overlap
// this tile's reductions into the output.
template <int NC = SP_TILE, int BN = SP_TILE, class Release>
__device__ __forceinline__ void fold_epilogue(uint32_t tl, int q, int lane, int bi, int bj, int f,
                                              const SplitParams& prm, Release release, int j0 = 0) {
  const int c = lane & 1;
  double o[NC];
#pragma unroll
  for (int cc = 0; cc < NC / 8; ++cc) {
    double T[16];
    load_fold16(tl + (uint32_t)(2 * j0 + 16 * cc), (uint32_t)(2 * BN), T);
#pragma unroll
    for (int jj = 0; jj < 8; ++jj) {
      // both lanes of a row pair send their (., Im_j) product to the other one
      const double pb = __shfl_xor_sync(0xffffffffu, T[2 * jj + 1], 1);
      o[8 * cc + jj] = c == 0 ? T[2 * jj] + pb : T[2 * jj] - pb;
    }
  }
  release();
  const int gil = bi * SP_TILE + 16 * q + lane / 2;
  if (gil >= prm.N) return;
  const double fac = fold_row_factor(prm.wsgn[f], prm.sA[gil], prm.wmax[f]);
  double* ob = prm.out + 2 * (int64_t)f * prm.npack + 2 * gil + c;
#pragma unroll
  for (int jj = 0; jj < NC; ++jj) {
    const int gj = bj * BN + j0 + jj;
    // one add per element per launch: launches are stream-ordered, so the sum is
    // deterministic, and the reduction needs no read round trip
    if (gil <= gj && gj < prm.N) atomicAdd(ob + (int64_t)gj * (gj + 1), fac * prm.sA[gj] * o[jj]);
  }
}

// The -DINV (real) epilogue: columns [j0, j0 + ncol) of a 128 x BROWS tile of real chi,
// TMEM lane = row i of the block, column = j; read and added 16 columns at a time,
// then the accumulator is released.
template <int BROWS, class Release>
__device__ __forceinline__ void real_epilogue(uint32_t tl, int q, int lane, int bi, int bj, int f,
                                              const SplitParams& prm, Release release, int j0,
                                              int ncol) {
  const int gi = bi * SP_ROWS + 32 * q + lane;
  const double fac = gi < prm.N ? fold_row_factor(prm.wsgn[f], prm.sA[gi], prm.wmax[f]) : 0.0;
  double* of = prm.out + (int64_t)f * prm.npack + gi;
#pragma unroll 1
  for (int cc = 0; cc < ncol / 16; ++cc) {
    double T[16];
    load_fold16(tl + (uint32_t)(j0 + 16 * cc), (uint32_t)BROWS, T);
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const int gj = bj * BROWS + j0 + 16 * cc + k;
      if (gi < prm.N && gi <= gj && gj < prm.N)
        atomicAdd(of + (int64_t)gj * (gj + 1) / 2, fac * prm.sA[gj] * T[k]);
    }
  }
  release();
}

// BN: complex columns of a tile (64 or 80; the -DINV form uses 64, i.e. 128 x 128
// real tiles). mapF loads 128-row A boxes, mapB (2 BN)-row B boxes.
template <bool REAL, int BN>
__global__ void __maxnreg__(SP1_REGS)
    split_gram_kernel(const __grid_constant__ CUtensorMap mapF, const __grid_constant__ CUtensorMap mapB,
                      SplitParams prm) {
  constexpr int BROWS = 2 * BN;
  constexpr uint32_t IDESC = sp_idesc(BROWS);
  // the -DINV form: tiles of 128 real rows x BROWS real columns (the same block
  // arithmetic as 64 x BN complex tiles)
  using Smem = SplitSmemT<BROWS>;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  Smem& sm = *reinterpret_cast<Smem*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < SP_ST; ++s) {
      mbar_init(&sm.full[s], 1);
      mbar_init(&sm.empty[s], 1);
    }
    mbar_init(&sm.tfull, 1);
    mbar_init(&sm.tempty, SP1_EPI);
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
      int j = 0;
      for (int item = blockIdx.x; item < prm.nitems && ok; item += gridDim.x, ++j) {
        const int f = item / prm.ntile;
        int bi, bj;
        split_decode_tile_bn<BN>(split_item_tile(item, prm.ntile, gridDim.x), prm.nbr, &bi, &bj);
        const int sg = prm.wsgn[f];
        // a diagonal square tile of a one-signed frequency multiplies A by itself
        const bool same = BN == SP_TILE && sg != 0 && bi == bj;
        const int za = f * SP_SLOT, zb = za + (sg == 0 ? SP_SF : 0);
        for (int ks = 0; ks < prm.nk; ++ks) {
          if (!mbar_wait(&sm.empty[st], ph ^ 1u, prm.timeout_ns, prm.status)) {
            ok = false;
            break;
          }
          const int kc = split_k_order(j, ks, prm.nk);
          mbar_arrive_expect_tx(&sm.full[st], (uint32_t)(SP_SF * (SP_PLANE + (same ? 0 : BROWS * SP_KB))));
          tma_load_4d(&sm.a[st][0][0], &mapF, 0, bi * SP_ROWS, kc, za, &sm.full[st]);
          if (!same) tma_load_4d(&sm.b[st][0][0], &mapB, 0, bj * BROWS, kc, zb, &sm.full[st]);
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
        const int f = item / prm.ntile;
        int bi, bj;
        split_decode_tile_bn<BN>(split_item_tile(item, prm.ntile, gridDim.x), prm.nbr, &bi, &bj);
        const bool same = BN == SP_TILE && prm.wsgn[f] != 0 && bi == bj;
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
          // order g = t + u lives at TMEM columns [BROWS g, BROWS g + BROWS); the
          // first product of every order in a slab (first K step) overwrites it
#pragma unroll
          for (int kk = 0; kk < SP_NKS; ++kk) {
            uint64_t da[SP_SF], db[SP_SF];
#pragma unroll
            for (int t = 0; t < SP_SF; ++t) {
              da[t] = desc_sw64(&sm.a[st][t][0]) + (uint64_t)(kk * 2);
              db[t] = same ? da[t] : desc_sw64(&sm.b[st][t][0]) + (uint64_t)(kk * 2);
            }
            const uint32_t k0 = (ks > 0 || kk > 0);
            mma_i8<1>(tmem + 0 * BROWS, da[0], db[0], IDESC, k0);
            mma_i8<2>(tmem + 1 * BROWS, da[0], db[1], IDESC, k0);
            mma_i8<3>(tmem + 2 * BROWS, da[0], db[2], IDESC, k0);
            mma_i8<1>(tmem + 1 * BROWS, da[1], db[0], IDESC, 1u);
            mma_i8<3>(tmem + 2 * BROWS, da[1], db[1], IDESC, 1u);
            mma_i8<0>(tmem + 2 * BROWS, da[2], db[0], IDESC, 1u);
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
    // ---- epilogue: SP1_EPI warps, SP1_EPI / 4 per TMEM lane quarter (column ranges) ----
    const int q = warp & 3, h = (warp - 2) >> 2;
    const uint32_t tl = tmem + ((uint32_t)(32 * q) << 16);
    int j = 0;
    for (int item = blockIdx.x; item < prm.nitems; item += gridDim.x, ++j) {
      if (!mbar_wait_idle(&sm.tfull, (uint32_t)(j & 1), prm.timeout_ns, prm.status)) break;
      tc_fence_after();
      const int f = item / prm.ntile;
      int bi, bj;
      split_decode_tile_bn<BN>(split_item_tile(item, prm.ntile, gridDim.x), prm.nbr, &bi, &bj);
      auto release = [&] {
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&sm.tempty);
      };
      constexpr int NC = BN * 4 / SP1_EPI;  // complex columns per epilogue warp
      if constexpr (REAL) real_epilogue<BROWS>(tl, q, lane, bi, bj, f, prm, release, 2 * NC * h, 2 * NC);
      else fold_epilogue<NC, BN>(tl, q, lane, bi, bj, f, prm, release, NC * h);
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
// half of the shared B tile (64 rows: CTA 0 the columns j of the first 32, CTA 1
// the next 32); the leader CTA issues the MMAs, which read both CTAs' shared memory
// and write each CTA's own TMEM. Every completion that crosses the pair is an
// explicit remote arrive or commit (no multicast).

constexpr int SP2_ST = 5;
constexpr int SP2_BROWS = SP_ROWS / 2;          // B rows staged per CTA
constexpr int SP2_BPLANE = SP2_BROWS * SP_KB;   // 4096 bytes
constexpr uint32_t SP2_IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(SP_ROWS / 8) << 17) |
                               ((uint32_t)(2 * SP_ROWS / 16) << 24);   // M = 256, N = 128

struct __align__(1024) Split2Smem {
  uint8_t a[SP2_ST][SP_SF][SP_PLANE];
  uint8_t b[SP2_ST][SP_SF][SP2_BPLANE];
  uint64_t full[SP2_ST];   // leader: both CTAs' bytes of a stage have landed
  uint64_t empty[SP2_ST];  // each CTA: the MMAs have read the stage
  uint64_t tfull;          // each CTA: accumulators ready
  uint64_t tempty;         // leader: both CTAs' epilogues have drained TMEM (8 warps)
  uint64_t mdone;
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

__global__ void __launch_bounds__(SP_THREADS, 1)
    split_gram2_kernel(const __grid_constant__ CUtensorMap mapF,
                       const __grid_constant__ CUtensorMap mapFh, SplitParams prm) {
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
      // Cursor over this cluster's (item, stage) sequence; it advances by increments
      // and decodes a tile only when it enters a new item.
      struct Cursor {
        int item, ks, ya, yb, za, zb, j;
      };
      auto enter = [&](Cursor& u) {
        int bI, bJ;
        pair_decode_tile(u.item % prm.ntile, &bI, &bJ);
        const int f = u.item / prm.ntile;
        u.ya = (2 * bI + (int)rank) * SP_ROWS;
        u.yb = bJ * SP_ROWS + (int)rank * SP2_BROWS;
        u.za = f * SP_SLOT;
        u.zb = u.za + (prm.wsgn[f] == 0 ? SP_SF : 0);
      };
      auto advance = [&](Cursor& u) {
        if (++u.ks == prm.nk) {
          u.ks = 0;
          u.item += ncl;
          ++u.j;
          if (u.item < prm.nitems) enter(u);
        }
      };
      Cursor ld{cid, 0, 0, 0, 0, 0, 0};
      if (cid < prm.nitems) enter(ld);
      while (ld.item < prm.nitems) {
        if (!mbar_wait(&sm.empty[st], ph ^ 1u, prm.timeout_ns, prm.status)) break;
        const uint32_t lead_full = mapa_shared(smem_u32(&sm.full[st]), 0);
        if (rank == 0)
          mbar_arrive_expect_tx(&sm.full[st], (uint32_t)(2 * SP_SF * (SP_PLANE + SP2_BPLANE)));
        const int kc = split_k_order(ld.j, ld.ks, prm.nk);
        tma_load_4d_pair(&sm.a[st][0][0], &mapF, 0, ld.ya, kc, ld.za, lead_full);
        tma_load_4d_pair(&sm.b[st][0][0], &mapFh, 0, ld.yb, kc, ld.zb, lead_full);
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
            uint64_t da[SP_SF], db[SP_SF];
#pragma unroll
            for (int t = 0; t < SP_SF; ++t) {
              da[t] = desc_sw64(&sm.a[st][t][0]) + (uint64_t)(kk * 2);
              db[t] = desc_sw64(&sm.b[st][t][0]) + (uint64_t)(kk * 2);
            }
            const uint32_t k0 = (ks > 0 || kk > 0);
            mma2_i8<1>(tmem + 0 * 128, da[0], db[0], SP2_IDESC, k0);
            mma2_i8<2>(tmem + 1 * 128, da[0], db[1], SP2_IDESC, k0);
            mma2_i8<3>(tmem + 2 * 128, da[0], db[2], SP2_IDESC, k0);
            mma2_i8<1>(tmem + 1 * 128, da[1], db[0], SP2_IDESC, 1u);
            mma2_i8<3>(tmem + 2 * 128, da[1], db[1], SP2_IDESC, 1u);
            mma2_i8<0>(tmem + 2 * 128, da[2], db[0], SP2_IDESC, 1u);
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
    const uint32_t tl = tmem + ((uint32_t)(32 * q) << 16);
    const uint32_t lead_tempty = mapa_shared(smem_u32(&sm.tempty), 0);
    int j = 0;
    for (int item = cid; item < prm.nitems; item += ncl, ++j) {
      if (!mbar_wait_idle(&sm.tfull, (uint32_t)(j & 1), prm.timeout_ns, prm.status)) break;
      tc_fence_after();
      const int f = item / prm.ntile;
      int bI, bJ;
      pair_decode_tile(item % prm.ntile, &bI, &bJ);
      const int bi = 2 * bI + (int)rank;
      auto release = [&] {
        tc_fence_before();
        __syncwarp();
        if (lane == 0) {
          if (rank == 0) mbar_arrive(&sm.tempty);
          else mbar_arrive_cluster(lead_tempty);
        }
      };
      // a tile wholly below the diagonal or past N has nothing to store
      if (bi <= bJ && bi * SP_TILE < prm.N) fold_epilogue(tl, q, lane, bi, bJ, f, prm, release);
      else release();
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

// Per frequency f over the slab: wmax[f] = max_p |w(p, f)|, the sign code wsgn[f]
// (+1 all weights >= 0, -1 all <= 0, 0 both signs), and the folded factors
// G[f][p] = sgn(w) sqrt(|w| / wmax) * 127 * 2^16 (0 past the slab's end).
__global__ void split_wstat_kernel(const double* __restrict__ W, int64_t ldw, int64_t p0, int len,
                                   int lenp, double* __restrict__ wmax, int* __restrict__ wsgn,
                                   double* __restrict__ G) {
  const int f = blockIdx.x;
  const double* wf = W + (int64_t)f * ldw + p0;
  double m = 0.0;
  int pos = 0, neg = 0;
  for (int p = threadIdx.x; p < len; p += blockDim.x) {
    const double w = wf[p];
    m = fmax(m, fabs(w));
    pos |= w > 0.0;
    neg |= w < 0.0;
  }
  for (int o = 16; o > 0; o >>= 1) {
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    pos |= __shfl_xor_sync(0xffffffffu, pos, o);
    neg |= __shfl_xor_sync(0xffffffffu, neg, o);
  }
  __shared__ double red[32];
  __shared__ int rpos[32], rneg[32];
  __shared__ double wm_s;
  if ((threadIdx.x & 31) == 0) {
    red[threadIdx.x >> 5] = m;
    rpos[threadIdx.x >> 5] = pos;
    rneg[threadIdx.x >> 5] = neg;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const bool v = threadIdx.x < (blockDim.x >> 5);
    m = v ? red[threadIdx.x] : 0.0;
    pos = v ? rpos[threadIdx.x] : 0;
    neg = v ? rneg[threadIdx.x] : 0;
    for (int o = 16; o > 0; o >>= 1) {
      m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
      pos |= __shfl_xor_sync(0xffffffffu, pos, o);
      neg |= __shfl_xor_sync(0xffffffffu, neg, o);
    }
    if (threadIdx.x == 0) {
      wmax[f] = m;
      wsgn[f] = (pos && neg) ? 0 : (neg ? -1 : 1);
      wm_s = m;
    }
  }
  __syncthreads();
  const double wm = wm_s;
  double* gf = G + (int64_t)f * lenp;
  for (int p = threadIdx.x; p < lenp; p += blockDim.x) {
    gf[p] = p < len ? fold_factor(wf[p], wm) : 0.0;
  }
}

// One thread = one complex column i and 8 consecutive pairs of the slab. Digit
// planes are stored [plane][k-block of 64 pairs][row][64 bytes]; a warp holds 4
// consecutive columns x the eight 8-pair pieces of one k-block, so its stores cover
// 8 adjacent rows x 64 bytes, and the TMA box (64 B, rows, 1 k-block, planes) lands
// as [plane][row][64 B] in shared memory. Rows interleave the parts: column i ->
// rows 128 (i / 64) + 2 (i % 64) (Re) and the next one (Im). For frequency f the
// planes f*6 + t hold the digits t of round(x |G| / s) (the folded operand), and,
// when the frequency's weights have both signs, planes f*6 + 3 + t those of
// round(x G / s). A block is 16 columns x one 64-pair k-block; the block stages the
// folded factors of its 64 pairs (SPQ_FCH frequencies at a time) in shared memory,
// so the frequency loop waits on no L2 round trip. The kernel is bound by the HBM
// writes of the planes; 96 registers keep five blocks per SM.
constexpr int SPQ_FCH = 24;
__global__ void __maxnreg__(96)
    split_quantize_kernel(const double2* __restrict__ M, int64_t ldc, int64_t p0, int len,
                          int nchunk, int N, int npad, int64_t R, int64_t Ps, int nw,
                          const double* __restrict__ sA, const int* __restrict__ wsgn,
                          const double* __restrict__ G, int8_t* __restrict__ F) {
  __shared__ __align__(16) double gs[SPQ_FCH][SP_KB];
  __shared__ int ss[SPQ_FCH];
  // thread -> (k-block, column group of 4, eighth of the k-block, column in group); the
  // 4 warps of a block share the k-block (npad / 4 is a multiple of 4)
  const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const bool active = tid < (int64_t)npad * nchunk * 2;
  const int ngroup = npad / 4;
  const int lane4 = (int)(tid & 3), eighth = (int)((tid >> 2) & 7);
  const int64_t rest = tid >> 5;
  const int i = (int)(rest % ngroup) * 4 + lane4;
  const int64_t kb = ((blockIdx.x * (int64_t)blockDim.x) >> 5) / ngroup;  // the block's k-block
  const int p = (int)(kb * SP_KB) + eighth * 8;
  const int lenp = nchunk * 16;
  const int64_t nkb = Ps / SP_KB;
  // planes are nkb * R * 64 bytes apart
  const int64_t pstride = nkb * R * SP_KB;
  const int64_t o_re = (kb * R + split_row_re(i)) * SP_KB + eighth * 8;
  const bool col_ok = active && i < N;
  const double2* col = M + (int64_t)(col_ok ? i : 0) * ldc + p0;
  double xr[8], xi[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    double2 v = make_double2(0.0, 0.0);
    if (col_ok && p + k < len) v = __ldg(col + p + k);
    xr[k] = v.x;
    xi[k] = v.y;
  }
  const double s = col_ok ? sA[i] : 0.0;
  const double inv = s > 0.0 ? 1.0 / s : 0.0;
  for (int f0 = 0; f0 < nw; f0 += SPQ_FCH) {
    const int nf = min(SPQ_FCH, nw - f0);
    __syncthreads();  // the previous chunk's factors are consumed
    // 16-byte chunk c = 4 e + j (eighth e, chunk j of its 8 pairs) is kept at
    // 4 e + (j ^ ((e >> 1) & 3)): the eight eighths a warp reads at once fall in
    // distinct banks
    for (int e = threadIdx.x; e < nf * (SP_KB / 2); e += blockDim.x) {
      const int f = e / (SP_KB / 2), c = e - f * (SP_KB / 2);
      const int ce = c >> 2, cj = c & 3;
      reinterpret_cast<double2*>(&gs[f][0])[4 * ce + (cj ^ ((ce >> 1) & 3))] =
          __ldg(reinterpret_cast<const double2*>(G + (int64_t)(f0 + f) * lenp + kb * SP_KB) + c);
    }
    for (int f = threadIdx.x; f < nf; f += blockDim.x) ss[f] = wsgn[f0 + f];
    __syncthreads();
    if (!active) continue;
#pragma unroll 1
    for (int f = 0; f < nf; ++f) {
      const bool mixed = ss[f] == 0;
      const double2* gq2 = reinterpret_cast<const double2*>(&gs[f][eighth * 8]);
      const int sw = (eighth >> 1) & 3;
      uint32_t ar[SP_SF][2], ai[SP_SF][2], br[SP_SF][2], bim[SP_SF][2];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        uint32_t yr[4], yi[4], pr[SP_SF], pi[SP_SF];
        double gq[4];
        const double2 g01 = gq2[(2 * q) ^ sw], g23 = gq2[(2 * q + 1) ^ sw];
        gq[0] = g01.x * inv, gq[1] = g01.y * inv, gq[2] = g23.x * inv, gq[3] = g23.y * inv;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const double ga = fabs(gq[e]);
          yr[e] = round_mul(xr[4 * q + e], ga);
          yi[e] = round_mul(xi[4 * q + e], ga);
        }
        digit_planes<SP_SF>(yr, pr);
        digit_planes<SP_SF>(yi, pi);
#pragma unroll
        for (int t = 0; t < SP_SF; ++t) ar[t][q] = pr[t], ai[t][q] = pi[t];
        if (mixed) {
#pragma unroll
          for (int e = 0; e < 4; ++e)
            if (gq[e] < 0.0) yr[e] = 0u - yr[e], yi[e] = 0u - yi[e];
          digit_planes<SP_SF>(yr, pr);
          digit_planes<SP_SF>(yi, pi);
#pragma unroll
          for (int t = 0; t < SP_SF; ++t) br[t][q] = pr[t], bim[t][q] = pi[t];
        }
      }
#pragma unroll
      for (int t = 0; t < SP_SF; ++t) {
        const int64_t plane = (int64_t)(f0 + f) * SP_SLOT + t;
        *reinterpret_cast<uint2*>(F + o_re + plane * pstride) = make_uint2(ar[t][0], ar[t][1]);
        *reinterpret_cast<uint2*>(F + o_re + SP_KB + plane * pstride) = make_uint2(ai[t][0], ai[t][1]);
      }
      if (mixed) {
#pragma unroll
        for (int t = 0; t < SP_SF; ++t) {
          const int64_t plane = (int64_t)(f0 + f) * SP_SLOT + SP_SF + t;
          *reinterpret_cast<uint2*>(F + o_re + plane * pstride) = make_uint2(br[t][0], br[t][1]);
          *reinterpret_cast<uint2*>(F + o_re + SP_KB + plane * pstride) = make_uint2(bim[t][0], bim[t][1]);
        }
      }
    }
  }
}

// -DINV (real M): column scales and digit planes with one plane row per column
// (rows 128 b .. 128 b + 127 hold the columns of 128-block b).
__global__ void split_colmax_real_kernel(const double* __restrict__ M, int64_t ldc, int64_t p0,
                                         int len, double* __restrict__ sA) {
  const int i = blockIdx.x;
  const double* col = M + (int64_t)i * ldc + p0;
  double m = 0.0;
  for (int p = threadIdx.x; p < len; p += blockDim.x) m = fmax(m, fabs(col[p]));
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

__global__ void __launch_bounds__(128, 4)
    split_quantize_real_kernel(const double* __restrict__ M, int64_t ldc, int64_t p0, int len,
                               int nchunk, int N, int npad, int64_t R, int64_t Ps, int nw,
                               const double* __restrict__ sA, const int* __restrict__ wsgn,
                               const double* __restrict__ G, int8_t* __restrict__ F) {
  const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (tid >= (int64_t)npad * nchunk) return;
  const int ngroup = npad / 8;
  const int lane8 = (int)(tid & 7), quarter = (int)((tid >> 3) & 3);
  const int64_t rest = tid >> 5;
  const int i = (int)(rest % ngroup) * 8 + lane8;
  const int64_t kb = rest / ngroup;
  const int p = (int)(kb * SP_KB) + quarter * 16;
  const int64_t pstride = (Ps / SP_KB) * R * SP_KB;
  const bool col_ok = i < N;
  quantize_task_real(M + (int64_t)(col_ok ? i : 0) * ldc + p0, col_ok, len, p, col_ok ? sA[i] : 0.0,
                     (kb * R + i) * SP_KB + quarter * 16, pstride, nw, wsgn, G, nchunk * 16, F);
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

// Generic tiled tensor map (no context): 0 on success, -1 without the driver entry
// point, else the driver's error code.
int encode_tmap(CUtensorMap* map, CUtensorMapDataType type, int rank, const void* base,
                const uint64_t* dims, const uint64_t* strides, const uint32_t* box,
                CUtensorMapSwizzle swz) {
  auto enc = get_encode();
  if (!enc) return -1;
  cuuint64_t d[5], st[4];
  cuuint32_t b[5], es[5];
  for (int i = 0; i < rank; ++i) {
    d[i] = dims[i];
    b[i] = box[i];
    es[i] = 1;
    if (i + 1 < rank) st[i] = strides[i];
  }
  return (int)enc(map, type, (cuuint32_t)rank, const_cast<void*>(base), d, st, b, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
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
  size_t f_bytes, g_bytes, s_bytes, w_bytes, sg_bytes;
};

// slab: band pairs per exact int32 slab, a multiple of SP_KB in [SP_KB, SP_SLAB]
static SplitLayout split_layout(int64_t P, int N, int nw, int slab = SP_SLAB) {
  SplitLayout L;
  L.Ps = std::min<int64_t>((int64_t)align_up((size_t)std::max<int64_t>(P, 1), SP_KB), slab);
  L.nblk = (N + SP_TILE - 1) / SP_TILE;
  // an even number of 64-blocks, so a CTA pair's second A tile always exists
  L.R = (int64_t)((L.nblk + 1) / 2 * 2) * SP_ROWS;
  L.f_bytes = align_up((size_t)SP_SLOT * nw * L.R * L.Ps, 1024);
  L.g_bytes = align_up(sizeof(double) * (size_t)nw * L.Ps, 256);
  L.s_bytes = align_up(sizeof(double) * (size_t)std::max(N, 1), 256);
  L.w_bytes = align_up(sizeof(double) * (size_t)std::max(nw, 1), 256);
  L.sg_bytes = align_up(sizeof(int) * (size_t)std::max(nw, 1), 256);
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
  return split_nbuf(P, slab) * (L.f_bytes + L.g_bytes + L.s_bytes + L.w_bytes + L.sg_bytes) + 1024;
}
size_t split_workspace_bytes(int64_t P, int N, int nw) {
  return split_workspace_bytes(P, N, nw, SP_SLAB);
}

void timing_mark(spx_ctx* ctx, cudaStream_t s, int kind);

// variant: 1 one CTA per 64 x 64 tile, 2 CTA pair, 5 one CTA per 64 x 80 tile, 0 the
// context's choice; slab: pairs per exact int32 slab (0 = 32768).
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
  const size_t set_bytes = L.f_bytes + L.g_bytes + L.s_bytes + L.w_bytes + L.sg_bytes;
  int8_t* F[2];
  double* G[2];
  double* sA[2];
  double* wmax[2];
  int* wsgn[2];
  for (int b = 0; b < 2; ++b) {
    uint8_t* s0 = base + (size_t)(b < nbuf ? b : 0) * set_bytes;
    F[b] = (int8_t*)s0;
    G[b] = (double*)(s0 + L.f_bytes);
    sA[b] = (double*)(s0 + L.f_bytes + L.g_bytes);
    wmax[b] = (double*)(s0 + L.f_bytes + L.g_bytes + L.s_bytes);
    wsgn[b] = (int*)(s0 + L.f_bytes + L.g_bytes + L.s_bytes + L.w_bytes);
  }

  // planes in HBM: [plane][k-block][row][K bytes]; TMA dims (K, row, k-block, plane)
  // with increasing strides; a box (K, rows, 1, 3 planes) lands as [plane][row][K]
  const uint64_t nkb = (uint64_t)(L.Ps / SP_KB);
  if (variant == 0) variant = ctx->opt.split_variant;
  if (variant == 0) variant = 5;  // untuned: one CTA per 64 x 80 tile
  const bool pair = variant == 2;
  const bool wide = variant == 5;                  // one CTA per 64 x 80 tile (N = 160)
  // only the CTA pair needs an even number of 64-column blocks in the planes (the
  // buffers are sized for it either way)
  if (!pair) L.R = (int64_t)L.nblk * SP_ROWS;
  CUtensorMap mapF[2], mapFh[2], mapW[2];
  for (int b = 0; b < nbuf; ++b) {
    const uint64_t st[3] = {SP_KB, (uint64_t)L.R * SP_KB, nkb * L.R * SP_KB};
    const uint64_t d[4] = {SP_KB, (uint64_t)L.R, nkb, (uint64_t)SP_SLOT * nw};
    const uint32_t bx[4] = {SP_KB, SP_ROWS, 1, SP_SF};
    int rc0 = make_tmap_u8_4d(ctx, &mapF[b], F[b], d, st, bx, CU_TENSOR_MAP_SWIZZLE_64B);
    if (rc0) return rc0;
    const uint32_t bh[4] = {SP_KB, SP2_BROWS, 1, SP_SF};
    rc0 = make_tmap_u8_4d(ctx, &mapFh[b], F[b], d, st, bh, CU_TENSOR_MAP_SWIZZLE_64B);
    if (rc0) return rc0;
    const uint32_t bw[4] = {SP_KB, 2 * SP_WIDE_BN, 1, SP_SF};
    rc0 = make_tmap_u8_4d(ctx, &mapW[b], F[b], d, st, bw, CU_TENSOR_MAP_SWIZZLE_64B);
    if (rc0) return rc0;
  }
  int rc = SPX_OK;

  const size_t smem = sizeof(SplitSmem) + 1024;
  const size_t smemw = sizeof(SplitSmemT<2 * SP_WIDE_BN>) + 1024;
  const size_t smem2 = sizeof(Split2Smem) + 1024;
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(split_gram_kernel<false, SP_TILE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(split_gram_kernel<false, SP_WIDE_BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemw);
    cudaFuncSetAttribute(split_gram_kernel<true, SP_TILE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(split_gram2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem2);
    attr_set = true;
  }
  const int nbr = (N + SP_TILE - 1) / SP_TILE;
  const int ntile = L.nblk * (L.nblk + 1) / 2;
  int ntile2 = 0, ntilew = 0;
  for (int bj = 0; bj < L.nblk; ++bj) ntile2 += bj / 2 + 1;
  for (int bj = 0; bj * SP_WIDE_BN < N; ++bj) ntilew += split_rows_of(bj, SP_WIDE_BN, nbr);
  const int ntile_used = pair ? ntile2 : (wide ? ntilew : ntile);
  const int nitems = ntile_used * nw;
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

  // Preparation (column scales, weight statistics, digit planes) of slab s+1 runs on
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
    split_wstat_kernel<<<nw, 256, 0, ps>>>(W, ldw, p0, len, lenp, wmax[b], wsgn[b], G[b]);
    const int64_t nthr = (int64_t)npad * nchunk * 2;  // 8-pair tasks
    split_quantize_kernel<<<(unsigned)((nthr + 127) / 128), 128, 0, ps>>>(
        M, ldc, p0, len, nchunk, N, npad, L.R, L.Ps, nw, sA[b], wsgn[b], G[b], F[b]);
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
    prm.nbr = nbr;
    prm.ntile = ntile_used;
    prm.nw = nw;
    prm.nitems = nitems;
    prm.nk = lenp / SP_KB;
    prm.sA = sA[b];
    prm.wmax = wmax[b];
    prm.wsgn = wsgn[b];
    prm.out = reinterpret_cast<double*>(out);
    prm.npack = (int64_t)N * (N + 1) / 2;
    prm.status = ctx->d_status;
    prm.timeout_ns =
        (uint64_t)(ctx->opt.timeout_ms > 0 ? ctx->opt.timeout_ms : 4000) * 1000000ull;
    if (pair) {
      rc = check_cuda(ctx, cudaLaunchKernelEx(&cfg, split_gram2_kernel, mapF[b], mapFh[b], prm),
                      "split_gram2_kernel launch");
    } else if (wide) {
      split_gram_kernel<false, SP_WIDE_BN><<<grid, SP1_THREADS, smemw, stream>>>(mapF[b], mapW[b], prm);
      rc = check_cuda(ctx, cudaGetLastError(), "split_gram_kernel (64 x 80) launch");
    } else {
      split_gram_kernel<false, SP_TILE><<<grid, SP1_THREADS, smem, stream>>>(mapF[b], mapF[b], prm);
      rc = check_cuda(ctx, cudaGetLastError(), "split_gram_kernel launch");
    }
    if (rc) return rc;
    *launches += 1;
    timing_mark(ctx, stream, 2);  // the accumulation interval ends with the kernel
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

// Real layout: 128 columns per block, one plane row per column.
static SplitLayout split_layout_real(int64_t P, int N, int nw, int slab) {
  SplitLayout L = split_layout(P, 1, nw, slab);
  L.nblk = (N + SP_ROWS - 1) / SP_ROWS;
  L.R = (int64_t)L.nblk * SP_ROWS;
  L.f_bytes = align_up((size_t)SP_SLOT * nw * L.R * L.Ps, 1024);
  L.s_bytes = align_up(sizeof(double) * (size_t)std::max(N, 1), 256);
  return L;
}

size_t split_workspace_bytes_real(int64_t P, int N, int nw) {
  SplitLayout L = split_layout_real(P, N, nw, SP_SLAB);
  return split_nbuf(P, SP_SLAB) * (L.f_bytes + L.g_bytes + L.s_bytes + L.w_bytes + L.sg_bytes) + 1024;
}

// The -DINV accumulation (src/susceptibility.f:1197, re(k) = cprod(k,i) * cprod(k,j)):
// real M (ldc, N), real packed out (npack, nw), the folded 6-product int8 contraction
// on 128 x 160 real tiles (N = 160 MMAs; 128 x 128 when the context's split variant is
// 1), one CTA per tile.
int split_chi0_real_slab(spx_ctx* ctx, const double* M, int64_t ldc, int64_t P, int N,
                         const double* W, int64_t ldw, int nw, double* out, void* ws,
                         size_t ws_bytes, cudaStream_t stream, int* launches) {
  if (P <= 0 || N <= 0 || nw <= 0) return SPX_OK;
  SplitLayout L = split_layout_real(P, N, nw, SP_SLAB);
  if (!ws || ws_bytes < split_workspace_bytes_real(P, N, nw))
    return set_error(ctx, SPX_EINVAL, "split workspace too small");
  uint8_t* base = (uint8_t*)align_up((size_t)ws, 1024);
  const int nbuf = split_nbuf(P, SP_SLAB);
  const size_t set_bytes = L.f_bytes + L.g_bytes + L.s_bytes + L.w_bytes + L.sg_bytes;
  int8_t* F[2];
  double *G[2], *sA[2], *wmax[2];
  int* wsgn[2];
  for (int b = 0; b < 2; ++b) {
    uint8_t* s0 = base + (size_t)(b < nbuf ? b : 0) * set_bytes;
    F[b] = (int8_t*)s0;
    G[b] = (double*)(s0 + L.f_bytes);
    sA[b] = (double*)(s0 + L.f_bytes + L.g_bytes);
    wmax[b] = (double*)(s0 + L.f_bytes + L.g_bytes + L.s_bytes);
    wsgn[b] = (int*)(s0 + L.f_bytes + L.g_bytes + L.s_bytes + L.w_bytes);
  }
  const uint64_t nkb = (uint64_t)(L.Ps / SP_KB);
  const bool wide = ctx->opt.split_variant != 1;
  CUtensorMap mapF[2], mapW[2];
  for (int b = 0; b < nbuf; ++b) {
    const uint64_t st[3] = {SP_KB, (uint64_t)L.R * SP_KB, nkb * L.R * SP_KB};
    const uint64_t d[4] = {SP_KB, (uint64_t)L.R, nkb, (uint64_t)SP_SLOT * nw};
    const uint32_t bx[4] = {SP_KB, SP_ROWS, 1, SP_SF};
    int rc0 = make_tmap_u8_4d(ctx, &mapF[b], F[b], d, st, bx, CU_TENSOR_MAP_SWIZZLE_64B);
    if (rc0) return rc0;
    const uint32_t bw[4] = {SP_KB, 2 * SP_WIDE_BN, 1, SP_SF};
    rc0 = make_tmap_u8_4d(ctx, &mapW[b], F[b], d, st, bw, CU_TENSOR_MAP_SWIZZLE_64B);
    if (rc0) return rc0;
  }
  const size_t smem = sizeof(SplitSmem) + 1024;
  const size_t smemw = sizeof(SplitSmemT<2 * SP_WIDE_BN>) + 1024;
  cudaFuncSetAttribute(split_gram_kernel<true, SP_TILE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaFuncSetAttribute(split_gram_kernel<true, SP_WIDE_BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemw);
  // tiles in 128-row blocks of the real rows; wide tiles in 160-column blocks
  const int nbr = L.nblk;
  int ntilew = 0;
  for (int bj = 0; bj * 2 * SP_WIDE_BN < N; ++bj) ntilew += split_rows_of(bj, SP_WIDE_BN, nbr);
  const int ntile = wide ? ntilew : L.nblk * (L.nblk + 1) / 2;
  const int nitems = ntile * nw;
  const int grid = std::min(nitems, ctx->num_sms);
  const int npad = (int)L.R;
  const int64_t nslab = (P + L.Ps - 1) / L.Ps;
  cudaStream_t ps = ctx->prep_stream;
  cudaEvent_t ev_start = ctx->sev[0];
  cudaEvent_t prep_done[2] = {ctx->sev[1], ctx->sev[2]};
  cudaEvent_t gram_done[2] = {ctx->sev[3], ctx->sev[4]};
  int rc;
  auto prep = [&](int64_t s) -> int {
    const int b = (int)(s % nbuf);
    const int64_t p0 = s * L.Ps;
    const int len = (int)std::min<int64_t>(L.Ps, P - p0);
    const int lenp = (int)align_up((size_t)len, SP_KB);
    const int nchunk = lenp / 16;
    split_colmax_real_kernel<<<N, 256, 0, ps>>>(M, ldc, p0, len, sA[b]);
    split_wstat_kernel<<<nw, 256, 0, ps>>>(W, ldw, p0, len, lenp, wmax[b], wsgn[b], G[b]);
    const int64_t nthr = (int64_t)npad * nchunk;
    split_quantize_real_kernel<<<(unsigned)((nthr + 127) / 128), 128, 0, ps>>>(
        M, ldc, p0, len, nchunk, N, npad, L.R, L.Ps, nw, sA[b], wsgn[b], G[b], F[b]);
    int r = check_cuda(ctx, cudaGetLastError(), "split operand preparation (real)");
    if (r) return r;
    *launches += 3;
    return check_cuda(ctx, cudaEventRecord(prep_done[b], ps), "event");
  };
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
    if (nbuf == 2 && s >= 1 && s + 1 < nslab &&
        (rc = check_cuda(ctx, cudaStreamWaitEvent(ps, gram_done[(s + 1) % 2], 0), "event")))
      return rc;
    timing_mark(ctx, stream, 1);
    SplitParams prm;
    prm.N = N;
    prm.nbr = nbr;
    prm.ntile = ntile;
    prm.nw = nw;
    prm.nitems = nitems;
    prm.nk = lenp / SP_KB;
    prm.sA = sA[b];
    prm.wmax = wmax[b];
    prm.wsgn = wsgn[b];
    prm.out = out;
    prm.npack = (int64_t)N * (N + 1) / 2;
    prm.status = ctx->d_status;
    prm.timeout_ns = (uint64_t)(ctx->opt.timeout_ms > 0 ? ctx->opt.timeout_ms : 4000) * 1000000ull;
    if (wide)
      split_gram_kernel<true, SP_WIDE_BN><<<grid, SP1_THREADS, smemw, stream>>>(mapF[b], mapW[b], prm);
    else
      split_gram_kernel<true, SP_TILE><<<grid, SP1_THREADS, smem, stream>>>(mapF[b], mapF[b], prm);
    if ((rc = check_cuda(ctx, cudaGetLastError(), "split_gram_kernel (real) launch"))) return rc;
    *launches += 1;
    timing_mark(ctx, stream, 2);
    if ((rc = check_cuda(ctx, cudaEventRecord(gram_done[b], stream), "event"))) return rc;
    if (s + 1 < nslab) {
      if (nbuf == 1 && (rc = check_cuda(ctx, cudaStreamWaitEvent(ps, gram_done[0], 0), "event")))
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
// concurrent CTAs share the large B tile through L2. The epilogue stages alpha times
// the tile in shared memory and writes (or adds) it into cprod's columns as runs of
// 32 consecutive complex values.

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
  int overwrite;           // 1: store (the output range holds nothing yet), 0: add
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
  long long xchg[2][SP_TILE][SG_TB];   // the Re-row and Im-row products, column k ^ (row & 15)
  double2 stage[SP_TILE][SG_TB];       // the output tile, column k ^ (row & 31)
  uint64_t full[SG_ST];
  uint64_t empty[SG_ST];
  uint64_t tfull[2], tempty[2];
  uint64_t xfull, xstage, xfree, mdone;
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
    mbar_init(&sm.xstage, 4);
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
      // the previous tile's staged values have been written out
      if (!mbar_wait(&sm.xfree, (xseq & 1u) ^ 1u, prm.timeout_ns, prm.status)) break;
#pragma unroll
      for (int k = 0; k < 32; ++k) sm.xchg[is_re ? 0 : 1][ii][k ^ (ii & 15)] = tim[k];
      __syncwarp();
      if (lane == 0) mbar_arrive(&sm.xfull);
      if (!mbar_wait(&sm.xfull, xseq & 1u, prm.timeout_ns, prm.status)) break;
      // this thread's part (Re or Im) of row ii, 32 columns, into the staged tile
      double* st = reinterpret_cast<double*>(&sm.stage[ii][0]) + (is_re ? 0 : 1);
#pragma unroll
      for (int k = 0; k < 32; ++k) {
        const long long partner = sm.xchg[is_re ? 1 : 0][ii][k ^ (ii & 15)];
        const long long v = is_re ? tre[k] + partner : tre[k] - partner;
        st[2 * (k ^ lane)] = fac * sbb[ct * SG_TB + k] * (double)v;
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&sm.xstage);
      if (!mbar_wait(&sm.xstage, xseq & 1u, prm.timeout_ns, prm.status)) break;
      // write out: warp q takes columns q, q + 4, ...; a lane one row of the two 32-row
      // halves, so each store is 32 consecutive complex values of one cprod column
      // (whole 32-byte sectors). Each element belongs to one thread of one launch.
      double2* ob = reinterpret_cast<double2*>(prm.out) + b * prm.sO2 + mt * SP_TILE;
#pragma unroll 2
      for (int k = q; k < SG_TB; k += 4) {
        const int gc = ct * SG_TB + k;
        if (gc >= prm.ncol) break;
        const int n = gc / prm.ncin, c = gc - n * prm.ncin;
        double2* oc = ob + n * prm.sOn + c * prm.sOc;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int row = 32 * h + lane;
          if (mt * SP_TILE + row >= prm.M) continue;
          const double2 v = sm.stage[row][k ^ lane];
          if (prm.overwrite) {
            oc[row] = v;
          } else {
            double2 o = oc[row];
            o.x += v.x;
            o.y += v.y;
            oc[row] = o;
          }
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
                   size_t ws_bytes, cudaStream_t s, int* launches, bool overwrite) {
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
    prm.overwrite = overwrite && kbeg == 0;  // later K slabs add to the first
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
