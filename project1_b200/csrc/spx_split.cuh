// Device code shared by the split-precision accumulation kernels (one call, and the
// persistent batched schedule): the digit-plane layout, the HILBERT NONE weight,
// the folded factors, the quantizer task and the TMEM read-back. Both schedules use
// these functions, so equal slabs give equal bits.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "spx_common.cuh"
#include "spx_tcgen05.cuh"

namespace spx {

constexpr int SP_TILE = 64;            // complex rows / columns per tile
constexpr int SP_ROWS = 128;           // real-stacked rows per tile (re/im interleaved)
constexpr int SP_KB = 64;              // band pairs (bytes) per pipeline stage: two MMA K steps
constexpr int SP_KSTEP = 32;           // int8 MMA K
constexpr int SP_NKS = SP_KB / SP_KSTEP;
constexpr int SP_SA = 3;               // digit slices of the product GEMM's A operand
constexpr int SP_SB = 4;               // digit slices of the product GEMM's B operand
constexpr int SP_SF = 3;               // digit slices of a folded accumulation operand
constexpr int SP_SLOT = 2 * SP_SF;     // planes per frequency: folded A, signed B (mixed signs)
constexpr int SP_SLAB = 32768;         // band pairs per exact int32 accumulation
constexpr int SP_PLANE = SP_ROWS * SP_KB;  // bytes of one slice of one stage
constexpr int SP_TMEM_COLS = 512;      // power-of-two allocation holding 3 orders x 128 columns
constexpr double SP_QF = 127.0 * 65536.0;  // integer scale of a 3-digit value

// idesc for kind::i8: D s32 (bits 4-5 = 2), A/B signed int8 (bits 7-9, 10-12 = 1),
// K-major A and B, N (bits 17-22 = N/8), M = 128 (bits 24-28 = M/16).
constexpr uint32_t sp_idesc(int n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n / 8) << 17) | ((uint32_t)(SP_ROWS / 16) << 24);
}
constexpr uint32_t SP_IDESC = sp_idesc(SP_ROWS);

#if defined(__CUDACC__)
// HILBERT NONE weight of src/susceptibility.f:950-975 for rdum = d, frqh/img = om,
// nkpts(k)/nkpt/nsym1 = s, with an explicit operation order (the same bits in
// every kernel that needs it).
__device__ __forceinline__ double hilbert_none_weight(double d, double om, double s) {
  return __dmul_rn(__ddiv_rn(__dmul_rn(-2.0, d), __fma_rn(om, om, __dmul_rn(d, d))), s);
}

// Folded factor of a weight: sgn(w) sqrt(|w| / wmax) * 127 * 2^16 (0 if wmax = 0).
__device__ __forceinline__ double fold_factor(double w, double wm) {
  if (!(wm > 0.0)) return 0.0;
  const double g = __dmul_rn(__dsqrt_rn(__ddiv_rn(fabs(w), wm)), SP_QF);
  return w < 0.0 ? -g : g;
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

// Real-stacked row of the real part of column i: rows interleave the parts, column
// i -> 128 (i / 64) + 2 (i % 64) (Re) and the next row (Im).
__device__ __forceinline__ int64_t split_row_re(int i) {
  return (int64_t)(i / SP_TILE) * SP_ROWS + 2 * (i % SP_TILE);
}

// One quantizer task: column i and the 16 pairs [p, p+16) of a slab of `len` pairs
// (`lenp` padded to 64). `col` points at M(p0 .. , i) (pairs contiguous). Planes are
// [plane][k-block of 64 pairs][row][64 bytes], `pstride` bytes apart; for frequency
// f, planes f*6 + t hold digit t of round(x |G| / s) (the folded operand) and, when
// the frequency's weights have both signs, planes f*6 + 3 + t those of
// round(x G / s). G[f*lenp + p] are the folded factors of the slab.
__device__ __forceinline__ void quantize_task(const double2* __restrict__ col, bool col_ok, int len,
                                              int p, double s, int64_t o_re, int64_t pstride,
                                              int nw, const int* __restrict__ wsgn,
                                              const double* __restrict__ G, int lenp,
                                              int8_t* __restrict__ F) {
  const int64_t o_im = o_re + SP_KB;
  double xr[16], xi[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    double2 v = make_double2(0.0, 0.0);
    if (col_ok && p + k < len) v = __ldg(col + p + k);
    xr[k] = v.x;
    xi[k] = v.y;
  }
  const double inv = s > 0.0 ? 1.0 / s : 0.0;
  for (int f = 0; f < nw; ++f) {
    const double* gf = G + (int64_t)f * lenp + p;
    double g[16];
#pragma unroll
    for (int k = 0; k < 16; k += 2) {
      const double2 v = *reinterpret_cast<const double2*>(gf + k);
      g[k] = v.x * inv;
      g[k + 1] = v.y * inv;
    }
    const bool mixed = wsgn[f] == 0;
    uint32_t ar[SP_SF][4], ai[SP_SF][4], br[SP_SF][4], bim[SP_SF][4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      uint32_t yr[4], yi[4], pr[SP_SF], pi[SP_SF];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const double ga = fabs(g[4 * q + e]);
        yr[e] = round_mul(xr[4 * q + e], ga);
        yi[e] = round_mul(xi[4 * q + e], ga);
      }
      digit_planes<SP_SF>(yr, pr);
      digit_planes<SP_SF>(yi, pi);
#pragma unroll
      for (int t = 0; t < SP_SF; ++t) ar[t][q] = pr[t], ai[t][q] = pi[t];
      if (mixed) {
        // the signed operand: the same integers, negated where w < 0 (rounding to
        // nearest is symmetric, so these are the digits of round(x G / s))
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          if (g[4 * q + e] < 0.0) yr[e] = 0u - yr[e], yi[e] = 0u - yi[e];
        }
        digit_planes<SP_SF>(yr, pr);
        digit_planes<SP_SF>(yi, pi);
#pragma unroll
        for (int t = 0; t < SP_SF; ++t) br[t][q] = pr[t], bim[t][q] = pi[t];
      }
    }
#pragma unroll
    for (int t = 0; t < SP_SF; ++t) {
      const int64_t plane = (int64_t)f * SP_SLOT + t;
      *reinterpret_cast<uint4*>(F + o_re + plane * pstride) = make_uint4(ar[t][0], ar[t][1], ar[t][2], ar[t][3]);
      *reinterpret_cast<uint4*>(F + o_im + plane * pstride) = make_uint4(ai[t][0], ai[t][1], ai[t][2], ai[t][3]);
    }
    if (mixed) {
#pragma unroll
      for (int t = 0; t < SP_SF; ++t) {
        const int64_t plane = (int64_t)f * SP_SLOT + SP_SF + t;
        *reinterpret_cast<uint4*>(F + o_re + plane * pstride) = make_uint4(br[t][0], br[t][1], br[t][2], br[t][3]);
        *reinterpret_cast<uint4*>(F + o_im + plane * pstride) = make_uint4(bim[t][0], bim[t][1], bim[t][2], bim[t][3]);
      }
    }
  }
}

// The real (-DINV) form of quantize_task: column i of a real M, one plane row per
// column (`o` its byte offset in plane 0).
__device__ __forceinline__ void quantize_task_real(const double* __restrict__ col, bool col_ok,
                                                   int len, int p, double s, int64_t o,
                                                   int64_t pstride, int nw,
                                                   const int* __restrict__ wsgn,
                                                   const double* __restrict__ G, int lenp,
                                                   int8_t* __restrict__ F) {
  double x[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) x[k] = (col_ok && p + k < len) ? __ldg(col + p + k) : 0.0;
  const double inv = s > 0.0 ? 1.0 / s : 0.0;
  for (int f = 0; f < nw; ++f) {
    const double* gf = G + (int64_t)f * lenp + p;
    const bool mixed = wsgn[f] == 0;
    uint32_t a[SP_SF][4], b[SP_SF][4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      uint32_t y[4], pd[SP_SF];
      bool neg[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const double g = gf[4 * q + e] * inv;
        neg[e] = g < 0.0;
        y[e] = round_mul(x[4 * q + e], fabs(g));
      }
      digit_planes<SP_SF>(y, pd);
#pragma unroll
      for (int t = 0; t < SP_SF; ++t) a[t][q] = pd[t];
      if (mixed) {
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (neg[e]) y[e] = 0u - y[e];
        digit_planes<SP_SF>(y, pd);
#pragma unroll
        for (int t = 0; t < SP_SF; ++t) b[t][q] = pd[t];
      }
    }
#pragma unroll
    for (int t = 0; t < SP_SF; ++t)
      *reinterpret_cast<uint4*>(F + o + ((int64_t)f * SP_SLOT + t) * pstride) = make_uint4(a[t][0], a[t][1], a[t][2], a[t][3]);
    if (mixed) {
#pragma unroll
      for (int t = 0; t < SP_SF; ++t)
        *reinterpret_cast<uint4*>(F + o + ((int64_t)f * SP_SLOT + SP_SF + t) * pstride) = make_uint4(b[t][0], b[t][1], b[t][2], b[t][3]);
    }
  }
}

// Upper-triangle tile t -> (bi, bj), bi <= bj, column-major over the triangle.
__device__ __forceinline__ void split_decode_tile(int t, int* bi, int* bj) {
  int j = (int)((sqrtf(8.0f * (float)t + 1.0f) - 1.0f) * 0.5f);
  while (j * (j + 1) / 2 > t) --j;
  while ((j + 1) * (j + 2) / 2 <= t) ++j;
  *bj = j;
  *bi = t - j * (j + 1) / 2;
}

// Tile t of the upper region for tiles of 64 rows x BN columns, column-major: column
// block bj holds row blocks 0 .. min((bj BN + BN - 1) / 64, nbr - 1) (nbr row blocks
// cover N). BN = 64 is the square case above.
__host__ __device__ __forceinline__ int split_rows_of(int bj, int bn, int nbr) {
  const int r = (bj * bn + bn - 1) / 64;
  return (r < nbr - 1 ? r : nbr - 1) + 1;
}
template <int BN>
__device__ __forceinline__ void split_decode_tile_bn(int t, int nbr, int* bi, int* bj) {
  if constexpr (BN == SP_TILE) {
    split_decode_tile(t, bi, bj);
  } else {
    int j = 0, c = 0;
    while (c + split_rows_of(j, BN, nbr) <= t) c += split_rows_of(j++, BN, nbr);
    *bj = j;
    *bi = t - c;
  }
}

// Tile of a frequency-major item when `grid` CTAs take items round-robin. A frequency's
// ntile tiles fall into two rounds of the grid: the first `a` of them beside the
// previous frequency's last tiles, the rest in the next round. The smaller part is made
// the one whose tiles cover the fewest panels (a prefix of the column-major order is
// the upper triangle of panels 0..p), so fewer panels are read again, from DRAM, in the
// round after. Every role of a CTA decodes an item the same way.
// `first` is the item number of the frequency's first tile.
__device__ __forceinline__ int split_round_tile(int t, int ntile, int64_t first, int grid) {
  const int a = grid - (int)(first % grid);
  return (a < ntile && a > ntile - a) ? ntile - 1 - t : t;
}
__device__ __forceinline__ int split_item_tile(int item, int ntile, int grid) {
  const int t = item % ntile;
  return split_round_tile(t, ntile, item - t, grid);
}

// K step `ks` of a CTA's j-th item: every second item runs the slab backwards, so it
// starts on the K blocks that the CTAs' previous items read last, which are the ones
// still in L2. The integer sums are exact, so the order does not change any bit.
__device__ __forceinline__ int split_k_order(int j, int ks, int nk) {
  return (j & 1) ? nk - 1 - ks : ks;
}

// 16 consecutive columns of this lane's row: the slab's exact integer sum
// (D0*256 + D1)*256 + D2 as doubles (|value| < 2^48, so every step is exact), with
// order g at TMEM columns [ostride g, ostride g + 16).
__device__ __forceinline__ void load_fold16(uint32_t taddr, uint32_t ostride, double (&T)[16]) {
  int32_t r0[16], r1[16], r2[16];
  tmem_ld16(taddr, r0);
  tmem_ld16(taddr + ostride, r1);
  tmem_ld16(taddr + 2 * ostride, r2);
  tmem_wait_ld();
#pragma unroll
  for (int k = 0; k < 16; ++k)
    T[k] = fma(fma((double)r0[k], 256.0, (double)r1[k]), 256.0, (double)r2[k]);
}

// Output factor of a tile row: sgn s_i wmax / (127^2 2^16) (times s_j per column).
__device__ __forceinline__ double fold_row_factor(int sg, double si, double wm) {
  return (sg < 0 ? -1.0 : 1.0) * si * wm * (1.0 / (127.0 * SP_QF));
}
#endif

}  // namespace spx
