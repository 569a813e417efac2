/*
 * Seeded synthetic inputs for the oracle side — TEST INFRASTRUCTURE ONLY.
 *
 * The CPU baseline and the checker regenerate the projections M_I,p here, so that
 * they never load the product library. The stream is the one the GPU library
 * draws (its kernels and its host generator): element (p, c) of an (rows x cols)
 * matrix holds stream elements 2*rows*(col0 + c) + 2p (real part) and the next
 * one (imaginary part), times `scale`. A pair of stream elements is one
 * Philox4x32-10 block (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
 * easy as 1, 2, 3", SC'11: ten rounds, multipliers 0xD2511F53 / 0xCD9E8D57, key
 * increments 0x9E3779B9 / 0xBB67AE85) turned into two normals by Box-Muller.
 * Identical bits need the identical sequence of IEEE-754 operations, so the
 * logarithm (2 atanh series in s = (m-1)/(m+1) through s^23, with ln 2 split into
 * the two parts published in fdlibm's e_log.c) and the sine / cosine of 2 pi u
 * (quarter-turn reduction, Taylor series through x^17 / x^18) are evaluated in the
 * same order as the library does, and this file is compiled without FMA
 * contraction. tests/test_inputs_oracle.py checks the bits against the library's
 * host generator.
 */
#include <stdint.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
  uint32_t x[4];
} block4;

static block4 philox10(block4 c, uint32_t k0, uint32_t k1) {
  for (int round = 0; round < 10; ++round) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c.x[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c.x[2];
    block4 n;
    n.x[0] = (uint32_t)(p1 >> 32) ^ c.x[1] ^ k0;
    n.x[1] = (uint32_t)p1;
    n.x[2] = (uint32_t)(p0 >> 32) ^ c.x[3] ^ k1;
    n.x[3] = (uint32_t)p0;
    c = n;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

/* ln x for finite normal x > 0 */
static double series_log(double x) {
  uint64_t bits;
  memcpy(&bits, &x, sizeof bits);
  int ex = (int)((bits >> 52) & 0x7ff) - 1023;
  bits = (bits & 0x000fffffffffffffull) | 0x3ff0000000000000ull;
  double m;
  memcpy(&m, &bits, sizeof m);
  if (m > 1.4142135623730951) {
    m = m * 0.5;
    ex += 1;
  }
  const double s = (m - 1.0) / (m + 1.0);
  const double z = s * s;
  static const double inv_odd[12] = {1.0 / 23.0, 1.0 / 21.0, 1.0 / 19.0, 1.0 / 17.0,
                                     1.0 / 15.0, 1.0 / 13.0, 1.0 / 11.0, 1.0 / 9.0,
                                     1.0 / 7.0,  1.0 / 5.0,  1.0 / 3.0,  1.0};
  double acc = inv_odd[0];
  for (int k = 1; k < 12; ++k) acc = acc * z + inv_odd[k];
  const double lnm = (2.0 * s) * acc;
  const double ln2_hi = 6.93147180369123816490e-01, ln2_lo = 1.90821492927058770002e-10;
  const double e = (double)ex;
  return e * ln2_hi + (e * ln2_lo + lnm);
}

/* sin and cos of 2 pi u, 0 <= u < 1 */
static void series_sincos_turns(double u, double* sn_out, double* cs_out) {
  const double q = u * 4.0;
  const double n = (double)(int64_t)(q + 0.5);
  const double x = (q - n) * 1.57079632679489661923;
  const double z = x * x;
  static const double sin_c[8] = {-1.0 / 355687428096000.0, 1.0 / 1307674368000.0,
                                  -1.0 / 6227020800.0,      1.0 / 39916800.0,
                                  -1.0 / 362880.0,          1.0 / 5040.0,
                                  -1.0 / 120.0,             1.0 / 6.0};
  static const double cos_c[9] = {1.0 / 6402373705728000.0, -1.0 / 20922789888000.0,
                                  1.0 / 87178291200.0,      -1.0 / 479001600.0,
                                  1.0 / 3628800.0,          -1.0 / 40320.0,
                                  1.0 / 720.0,              -1.0 / 24.0,
                                  0.5};
  double ps = sin_c[0];
  for (int k = 1; k < 8; ++k) ps = ps * z + sin_c[k];
  const double sn = x - (x * z) * ps;
  double pc = cos_c[0];
  for (int k = 1; k < 9; ++k) pc = pc * z + cos_c[k];
  const double cs = 1.0 - z * pc;
  switch (((int)n) & 3) {
    case 0: *sn_out = sn; *cs_out = cs; break;
    case 1: *sn_out = cs; *cs_out = -sn; break;
    case 2: *sn_out = -sn; *cs_out = -cs; break;
    default: *sn_out = -cs; *cs_out = sn; break;
  }
}

/* the two normals of Philox block `idx` of stream (seed, stream_id) */
static void normal_block(uint64_t seed, uint32_t stream_id, uint64_t idx, double* z0, double* z1) {
  block4 c = {{(uint32_t)idx, (uint32_t)(idx >> 32), stream_id, 0x53505831u}};
  const block4 r = philox10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const uint64_t a = ((uint64_t)(r.x[0] >> 5) << 26) | (uint64_t)(r.x[1] >> 6);
  const uint64_t b = ((uint64_t)(r.x[2] >> 5) << 26) | (uint64_t)(r.x[3] >> 6);
  const double two_m53 = 1.1102230246251565404e-16;
  const double u1 = ((double)a + 0.5) * two_m53;
  const double u2 = (double)b * two_m53;
  const double rad = __builtin_sqrt(-2.0 * series_log(u1));
  double sn, cs;
  series_sincos_turns(u2, &sn, &cs);
  *z0 = rad * cs;
  *z1 = rad * sn;
}

/* out (complex interleaved, column-major, leading dimension ld) = columns
 * [col0, col0 + cols) of the rows x ... stream matrix, times scale */
void oracle_gen_cmatrix(uint64_t seed, uint32_t stream_id, int64_t rows, int64_t cols, int64_t ld,
                        int64_t col0, double scale, double* out, int threads) {
#ifdef _OPENMP
  if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(threads) collapse(2)
#endif
  for (int64_t c = 0; c < cols; ++c)
    for (int64_t p = 0; p < rows; ++p) {
      double z0, z1;
      normal_block(seed, stream_id, (uint64_t)(rows * (col0 + c) + p), &z0, &z1);
      out[2 * (c * ld + p)] = scale * z0;
      out[2 * (c * ld + p) + 1] = scale * z1;
    }
}

/* test hooks: the series functions on an array */
void oracle_series_log(int64_t n, const double* x, double* y) {
  for (int64_t k = 0; k < n; ++k) y[k] = series_log(x[k]);
}
void oracle_series_sincos_turns(int64_t n, const double* u, double* s, double* c) {
  for (int64_t k = 0; k < n; ++k) series_sincos_turns(u[k], &s[k], &c[k]);
}
