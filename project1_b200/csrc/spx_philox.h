// Counter-based seeded normals shared by host and device code.
//
// Philox4x32-10 follows Salmon, Moraes, Dror and Shaw, "Parallel random numbers:
// as easy as 1, 2, 3" (SC'11): ten rounds of two 32x32->64 multiplies with the
// published multipliers and Weyl key increments. A normal pair comes from one
// Philox block through the Box-Muller transform. The logarithm and the
// sine/cosine are evaluated here from their Taylor / atanh series using only
// IEEE-754 add, multiply, divide and square root, each correctly rounded and
// never contracted into an FMA, so that gcc on the host and nvcc on the device
// produce the same bits.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define SPX_HD __host__ __device__ __forceinline__
#else
#define SPX_HD static inline
#endif

#if defined(__CUDA_ARCH__)
#define SPX_ADD(a, b) __dadd_rn((a), (b))
#define SPX_SUB(a, b) __dsub_rn((a), (b))
#define SPX_MUL(a, b) __dmul_rn((a), (b))
#define SPX_DIV(a, b) __ddiv_rn((a), (b))
#define SPX_SQRT(a) __dsqrt_rn((a))
#else
#include <math.h>
// Host code is compiled with -ffp-contract=off; these stay single IEEE ops.
#define SPX_ADD(a, b) ((a) + (b))
#define SPX_SUB(a, b) ((a) - (b))
#define SPX_MUL(a, b) ((a) * (b))
#define SPX_DIV(a, b) ((a) / (b))
#define SPX_SQRT(a) sqrt((a))
#endif

namespace spx {

struct u32x4 {
  uint32_t v[4];
};

SPX_HD void mulhilo32(uint32_t a, uint32_t b, uint32_t* hi, uint32_t* lo) {
  uint64_t p = (uint64_t)a * (uint64_t)b;
  *hi = (uint32_t)(p >> 32);
  *lo = (uint32_t)p;
}

// One Philox4x32 block: counter c, key k, 10 rounds.
SPX_HD u32x4 philox4x32_10(u32x4 c, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(M0, c.v[0], &hi0, &lo0);
    mulhilo32(M1, c.v[2], &hi1, &lo1);
    u32x4 n;
    n.v[0] = hi1 ^ c.v[1] ^ k0;
    n.v[1] = lo1;
    n.v[2] = hi0 ^ c.v[3] ^ k1;
    n.v[3] = lo0;
    c = n;
    k0 += W0;
    k1 += W1;
  }
  return c;
}

// Natural log for x > 0 (finite, normal): x = m * 2^e with m in [sqrt(1/2), sqrt(2)),
// ln m = 2 atanh(s), s = (m-1)/(m+1), series through s^23.
SPX_HD double ln_ieee(double x) {
  union {
    double d;
    uint64_t u;
  } b;
  b.d = x;
  int e = (int)((b.u >> 52) & 0x7ff) - 1023;
  b.u = (b.u & 0x000fffffffffffffull) | 0x3ff0000000000000ull;  // m in [1, 2)
  double m = b.d;
  if (m > 1.4142135623730951) {  // move to [sqrt(1/2), sqrt(2))
    m = SPX_MUL(m, 0.5);         // exact
    e += 1;
  }
  double s = SPX_DIV(SPX_SUB(m, 1.0), SPX_ADD(m, 1.0));
  double s2 = SPX_MUL(s, s);
  // 1 + s2/3 + s2^2/5 + ... + s2^11/23, Horner from the top
  double p = 1.0 / 23.0;
  p = SPX_ADD(SPX_MUL(p, s2), 1.0 / 21.0);
  p = SPX_ADD(SPX_MUL(p, s2), 1.0 / 19.0);
  p = SPX_ADD(SPX_MUL(p, s2), 1.0 / 17.0);
  p = SPX_ADD(SPX_MUL(p, s2), 1.0 / 15.0);
  p = SPX_ADD(SPX_MUL(p, s2), 1.0 / 13.0);
  p = SPX_ADD(SPX_MUL(p, s2), 1.0 / 11.0);
  p = SPX_ADD(SPX_MUL(p, s2), 1.0 / 9.0);
  p = SPX_ADD(SPX_MUL(p, s2), 1.0 / 7.0);
  p = SPX_ADD(SPX_MUL(p, s2), 1.0 / 5.0);
  p = SPX_ADD(SPX_MUL(p, s2), 1.0 / 3.0);
  p = SPX_ADD(SPX_MUL(p, s2), 1.0);
  double lnm = SPX_MUL(SPX_MUL(2.0, s), p);
  // ln 2 as a 2-term sum: hi has 32 significant bits, so e*hi is exact for |e| < 2^20.
  const double LN2_HI = 6.93147180369123816490e-01;
  const double LN2_LO = 1.90821492927058770002e-10;
  double de = (double)e;
  return SPX_ADD(SPX_MUL(de, LN2_HI), SPX_ADD(SPX_MUL(de, LN2_LO), lnm));
}

// sin and cos of 2*pi*u for u in [0, 1): quadrant reduction in turns (exact),
// then Taylor series on [-pi/4, pi/4].
SPX_HD void sincos_turns(double u, double* s_out, double* c_out) {
  double q = SPX_MUL(u, 4.0);                    // exact
  double n = (double)(int64_t)SPX_ADD(q, 0.5);   // nearest quadrant, 0..4
  double f = SPX_SUB(q, n);                      // exact, in [-0.5, 0.5]
  const double HALF_PI = 1.57079632679489661923;
  double x = SPX_MUL(f, HALF_PI);
  double x2 = SPX_MUL(x, x);
  // sin x = x (1 - x2/3! + x2^2/5! - ... ), through x^17
  double ps = -1.0 / 355687428096000.0;                // -1/17!
  ps = SPX_ADD(SPX_MUL(ps, x2), 1.0 / 1307674368000.0);  // 1/15!
  ps = SPX_ADD(SPX_MUL(ps, x2), -1.0 / 6227020800.0);    // -1/13!
  ps = SPX_ADD(SPX_MUL(ps, x2), 1.0 / 39916800.0);       // 1/11!
  ps = SPX_ADD(SPX_MUL(ps, x2), -1.0 / 362880.0);        // -1/9!
  ps = SPX_ADD(SPX_MUL(ps, x2), 1.0 / 5040.0);           // 1/7!
  ps = SPX_ADD(SPX_MUL(ps, x2), -1.0 / 120.0);           // -1/5!
  ps = SPX_ADD(SPX_MUL(ps, x2), 1.0 / 6.0);              // 1/3!
  // sin = x - x*x2*ps' where ps' built with alternating signs above -> rewrite:
  double sn = SPX_SUB(x, SPX_MUL(SPX_MUL(x, x2), ps));
  // cos x = 1 - x2/2 + x2^2/4! - ..., through x^18
  double pc = 1.0 / 6402373705728000.0;                  // 1/18!
  pc = SPX_ADD(SPX_MUL(pc, x2), -1.0 / 20922789888000.0);  // -1/16!
  pc = SPX_ADD(SPX_MUL(pc, x2), 1.0 / 87178291200.0);      // 1/14!
  pc = SPX_ADD(SPX_MUL(pc, x2), -1.0 / 479001600.0);       // -1/12!
  pc = SPX_ADD(SPX_MUL(pc, x2), 1.0 / 3628800.0);          // 1/10!
  pc = SPX_ADD(SPX_MUL(pc, x2), -1.0 / 40320.0);           // -1/8!
  pc = SPX_ADD(SPX_MUL(pc, x2), 1.0 / 720.0);              // 1/6!
  pc = SPX_ADD(SPX_MUL(pc, x2), -1.0 / 24.0);              // -1/4!
  pc = SPX_ADD(SPX_MUL(pc, x2), 0.5);                      // 1/2!
  double cs = SPX_SUB(1.0, SPX_MUL(x2, pc));
  int k = ((int)n) & 3;
  if (k == 0) {
    *s_out = sn;
    *c_out = cs;
  } else if (k == 1) {
    *s_out = cs;
    *c_out = -sn;
  } else if (k == 2) {
    *s_out = -sn;
    *c_out = -cs;
  } else {
    *s_out = -cs;
    *c_out = sn;
  }
}

// Two standard normals from the Philox block with counter index `pair`.
SPX_HD void normal_pair(uint64_t seed, uint32_t stream_id, uint64_t pair, double* z0,
                        double* z1) {
  u32x4 c;
  c.v[0] = (uint32_t)pair;
  c.v[1] = (uint32_t)(pair >> 32);
  c.v[2] = stream_id;
  c.v[3] = 0x53505831u;  // domain tag
  u32x4 r = philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const double TWO_M53 = 1.1102230246251565404e-16;  // 2^-53
  uint64_t a = ((uint64_t)(r.v[0] >> 5) << 26) | (uint64_t)(r.v[1] >> 6);
  uint64_t bb = ((uint64_t)(r.v[2] >> 5) << 26) | (uint64_t)(r.v[3] >> 6);
  double u1 = SPX_MUL(SPX_ADD((double)a, 0.5), TWO_M53);  // (0, 1)
  double u2 = SPX_MUL((double)bb, TWO_M53);               // [0, 1)
  double rad = SPX_SQRT(SPX_MUL(-2.0, ln_ieee(u1)));
  double sn, cs;
  sincos_turns(u2, &sn, &cs);
  *z0 = SPX_MUL(rad, cs);
  *z1 = SPX_MUL(rad, sn);
}

// Element e of the stream.
SPX_HD double normal_at(uint64_t seed, uint32_t stream_id, uint64_t e) {
  double z0, z1;
  normal_pair(seed, stream_id, e >> 1, &z0, &z1);
  return (e & 1) ? z1 : z0;
}

}  // namespace spx
