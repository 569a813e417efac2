/*
 * CPU oracle for the SPEX 05.10 imaginary-frequency polarisation (HILBERT NONE).
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker and the timed CPU
 * baseline; nothing in the product links it. It restates, in plain C, the
 * reference's own loops so that the GPU library can be compared with them on
 * identical inputs.
 *
 * PARITY UNPINNED: the reference is Fortran (no compiler in this image) and
 * ships no tests, golden vectors or fixtures for this path, so this
 * restatement is checked only against an independent numpy formulation
 * (tests/golden) and against its own extended-precision variant.
 *
 * Conventions (all arrays column-major, complex interleaved re/im):
 *   cprod(p, i), p < npair, i < nbas, leading dimension ldc (complex elements)
 *   w(p, f), f < nw, leading dimension npair
 *   susceph(ij, f), ij = j*(j+1)/2 + i for i <= j, leading dimension nbas*(nbas+1)/2
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* HILBERT NONE weights, src/susceptibility.f:950-975:
 *   wghtSr(i,ifrq) = -2*rdum / ((frqh(ifrq)/img)**2 + rdum**2) / nkpt / nsym1 * nkpts(k)
 * with rdum = ene(i2,k+q) - ene(i1,k) = ediff[p] and frqh/img = omega[f].
 * wscale[p] carries nkpts(k)/nkpt/nsym1 (NULL means 1), scale_all a global factor. */
void oracle_weights(int64_t npair, const double* ediff, const double* wscale,
                    double scale_all, int32_t nw, const double* omega, double* w) {
  for (int32_t f = 0; f < nw; ++f) {
    double om2 = omega[f] * omega[f];
    for (int64_t p = 0; p < npair; ++p) {
      double d = ediff[p];
      double s = (wscale ? wscale[p] : 1.0) * scale_all;
      w[p + npair * (int64_t)f] = -2.0 * d / (om2 + d * d) * s;
    }
  }
}

static inline int64_t packed_index(int64_t i, int64_t j) { return j * (j + 1) / 2 + i; }

/* Faithful restatement of the body loop, src/susceptibility.f:1182-1240, and of
 * spectral_function's HILBERT NONE branch, :1766-1789:
 *   do j = 1,dim ; do i = 1,j
 *     re(k) + i im(k) = cprod(k,i) * conjg(cprod(k,j)),  k = 1..n
 *     sus1(f) = ddot(n,re,1,wghtSr(1,f),1) ; sus2(f) = ddot(n,im,1,wghtSr(1,f),1)
 *     susceph(j*(j-1)/2+i, f) += sus1(f) + img*sus2(f)
 * The (i,j) pairs are split into contiguous ranges over threads, as the
 * reference splits them into contiguous ranges m1..m2 over MPI ranks
 * (:1164-1191). `threads` <= 0 uses all available. */
void oracle_chi0_faithful(int64_t npair, int32_t nbas, const double* cprod, int64_t ldc,
                          const double* w, int32_t nw, double* susceph, int threads) {
  const int64_t npack = (int64_t)nbas * (nbas + 1) / 2;
#ifdef _OPENMP
  if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel num_threads(threads)
#endif
  {
    double* re = (double*)malloc(sizeof(double) * (size_t)(npair > 0 ? npair : 1));
    double* im = (double*)malloc(sizeof(double) * (size_t)(npair > 0 ? npair : 1));
    int nth = 1, tid = 0;
#ifdef _OPENMP
    nth = omp_get_num_threads();
    tid = omp_get_thread_num();
#endif
    int64_t m1 = tid * npack / nth, m2 = (tid + 1) * npack / nth;  /* [m1, m2) */
    /* locate the first (i, j) of this range */
    int64_t j = 0;
    while ((j + 1) * (j + 2) / 2 <= m1) ++j;
    int64_t i = m1 - j * (j + 1) / 2;
    for (int64_t m = m1; m < m2; ++m) {
      const double* ci = cprod + 2 * ldc * i;
      const double* cj = cprod + 2 * ldc * j;
      for (int64_t k = 0; k < npair; ++k) {
        double ar = ci[2 * k], ai = ci[2 * k + 1];
        double br = cj[2 * k], bi = cj[2 * k + 1];
        re[k] = ar * br + ai * bi;   /* Re( a * conj(b) ) */
        im[k] = ai * br - ar * bi;   /* Im( a * conj(b) ) */
      }
      int64_t ij = packed_index(i, j);
      for (int32_t f = 0; f < nw; ++f) {
        const double* wf = w + npair * (int64_t)f;
        double s1 = 0.0, s2 = 0.0;
        for (int64_t k = 0; k < npair; ++k) {
          s1 += re[k] * wf[k];
          s2 += im[k] * wf[k];
        }
        double* out = susceph + 2 * (ij + npack * (int64_t)f);
        out[0] += s1;
        out[1] += s2;
      }
      if (++i > j) {
        ++j;
        i = 0;
      }
    }
    free(re);
    free(im);
  }
}

/* The same sums in extended precision (x87 long double, 64-bit significand) with
 * the products formed exactly in long double; used as the FP64 reference when
 * measuring the error of the split-precision path. */
void oracle_chi0_accurate(int64_t npair, int32_t nbas, const double* cprod, int64_t ldc,
                          const double* w, int32_t nw, double* susceph, int threads) {
  const int64_t npack = (int64_t)nbas * (nbas + 1) / 2;
#ifdef _OPENMP
  if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 8) num_threads(threads)
#endif
  for (int64_t m = 0; m < npack; ++m) {
    int64_t j = (int64_t)((sqrt(8.0 * (double)m + 1.0) - 1.0) / 2.0);
    while (j * (j + 1) / 2 > m) --j;
    while ((j + 1) * (j + 2) / 2 <= m) ++j;
    int64_t i = m - j * (j + 1) / 2;
    const double* ci = cprod + 2 * ldc * i;
    const double* cj = cprod + 2 * ldc * j;
    long double acc_r[64], acc_i[64];
    for (int32_t f0 = 0; f0 < nw; f0 += 64) {
      int32_t nf = nw - f0 < 64 ? nw - f0 : 64;
      for (int32_t f = 0; f < nf; ++f) acc_r[f] = acc_i[f] = 0.0L;
      for (int64_t k = 0; k < npair; ++k) {
        long double ar = ci[2 * k], ai = ci[2 * k + 1];
        long double br = cj[2 * k], bi = cj[2 * k + 1];
        long double re = ar * br + ai * bi;
        long double im = ai * br - ar * bi;
        for (int32_t f = 0; f < nf; ++f) {
          long double wk = w[k + npair * (int64_t)(f0 + f)];
          acc_r[f] += re * wk;
          acc_i[f] += im * wk;
        }
      }
      for (int32_t f = 0; f < nf; ++f) {
        double* out = susceph + 2 * (m + npack * (int64_t)(f0 + f));
        out[0] += (double)acc_r[f];
        out[1] += (double)acc_i[f];
      }
    }
  }
}

/* chi(i,j,f) for explicitly given columns a = cprod(:,i), b = cprod(:,j)
 * (length npair each, complex interleaved), extended precision. Used to check
 * sampled elements of full-size runs without holding all of cprod. */
void oracle_chi0_element(int64_t npair, const double* a, const double* b, const double* w,
                         int32_t nw, double* out /* 2*nw */) {
  for (int32_t f = 0; f < nw; ++f) {
    long double sr = 0.0L, si = 0.0L;
    const double* wf = w + npair * (int64_t)f;
    for (int64_t k = 0; k < npair; ++k) {
      long double ar = a[2 * k], ai = a[2 * k + 1], br = b[2 * k], bi = b[2 * k + 1];
      sr += (ar * br + ai * bi) * (long double)wf[k];
      si += (ai * br - ar * bi) * (long double)wf[k];
    }
    out[2 * f] = (double)sr;
    out[2 * f + 1] = (double)si;
  }
}

/* Spin factor, src/susceptibility.f:1331-1343: susceph = susceph * 2 when
 * nspin == 1 and there is no spin-orbit coupling. n complex elements. */
void oracle_scale(double* z, int64_t n, double factor) {
  for (int64_t t = 0; t < 2 * n; ++t) z[t] *= factor;
}

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
