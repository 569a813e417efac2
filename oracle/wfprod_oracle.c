/*
 * CPU oracle for the mixed-product-basis projections of SPEX 05.10
 * (wavefproducts2_mt and the explicit-convolution branch of wavefproducts2_pw).
 *
 * TEST INFRASTRUCTURE ONLY: the checker, never linked by the product.
 * PARITY UNPINNED (see chi0_oracle.c): restated from src/wavefproducts.f.
 *
 * Index conventions (0-based here, 1-based in the reference):
 *   wave-function MT index lm = lmstart(l,m) + n, lmstart runs over l, then m = -l..l,
 *   with nrad radial functions each (src/wavefproducts.f:225-232);
 *   mixed-basis MT index llm over LL, MM = -LL..LL, nn = 0..nradm-1 (:299-337);
 *   gaunt1[l1][l][LL][m+lcut][MM+lcutm] laid out with l1 fastest (Fortran order);
 *   integral(ln, ln1, lln): ln over (l, n), ln1 the running index over the allowed
 *   (l1, n1) for the given (l, LL) (:200-222, :311-328), lln over (LL, nn).
 *   cmt[(((k*nb + b)*natom + a)*maxlm + lm)] complex: coefficient lm of band b, atom a, k.
 *   cprod(p, I), p = n' + nu*(n + no*k), leading dimension ldc, complex.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  double re, im;
} cplx;

static inline cplx cmul(cplx a, cplx b) {
  cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
  return r;
}
static inline cplx cconj(cplx a) {
  cplx r = {a.re, -a.im};
  return r;
}

/* gaunt1(l1,l,LL,m,MM) with m in -lcut..lcut, MM in -lcutm..lcutm */
static inline double gaunt1(const double* g, int lcut, int lcutm, int l1, int l, int LL, int m,
                            int MM) {
  const int n0 = lcut + 1, n1 = lcut + 1, n2 = lcutm + 1, n3 = 2 * lcut + 1;
  return g[l1 + n0 * (l + n1 * (LL + n2 * ((m + lcut) + n3 * (MM + lcutm))))];
}

/* wavefproducts2_mt, src/wavefproducts.f:95-431 (non-INV, no SOC, SUBTYPE 2):
 *   mat(lm1', LLM) = sum cmt1(lm) * integral(ln, ln1, lln) * gaunt1(l1,l,LL,m,MM),
 *   cprod(:, n, k, llm0+LLM) += cexp * conj( cmt2^H . mat )                      (:359)
 * integral has dims (nln, nln1, nlln) = ((lcut+1)*nrad, ld1, (lcutm+1)*nradm). */
void oracle_wfprod_mt(int natom, int lcut, int nrad, int lcutm, int nradm, const double* gaunt,
                      const double* integral, int ld1, const double* cexp, int nk, int nocc,
                      int nunocc, const double* cmt_occ, const double* cmt_unocc, double* cprod_,
                      int64_t ldc) {
  const int maxlm = (lcut + 1) * (lcut + 1) * nrad;
  const int maxllm = (lcutm + 1) * (lcutm + 1) * nradm;
  const int nln = (lcut + 1) * nrad;
  const cplx* c1 = (const cplx*)cmt_occ;
  const cplx* c2 = (const cplx*)cmt_unocc;
  cplx* cprod = (cplx*)cprod_;
  const cplx* ce = (const cplx*)cexp;
  cplx* mat = (cplx*)malloc(sizeof(cplx) * maxlm * maxllm);
  /* lmstart(m, l): first index of the (l, m) block */
  int lmstart[32][64];
  {
    int lm = 0;
    for (int l = 0; l <= lcut; ++l)
      for (int m = -l; m <= l; ++m) {
        lmstart[l][m + lcut] = lm;
        lm += nrad;
      }
  }
  for (int a = 0; a < natom; ++a) {
    const int llm0 = a * maxllm;
    for (int k = 0; k < nk; ++k)
      for (int n = 0; n < nocc; ++n) {
        const cplx* cm1 = c1 + ((int64_t)(k * nocc + n) * natom + a) * maxlm;
        memset(mat, 0, sizeof(cplx) * maxlm * maxllm);
        int llm = 0, lln = 0;
        for (int LL = 0; LL <= lcutm; ++LL) {
          for (int MM = -LL; MM <= LL; ++MM) {
            int lm = 0, ln = 0;
            for (int l = 0; l <= lcut; ++l) {
              const int nx = nrad;
              for (int m = -l; m <= l; ++m) {
                const int m1 = m + MM;
                int ln1 = 0;
                int l1lo = abs(l - LL), l1hi = l + LL < lcut ? l + LL : lcut;
                for (int l1 = l1lo; l1 <= l1hi; l1 += 2) {
                  const int nx1 = nrad;
                  if (l1 >= abs(m1)) {
                    const double gnt = gaunt1(gaunt, lcut, lcutm, l1, l, LL, m, MM);
                    if (gnt != 0.0) {
                      const int lm1 = lmstart[l1][m1 + lcut];
                      for (int nn = 0; nn < nradm; ++nn)
                        for (int j = 0; j < nx1; ++j) {
                          double sr = 0.0, si = 0.0;
                          for (int i = 0; i < nx; ++i) {
                            const double v =
                                integral[(ln + i) + (int64_t)nln * ((ln1 + j) + (int64_t)ld1 * (lln + nn))];
                            sr += cm1[lm + i].re * v;
                            si += cm1[lm + i].im * v;
                          }
                          cplx* o = &mat[(lm1 + j) + (int64_t)maxlm * (llm + nn)];
                          o->re += sr * gnt;
                          o->im += si * gnt;
                        }
                    }
                  }
                  ln1 += nx1;
                }
                lm += nx;
              }
              ln += nx;
            }
            llm += nradm;
          }
          lln += nradm;
        }
        /* cprod(n', n, k, llm0+I) += cexp * sum_lm1 cmt2(lm1,n') * conj(mat(lm1,I)) */
        for (int I = 0; I < maxllm; ++I)
          for (int np = 0; np < nunocc; ++np) {
            const cplx* cm2 = c2 + ((int64_t)(k * nunocc + np) * natom + a) * maxlm;
            cplx s = {0.0, 0.0};
            for (int lm1 = 0; lm1 < maxlm; ++lm1) {
              cplx t = cmul(cm2[lm1], cconj(mat[lm1 + (int64_t)maxlm * I]));
              s.re += t.re;
              s.im += t.im;
            }
            s = cmul(ce[a], s);
            cplx* o = &cprod[(np + (int64_t)nunocc * (n + (int64_t)nocc * k)) + ldc * (llm0 + I)];
            o->re += s.re;
            o->im += s.im;
          }
      }
  }
  free(mat);
}

/* Explicit-convolution branch of wavefproducts2_pw with FULLPW, src/wavefproducts.f:760-997:
 *   cpw0(G0) = sum_G1 cstep(G0 - G1) cpw1(G1)                                 (:870-888)
 *   cpw3(ig2, ig) = cpw0(G2(ig2) - GM(ig) + g)                                (:917-932)
 *   cprod(:, n, k, col0+ig) += conj( cpw2^H . cpw3 ) / sqrt(vol)              (:945)
 * gpt1 (3 x ngpt1) are the G vectors of the occupied states at k (:870), gpt2
 * (3 x ngpt2) those of the unoccupied states at k+q (:917), gptm (3 x ngptm) the
 * mixed-basis plane waves; one set for every k. gsh is the backfolding vector g.
 * cstep is given on the box [-sr, sr]^3 (x fastest).
 * cpw_occ[((k*nocc + n)*ngpt1 + ig)], cpw_unocc[((k*nunocc + n')*ngpt2 + ig)] complex. */
void oracle_wfprod_pw(int ngpt1, const int* gpt1, int ngpt2, const int* gpt2, int ngptm,
                      const int* gptm, const int* gsh, int sr, const double* cstep_, double vol,
                      int nk, int nocc, int nunocc, const double* cpw_occ,
                      const double* cpw_unocc, double* cprod_, int64_t ldc, int col0) {
  const cplx* c1 = (const cplx*)cpw_occ;
  const cplx* c2 = (const cplx*)cpw_unocc;
  const cplx* cstep = (const cplx*)cstep_;
  cplx* cprod = (cplx*)cprod_;
  const double sqv = 1.0 / sqrt(vol);
  const int ns = 2 * sr + 1;
  cplx* cpw3 = (cplx*)malloc(sizeof(cplx) * (size_t)ngpt2 * ngptm);
  for (int k = 0; k < nk; ++k)
    for (int n = 0; n < nocc; ++n) {
      const cplx* cp1 = c1 + (int64_t)(k * nocc + n) * ngpt1;
      for (int ig = 0; ig < ngptm; ++ig)
        for (int ig2 = 0; ig2 < ngpt2; ++ig2) {
          const int G0[3] = {gpt2[3 * ig2] - gptm[3 * ig] + gsh[0],
                             gpt2[3 * ig2 + 1] - gptm[3 * ig + 1] + gsh[1],
                             gpt2[3 * ig2 + 2] - gptm[3 * ig + 2] + gsh[2]};
          cplx s = {0.0, 0.0};
          for (int ig1 = 0; ig1 < ngpt1; ++ig1) {
            const int d0 = G0[0] - gpt1[3 * ig1], d1 = G0[1] - gpt1[3 * ig1 + 1],
                      d2 = G0[2] - gpt1[3 * ig1 + 2];
            if (abs(d0) > sr || abs(d1) > sr || abs(d2) > sr) continue;
            const cplx st = cstep[(d0 + sr) + ns * ((d1 + sr) + ns * (d2 + sr))];
            cplx t = cmul(st, cp1[ig1]);
            s.re += t.re;
            s.im += t.im;
          }
          cpw3[ig2 + (int64_t)ngpt2 * ig] = s;
        }
      for (int ig = 0; ig < ngptm; ++ig)
        for (int np = 0; np < nunocc; ++np) {
          const cplx* cp2 = c2 + (int64_t)(k * nunocc + np) * ngpt2;
          cplx s = {0.0, 0.0};
          for (int ig2 = 0; ig2 < ngpt2; ++ig2) {
            cplx t = cmul(cp2[ig2], cconj(cpw3[ig2 + (int64_t)ngpt2 * ig]));  /* conj(a^H b) */
            s.re += t.re;
            s.im += t.im;
          }
          cplx* o = &cprod[(np + (int64_t)nunocc * (n + (int64_t)nocc * k)) + ldc * (col0 + ig)];
          o->re += s.re * sqv;
          o->im += s.im * sqv;
        }
    }
  free(cpw3);
}

int oracle_wfprod_version(void) { return 3; }
