/*
 * spexgpu.h — C ABI of the B200 (sm_100a) Kohn-Sham polarisation library.
 *
 * The library replaces, inside SPEX 05.10, the HILBERT NONE band-pair
 * accumulation of the imaginary-frequency polarisation and the wave-function
 * products that feed it. Every entry point is `extern "C"`, takes plain
 * pointers and 64-bit sizes, returns an int status (SPX_OK == 0, negative on
 * error) and never aborts. spx_last_error() returns the message of the last
 * failing call on a context.
 *
 * Array conventions follow the Fortran caller (column-major, 1-based indices
 * in the reference become 0-based offsets here):
 *   - complex arrays are interleaved (re, im) doubles: Fortran complex(8),
 *     C99 double _Complex and cuDoubleComplex all share this layout;
 *   - cprod(npair, nbas): band-pair index p fastest, with p = n' + nu*(n + no*k)
 *     (unoccupied n' fastest, then occupied n, then k; reference
 *     src/susceptibility.f:861-865 and :956-960), leading dimension ldc >= npair;
 *   - susceph(nbas*(nbas+1)/2, nw): packed upper triangle, element (i, j) with
 *     i <= j (0-based) at j*(j+1)/2 + i, frequency outermost
 *     (src/susceptibility.f:1210, ij = j*(j-1)/2 + i in 1-based form).
 *
 * A context is bound to one device, is not thread-safe, and orders all of its
 * work on one CUDA stream unless a stream is passed explicitly.
 */
#ifndef SPEXGPU_H
#define SPEXGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SPX_ABI_VERSION 1

/* status codes */
#define SPX_OK        0
#define SPX_EINVAL   -1   /* bad argument (null pointer, negative size, ...)     */
#define SPX_ENOMEM   -2   /* device or pinned-host allocation failed             */
#define SPX_ECUDA    -3   /* a CUDA runtime call failed                          */
#define SPX_ETIMEOUT -4   /* a bounded device-side wait ran out                  */
#define SPX_ENOTSUP  -5   /* feature not available (no sm_100 device, ...)       */
#define SPX_ENODEV   -6   /* no CUDA device                                      */

/* precision of the band-pair accumulation */
#define SPX_FP64  0       /* complex FP64 on the DMMA tensor path: the drop-in   */
#define SPX_SPLIT 1       /* int8 digit slices on tcgen05, exact int32 TMEM
                             partials, FP64 reduction; weights always in FP64;
                             per element |error| <= 1e-6 sqrt|chi_ii chi_jj|     */

/* spx_options.products: the interstitial (explicit-convolution) product GEMM
 * AUTO: FP64, except inside spx_chi0_from_coeffs_dev with SPX_SPLIT, where it runs
 *       on int8 digit slices (A 3, B 4 digits, exact int32 sums; per value the
 *       slicing error is 2^-17/127 of the row scale, the same as the split
 *       accumulation's own slicing of M);
 * FP64: always FP64 (the drop-in); SPLIT: always int8 slices.                  */
#define SPX_PRODUCTS_AUTO  0
#define SPX_PRODUCTS_FP64  1
#define SPX_PRODUCTS_SPLIT 2

typedef struct spx_ctx spx_ctx;

typedef struct spx_options {
  int32_t struct_size;      /* sizeof(spx_options), for forward compatibility   */
  int32_t verbose;          /* 0 = silent                                        */
  int64_t workspace_limit;  /* device bytes the context may allocate, 0 = auto   */
  int64_t pinned_limit;     /* pinned host staging bytes, 0 = auto               */
  int32_t chunk_pairs;      /* band pairs per streamed chunk, 0 = auto           */
  int32_t timeout_ms;       /* bound on every device-side wait, 0 = 4000 ms      */
  int32_t split_variant;    /* split-path kernel: 0 auto (the tuning table's choice,
                               else 5), 1 one CTA per 64 x 64
                               tile, 2 CTA pair (tcgen05 cta_group::2), 3 the
                               persistent schedule with its own preparation warps,
                               5 one CTA per 64 x 80 tile (N = 160 MMAs)         */
  int32_t products;         /* interstitial product GEMM: SPX_PRODUCTS_*         */
} spx_options;

/* Per-call statistics filled by the accumulation entry points (may be NULL). */
typedef struct spx_chi0_stats {
  double  ms_total;         /* wall time of the call, host-observed              */
  double  ms_gram;          /* device time of the band-pair accumulation kernels */
  double  ms_prep;          /* device time of weight / operand preparation       */
  double  flops;            /* algorithmic real flops, 8*N^2*P*nw                */
  int64_t h2d_bytes;        /* host-to-device bytes moved by the call            */
  int64_t d2h_bytes;        /* device-to-host bytes moved by the call            */
  int32_t kernel_launches;  /* kernels launched by the call                      */
  int32_t precision;        /* precision actually used                           */
} spx_chi0_stats;

/* ---- library and context --------------------------------------------------- */

int         spx_abi_version(void);
const char* spx_strerror(int status);

/* Creates a context on `device` (CUDA ordinal). opt may be NULL. */
int         spx_ctx_create(int device, const spx_options* opt, spx_ctx** out);
int         spx_ctx_destroy(spx_ctx* ctx);
const char* spx_last_error(const spx_ctx* ctx);
/* Waits for all work of the context. */
int         spx_ctx_synchronize(spx_ctx* ctx);

/* ---- frequency weights (K6) -------------------------------------------------
 * Replaces the HILBERT NONE weight loop, src/susceptibility.f:950-975:
 *   w(p, f) = -2*d_p / (omega_f^2 + d_p^2) * scale_p * scale_all,
 * d_p = e_n'(k+q) - e_n(k) (ediff), omega_f the imaginary-axis magnitude
 * (frqh(f)/img), scale_p = nkpts(k)/nkpt/nsym1 (wscale, NULL = 1). A pair whose
 * unoccupied band lies above nband gets scale_p = 0. Device pointers.
 * w is (npair, nw) column-major with leading dimension npair. */
int spx_weights_dev(spx_ctx* ctx, int64_t npair, const double* ediff,
                    const double* wscale, double scale_all,
                    int32_t nw, const double* omega, double* w, void* stream);

/* ---- band-pair accumulation (K1/K2, with K6 inside) -------------------------
 * Replaces src/susceptibility.f:950-975 (weights), :1182-1240 (body loop) and
 * :1766-1789 (spectral_function, HILBERT NONE branch):
 *   susceph(ij(i,j), f) += sum_p cprod(p,i) * conj(cprod(p,j)) * w(p,f),  i<=j.
 * The result is ADDED to susceph, like the reference's `+=`; the caller zeroes
 * it once per q point (src/susceptibility.f:211-223).
 * Host-pointer form: cprod, ediff, wscale, omega and susceph are host arrays;
 * the call streams cprod to the device in chunks, overlapping copy and compute,
 * and returns after susceph has been updated. */
int spx_chi0_accumulate(spx_ctx* ctx, const double* cprod, int64_t ldc,
                        int64_t npair, int32_t nbas,
                        const double* ediff, const double* wscale, double scale_all,
                        int32_t nw, const double* omega, int32_t precision,
                        double* susceph, spx_chi0_stats* stats);

/* Device-pointer form of spx_chi0_accumulate; ordered on `stream` (NULL = the
 * context stream). Returns once the work is enqueued unless stats != NULL. */
int spx_chi0_accumulate_dev(spx_ctx* ctx, const double* cprod, int64_t ldc,
                            int64_t npair, int32_t nbas,
                            const double* ediff, const double* wscale, double scale_all,
                            int32_t nw, const double* omega, int32_t precision,
                            double* susceph, void* stream, spx_chi0_stats* stats);

/* The -DINV build (spex.inv: MCOMPLEX_dp = real_dp, src/cppmacro.h:53-64): real
 * cprod (ldc, nbas) and real packed susceph (nbas(nbas+1)/2, nw), with
 * re(k) = cprod(k,i) * cprod(k,j) (src/susceptibility.f:1197),
 *   susceph(ij, f) += sum_p cprod(p, i) cprod(p, j) w(p, f),  ij = j(j+1)/2 + i.
 * Device arrays; the weights, precision and stream as spx_chi0_accumulate_dev. */
int spx_chi0_accumulate_real_dev(spx_ctx* ctx, const double* cprod, int64_t ldc,
                                 int64_t npair, int32_t nbas,
                                 const double* ediff, const double* wscale, double scale_all,
                                 int32_t nw, const double* omega, int32_t precision,
                                 double* susceph, void* stream, spx_chi0_stats* stats);

/* Allocation-free FP64 accumulation; no counterpart in the reference.
 * For callers that cannot call cudaMalloc, such as a Fortran host whose device
 * memory belongs to its OpenMP/OpenACC offload runtime or to a pool allocator.
 * It takes no context and allocates nothing. Its scratch (the FP64 weights of
 * one slab of pairs) is a static 32 MiB device array that every GPU loading
 * the library keeps until exit. Each call reads a status word back and
 * synchronizes `stream`, so it must not be called while that stream is being
 * captured into a graph. The scratch addresses are looked up on the first call on
 * a device and again after the device's context has been replaced (e.g. by
 * cudaDeviceReset). Calls that overlap on the GPU race on the shared scratch.
 * nw > 262144 and nbas > 46340 are rejected with SPX_EINVAL. Device pointers, on
 * the current device; returns after `stream` has finished the work. */
int spx_chi0_accumulate_dev_noalloc(const double* cprod, int64_t ldc, int64_t npair,
                                    int32_t nbas, const double* ediff, const double* wscale,
                                    double scale_all, int32_t nw, const double* omega,
                                    double* susceph, void* stream);

/* Multiplies n complex elements of a device array by a real factor: the spin
 * factor 2 of src/susceptibility.f:1331-1343 for unpolarised, non-SOC runs. */
int spx_scale_dev(spx_ctx* ctx, double* z, int64_t n, double factor, void* stream);

/* ---- mixed-product-basis projections (K4) -----------------------------------
 * Muffin-tin part, replaces wavefproducts2_mt (src/wavefproducts.f:95-431, the
 * non-INV, no-SOC branch): for every atom a, k point k, occupied band n and
 * unoccupied band n',
 *   cprod(p, a*maxllm + I) += cexp_a * sum_lm1 cmt_unocc(lm1, n') * conj(mat_n(lm1, I)),
 *   mat_n(lm1, I) = sum_lm cmt_occ(lm, n) * integral(ln, ln1, lln) * gaunt1(l1, l, LL, m, MM),
 * p = n' + nunocc*(n + nocc*k), with the index nest of :299-337. All atoms share
 * gaunt1 and integral (one atom type); maxlm = (lcut+1)^2 nrad,
 * maxllm = (lcutm+1)^2 nradm. The descriptor arrays are host memory. */
typedef struct spx_mt_desc {
  int32_t natom, lcut, nrad, lcutm, nradm;
  int32_t ld1;              /* second dimension of integral (>= (lcut+1)*nrad)       */
  const double* gaunt;      /* gaunt1(0:lcut, 0:lcut, 0:lcutm, -lcut:lcut, -lcutm:lcutm),
                               column-major                                          */
  const double* integral;   /* integral((lcut+1)*nrad, ld1, (lcutm+1)*nradm), col-major */
  const double* cexp;       /* complex (natom): exp(-2 pi i q.R_a)                    */
} spx_mt_desc;

/* Interstitial part, replaces wavefproducts2_pw with the step function: the
 * explicit-convolution branch (src/wavefproducts.f:760-997) or, with nfft > 0,
 * the FFT branch (:576-758), which computes the same sum on a grid:
 *   cpw0(G0) = sum_G1 cstep(G0 - G1) cpw_occ(G1),
 *   cprod(p, col0 + ig) += 1/sqrt(vol) * sum_ig2 cpw_unocc(ig2, n') * conj(cpw0(G2(ig2) - GM(ig) + g)).
 * gpt1 lists the G vectors of the occupied states (at k), gpt2 those of the
 * unoccupied states (at k+q), gptm the mixed-basis plane waves; one set is used
 * for every k of a call (call once per k when the sets differ). Host arrays. */
typedef struct spx_pw_desc {
  int32_t ngpt1, ngpt2, ngptm;
  int32_t step_radius;      /* cstep is given on [-sr, sr]^3, sr <= 4                 */
  const int32_t* gpt1;      /* (3, ngpt1) integer G vectors                           */
  const int32_t* gpt2;      /* (3, ngpt2)                                             */
  const int32_t* gptm;      /* (3, ngptm)                                             */
  int32_t gshift[3];        /* backfolding vector g (src/wavefproducts.f:549-551)     */
  int32_t nfft;             /* 0: explicit convolution (:760-997); n > 0: the FFT
                               branch (:576-758) on an n^3 grid, 2 <= n <= 64, at most
                               16 distinct (G_M - g) mod n per axis, ngptm <= 4096   */
  const double* cstep;      /* complex (2sr+1)^3, x fastest                            */
  double vol;               /* unit-cell volume                                        */
} spx_pw_desc;

/* Coefficient layouts (complex, C order, device memory):
 *   cmt_occ (nk, nocc, natom, maxlm), cmt_unocc (nk, nunocc, natom, maxlm),
 *   cpw_occ (nk, nocc, ngpt1), cpw_unocc (nk, nunocc, ngpt2);
 * cprod is the column-major (ldc, ncol) complex matrix of spx_chi0_accumulate,
 * ldc >= nk*nocc*nunocc. Both calls ADD into cprod. Ordered on `stream`. */
int spx_wfprod_mt_dev(spx_ctx* ctx, const spx_mt_desc* mt, int32_t nk, int32_t nocc,
                      int32_t nunocc, const double* cmt_occ, const double* cmt_unocc,
                      double* cprod, int64_t ldc, void* stream);
int spx_wfprod_pw_dev(spx_ctx* ctx, const spx_pw_desc* pw, int32_t nk, int32_t nocc,
                      int32_t nunocc, const double* cpw_occ, const double* cpw_unocc,
                      double* cprod, int64_t ldc, int32_t col0, void* stream);

/* Products and polarisation in one call, with M kept on the device: the packet
 * loop of src/susceptibility.f:751-1276 from the wave-function coefficients
 * (products :778,790, weights :950-975, accumulation :1182-1240). The mixed
 * basis is the natom*maxllm MT functions followed by the ngptm plane waves;
 * pairs p = n' + nunocc*(n + nocc*k). ediff, wscale (may be NULL), omega and
 * susceph as in spx_chi0_accumulate_dev; all arrays device memory. */
int spx_chi0_from_coeffs_dev(spx_ctx* ctx, const spx_mt_desc* mt, const spx_pw_desc* pw,
                             int32_t nk, int32_t nocc, int32_t nunocc,
                             const double* cmt_occ, const double* cmt_unocc,
                             const double* cpw_occ, const double* cpw_unocc,
                             const double* ediff, const double* wscale, double scale_all,
                             int32_t nw, const double* omega, int32_t precision,
                             double* susceph, void* stream, spx_chi0_stats* stats);

/* ---- Hilbert-mesh path, imaginary axis -------------------------------------
 * The default HILBERT path accumulates the spectral function on a frequency mesh
 * (tetrahedron weights wtetra(p, s), src/susceptibility.f:996-1078) and
 * Hilbert-transforms it with the getwghtS weights (src/hilbert.f:193-300). For
 * imaginary frequencies the two collapse into effective pair weights
 *   w(p, f) = scale_all * sum_s [wtetra(p, s) > thr] wtetra(p, s) * wghtSr(s, f),
 * which spx_chi0_accumulate_w_dev then accumulates (weights of any sign).
 * Device arrays: wtetra (ldt, nfrqs), wghtSr (nfrqs, nw), w (ldw, nw);
 * nfrqs * nw <= 25600. */
int spx_weights_hilbert_dev(spx_ctx* ctx, int64_t npair, int32_t nfrqs, const double* wtetra,
                            int64_t ldt, double thr, int32_t nw, const double* wghtSr,
                            double scale_all, double* w, int64_t ldw, void* stream);
int spx_chi0_accumulate_w_dev(spx_ctx* ctx, const double* cprod, int64_t ldc, int64_t npair,
                              int32_t nbas, const double* w, int64_t ldw, int32_t nw,
                              int32_t precision, double* susceph, void* stream,
                              spx_chi0_stats* stats);

/* ---- real-frequency polarisation (Hilbert path, suscepc) ----------------------
 * Replaces the suscepc accumulation of src/susceptibility.f:1229-1235 (the
 * full-matrix layout, ACCESS_CONTIG unset) with spectral_function's wghtSr and
 * wghtSi terms (:1829-1838): with complex pair weights wr + i wi (the tetrahedron
 * weights contracted with getwghtS's wghtSr / wghtSi of the real frequencies,
 * spx_weights_hilbert_dev applied to each),
 *   suscepc(i, j, f) += sum_p M(p, i) conj(M(p, j)) (wr(p, f) + i wi(p, f)),
 * for all i, j: non-Hermitian. Evaluated as the two Hermitian sums S1 (weights
 * wr) and S2 (weights wi) of spx_chi0_accumulate_w_dev (FP64 or split, weights of
 * any sign) and suscepc(i,j) = S1 + i S2, suscepc(j,i) = conj(S1) + i conj(S2).
 * Device arrays: wr, wi (ldw, nw); suscepc complex (ldo, nbas, nw), accumulated. */
int spx_chi0_accumulate_c_dev(spx_ctx* ctx, const double* cprod, int64_t ldc, int64_t npair,
                              int32_t nbas, const double* wr, const double* wi, int64_t ldw,
                              int32_t nw, int32_t precision, double* suscepc, int64_t ldo,
                              void* stream, spx_chi0_stats* stats);

/* ---- q -> 0 head and wings (FP64) --------------------------------------------
 * Replaces src/susceptibility.f:1092-1157 for HILBERT NONE-style weights: with the
 * momentum-matrix products dcprod(p, 1:3) (src/dwavefproducts.f),
 *   head(ij(k1,k2), f) += sum_p dcprod(p,k1) conj(dcprod(p,k2)) w(p,f),  k1 <= k2,
 *                         ij = k2(k2+1)/2 + k1 (0-based), head is (6, nw),
 *   wing(k2, i, f)     += sum_p cprod(p,i) conj(dcprod(p,k2)) w(p,f), wing (3, dim, nw).
 * Column-major complex device arrays: cprod (ldc, dim), dcprod (ldd, 3); w (ldw, nw)
 * real. Always FP64 (complex DMMA, split over the pairs, summed in a fixed order). */
int spx_headwings_dev(spx_ctx* ctx, const double* cprod, int64_t ldc, int64_t npair,
                      int32_t dim, const double* dcprod, int64_t ldd, const double* w,
                      int64_t ldw, int32_t nw, double* head, double* wing, void* stream);

/* ---- q -> 0 momentum matrix -------------------------------------------------
 * Replaces momentum_matrix (src/dwavefproducts.f:89-330, non-SOC, without storeibz)
 * and the scaling of src/susceptibility.f:848-870: the head/wings input
 *   dcprod(p, x) = momentum(n', n, k, x) / sqrt(vol) / ediff(p)   (0 if |ediff| <= 1e-8;
 *                  no energy division when ediff is NULL, the multdiff mode),
 * p = n' + nunocc*(n + nocc*k), x = 1..3 Cartesian, with
 *   momentum = -i <phi_n | d/dx | phi_n'> from the MT coefficients (F/G coefficients
 *   times the radial integrals qmat1, qmat2) and the plane waves (olapvec of the
 *   occupied coefficients against (k+G)_x times the unoccupied ones).
 * One atom type; cmt layouts as spx_wfprod_mt_dev, cpw as spx_wfprod_pw_dev (one G
 * list for all k). Descriptor arrays are host memory; coefficients, ediff, dcprod
 * (ldd, 3) complex are device memory. */
typedef struct spx_mom_desc {
  int32_t natom, lcut, nrad;  /* maxlm = (lcut+1)^2 nrad                               */
  int32_t ngpt;               /* plane waves per k (0: no interstitial part)           */
  const double* qmat1;        /* (nrad, nrad, lcut+1): l-1 radial function n1 against l n2,
                                 int(u' u) + (l+1) int(u u / r) (:153-159)             */
  const double* qmat2;        /* (nrad, nrad, lcut+1): l+1 n1 against l n2,
                                 int(u' u) - l int(u u / r) (:160-166)                 */
  const int32_t* gpt;         /* (3, ngpt) integer G vectors                           */
  const double* kpt;          /* (3, nk) k points in reciprocal-lattice coordinates     */
  const double* rlat;         /* (3, 3) column-major reciprocal lattice                 */
  const double* cstep;        /* complex (2sr+1)^3, x fastest                          */
  int32_t step_radius;
  int32_t reserved;
  double vol;                 /* unit-cell volume                                      */
} spx_mom_desc;

int spx_dcprod_dev(spx_ctx* ctx, const spx_mom_desc* d, int32_t nk, int32_t nocc,
                   int32_t nunocc, const double* cmt_occ, const double* cmt_unocc,
                   const double* cpw_occ, const double* cpw_unocc, const double* ediff,
                   double* dcprod, int64_t ldd, void* stream);

/* ---- transform to the Coulomb eigenbasis ------------------------------------
 * Replaces src/susceptibility.f:806-832 (the FULLPW branch of the complex build):
 * cprod(:, :dim) = conj(conj(cprod) * ctrafo), i.e.
 *   out(p, j) = sum_{i < nbas} cprod(p, i) * conj(ctrafo(i, j)),  p < npair, j < dim.
 * Column-major device arrays: cprod (ldc, nbas), ctrafo (ldt, dim), out (ldo, dim).
 * out may be cprod itself (in place, as in the reference; then ldo == ldc); a
 * partial overlap is rejected. FP64 on the DMMA path. Ordered on `stream`. */
int spx_trafo_dev(spx_ctx* ctx, const double* cprod, int64_t ldc, int64_t npair,
                  int32_t nbas, const double* ctrafo, int64_t ldt, int32_t dim,
                  double* out, int64_t ldo, void* stream);

/* The same transform for the basis without FULLPW (src/susceptibility.f:814-824):
 * wavefproducts then returns <M~ phi|phi>, so the interstitial rows of ctrafo are
 * first multiplied by the plane-wave overlap (olapvec, src/overlap.f:298-316),
 *   ctrafo1(nbasp + i, j) = sum_k conj(cstep(G_k - G_i)) ctrafo(nbasp + k, j),
 * G = pw->gptm (the ngptm MPB plane waves, nbas = nbasp + ngptm), with pw->cstep on
 * its box (differences outside it count as 0); the muffin-tin rows are unchanged,
 * and out = conj(conj(cprod) * ctrafo1) as spx_trafo_dev. */
int spx_trafo_olap_dev(spx_ctx* ctx, const double* cprod, int64_t ldc, int64_t npair,
                       int32_t nbas, int32_t nbasp, const double* ctrafo, int64_t ldt,
                       int32_t dim, const spx_pw_desc* pw, double* out, int64_t ldo,
                       void* stream);

/* ---- dielectric matrix and its inverse (FP64) ------------------------------
 * Replaces src/correlation.f:614-636 and :703-745 for the imaginary frequencies: in
 * place on the packed susceph (npack, nw),
 *   eps_ij = delta_ij - sqrt(coul_i) chi_ij sqrt(coul_j),
 * and with invert != 0 its inverse (the library's block Gauss-Jordan sweep on the
 * DMMA path, all frequencies at once; eps must be positive definite, as it is for a
 * negative semi-definite chi, otherwise SPX_EINVAL names the frequency).
 * coul: Coulomb eigenvalues (nbas), device. head (6, nw) and wing (3, nbas, nw) may
 * be NULL; if given they become 1 - 4 pi head and -sqrt(4 pi) sqrt(coul_i) wing. */
int spx_dielec_dev(spx_ctx* ctx, int32_t nbas, int32_t nw, double* susceph,
                   const double* coul, int32_t invert, double* head, double* wing,
                   void* stream);

/* ---- many q points in one launch (K7) ---------------------------------------
 * The q loop of the reference driver (src/correlation.f:293-339 calls
 * `susceptibility` once per q point) as one call: every q has its own N_MB,
 * band window and output. Each q is accumulated exactly as by
 * spx_chi0_accumulate_dev (same slabs and kernels, so the same bits). Its M is
 * a device array, or is generated on the device slab by slab from the seeded
 * Philox stream (cprod = NULL), so that no q's M is ever held whole.
 * With SPX_SPLIT the whole batch runs as ONE persistent kernel: every SM takes
 * accumulation items (slab, tile, frequency) and operand-preparation items
 * (generation of M, weights, digit planes) from two device work queues, the q
 * with most work first, with bounded waits on the slabs' readiness; the tile
 * shape and slab size come from the tuning table (spx_autotune_batched). With
 * SPX_FP64, or SPX_SPLIT with SPX_BATCH_KERNELS, the schedule is the sequence of
 * per-slab kernels of spx_chi0_accumulate_dev. Unless SPX_BATCH_NOGRAPH is
 * given, the schedule is captured once into a CUDA graph, cached in the context
 * under the batch's signature, and replayed with a single graph launch. */
typedef struct spx_q_desc {
  int32_t nbas;             /* N_MB of this q                                         */
  int32_t variant;          /* split kernel: 0 tuned / context default, 1 one CTA per
                               64 x 64 tile, 2 CTA pair, 5 one CTA per 64 x 80 tile   */
  int64_t npair;
  int32_t slab_pairs;       /* pairs per exact int32 slab, multiple of 64 and
                               <= 32768; 0 tuned / 32768                              */
  int32_t reserved0;
  const double* cprod;      /* device (ldc, nbas) complex, or NULL = generated        */
  int64_t ldc;
  uint64_t seed;            /* generated M: element (p, c) of stream (seed, stream_id) */
  uint32_t stream_id;       /* laid out as spx_gen_cmatrix_*, times m_scale           */
  int32_t reserved1;
  double m_scale;
  const double* ediff;      /* device (npair)                                         */
  const double* wscale;     /* device (npair) or NULL                                 */
  double scale_all;
  double* susceph;          /* device packed (nbas(nbas+1)/2, nw), accumulated        */
} spx_q_desc;

#define SPX_BATCH_AUTOTUNE 1  /* measure (N, P) buckets missing from the table first  */
#define SPX_BATCH_NOGRAPH  2  /* enqueue the schedule directly, without a graph       */
#define SPX_BATCH_KERNELS  4  /* split precision as per-slab kernels, not persistent  */

/* omega: device (nw). Ordered on `stream`; returns once enqueued unless stats. */
int spx_chi0_batched(spx_ctx* ctx, int32_t nq, const spx_q_desc* q, int32_t nw,
                     const double* omega, int32_t precision, int32_t flags, void* stream,
                     spx_chi0_stats* stats);

/* Split-path tuning table of a context: per (N_MB bucket, pair bucket, nw) the
 * kernel variant and slab size that measured fastest on a probe of that shape,
 * for single calls (variant 1, 2, 3 or 5) and for the batched schedule (variant 4,
 * with its tile shape). */
typedef struct spx_tune_entry {
  int32_t nbas_bucket;      /* ceil(nbas / 128)                                        */
  int32_t npair_bucket;     /* 0: npair <= 16384, 1: <= 32768, 2: more                 */
  int32_t nw;
  int32_t variant;          /* single calls: 1 one CTA per 64 x 64 tile, 2 CTA pair,
                               3 the persistent schedule, 5 one CTA per 64 x 80 tile;
                               4 an entry of the batched table                        */
  int32_t slab_pairs;
  int32_t tile;             /* variants 3 and 4: tile columns (64, 32 or 80) + 256 *
                               pipeline stages (3, or 4 for 32 columns); 0 otherwise  */
  double  tflops;           /* measured throughput of the chosen configuration        */
} spx_tune_entry;

/* Measures the candidates (kernel variants 1, 5, 2, 3 x slabs of 8192, 12288, 16384
 * and 32768 pairs) on a seeded probe of (nbas, min(npair, 262144), nw), stores the
 * best in the table (the best kernel's smallest slab within 2 % of its fastest) and
 * returns it in *out (may be NULL). */
int spx_autotune_split(spx_ctx* ctx, int32_t nbas, int64_t npair, int32_t nw,
                       spx_tune_entry* out);
/* SPX_OK and *out if the bucket of (nbas, npair, nw) is in the table, else SPX_ENOTSUP. */
int spx_tune_lookup(const spx_ctx* ctx, int32_t nbas, int64_t npair, int32_t nw,
                    spx_tune_entry* out);
/* The same for the persistent batched schedule: measures its tile shapes (64 x 64
 * complex with 3 pipeline stages, 64 x 80 with 3, 64 x 32 with 4; tables may also
 * name 64 x 32 with 3) and slab sizes on a seeded probe of one q, stores the fastest
 * (variant 4), and looks entries up. Untuned batches run 64 x 80 tiles. */
int spx_autotune_batched(spx_ctx* ctx, int32_t nbas, int64_t npair, int32_t nw,
                         spx_tune_entry* out);
int spx_tune_lookup_batched(const spx_ctx* ctx, int32_t nbas, int64_t npair, int32_t nw,
                            spx_tune_entry* out);
/* The table as a JSON file, and back (entries are merged into the table). */
int spx_tune_save(const spx_ctx* ctx, const char* path);
int spx_tune_load(spx_ctx* ctx, const char* path);

/* Role profile of the persistent schedule (no counterpart in the reference, which
 * has no device schedule): while enabled, every launch of the persistent kernel
 * (batched split calls, single calls of variant 3) adds per-CTA cycle counts of its
 * roles into the context's counters. Launches captured into a cached graph keep
 * the setting they were captured with. enable(1) allocates the counters on first
 * use and zeroes them; read waits for the device and returns the first n (at most
 * SPX_PB_PROF_N) counters:
 *   0 CTA cycles                       7 epilogue: waiting for slab s-1's adds
 *   1 TMA: waiting for a slab's planes 8 preparation: waiting (buffer, maxima)
 *   2 TMA: waiting for a free stage    9 preparation: M and column maxima
 *   3 MMA: waiting for operands       10 preparation: weights and factors
 *   4 MMA: waiting for the epilogue   11 preparation: digit planes
 *   5 MMA: waiting for an item        12 accumulation items
 *   6 epilogue: waiting for a tile    13 preparation items
 * (cycles of one thread per role and CTA, summed over CTAs; 6 and 7 of the first
 * epilogue warp). */
#define SPX_PB_PROF_N 14
int spx_pb_profile_enable(spx_ctx* ctx, int32_t on);
int spx_pb_profile_read(spx_ctx* ctx, double* out, int32_t n);

/* ---- diagnostics ------------------------------------------------------------
 * Runs one kernel that waits, with the library's bounded device wait, on a barrier
 * phase that nothing completes. It returns SPX_ETIMEOUT after about timeout_ms
 * (1..10000) and leaves the context usable: the failure path every kernel of the
 * library takes when a wait runs out. No counterpart in the reference. */
int spx_selftest_wait_dev(spx_ctx* ctx, int32_t timeout_ms);

/* Measures the device's FP64 tensor (DMMA) peak in TFLOP/s: back-to-back
 * m16n8k8 DMMAs on register operands, timed with CUDA events (the roofline
 * denominator of the FP64 accumulation). No counterpart in the reference. */
int spx_measure_dmma_peak(spx_ctx* ctx, double* tflops);

/* ---- seeded synthetic inputs (K8) -------------------------------------------
 * Philox4x32-10 (Salmon et al., SC'11) with a Box-Muller transform written from
 * basic IEEE operations only, so host and device produce identical bits.
 * Element e of stream (seed, stream_id) is a standard normal times `scale`;
 * out[t] receives element offset + t, t < n. */
void spx_gen_normal_host(uint64_t seed, uint32_t stream_id, int64_t offset,
                         int64_t n, double scale, double* out);
int  spx_gen_normal_dev(spx_ctx* ctx, uint64_t seed, uint32_t stream_id,
                        int64_t offset, int64_t n, double scale, double* out,
                        void* stream);
/* Fills a column-major complex (rows x cols, leading dimension ld) matrix whose
 * column c holds elements [2*rows*c, 2*rows*(c+1)) of the stream, interleaved
 * re/im: the layout of a cprod packet generated column by column. */
void spx_gen_cmatrix_host(uint64_t seed, uint32_t stream_id, int64_t rows,
                          int64_t cols, int64_t ld, int64_t col0, double scale,
                          double* out);
int  spx_gen_cmatrix_dev(spx_ctx* ctx, uint64_t seed, uint32_t stream_id,
                         int64_t rows, int64_t cols, int64_t ld, int64_t col0,
                         double scale, double* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SPEXGPU_H */
