// K5: the FFT branch of the interstitial products (src/wavefproducts.f:576-758).
//
// The reference, per k point: scatters each band's plane-wave coefficients to an
// nfft^3 grid and transforms G -> r (FFTW_BACKWARD); the occupied bands become
// conj(phi_n(r))/sqrt(vol) times the step function theta(r), the unoccupied
// ones phi_n'(r)/nnfft; every pair's pointwise product is transformed r -> G
// (FFTW_FORWARD) and the mixed-basis plane waves G_M - g are gathered out of it.
//
// Here only what the gather needs is computed:
//   * band grids (K5a, `dft_pass_kernel` x3): the coefficients live in a small
//     G box, so each of the three separable passes sums only over the box
//     extent of its axis (19 of 48 for a 3000-wave sphere on a 48^3 grid); the last pass applies
//     conj, 1/sqrt(vol), theta or 1/nnfft;
//   * pair z and y passes (K5b): one CTA per (occupied band, x plane, group of
//     unoccupied bands) forms the product line by line and transforms it along z,
//     keeping the kz values that occur in G_M - g only (13 of 48), then along y to
//     the needed ky values, in shared memory. Grid edges n = 16 r (r <= 4, the
//     48^3 grid among them) use a radix-16 x r line FFT
//     (`fft_pair_zy_radix_kernel`, the transform the reference gets from FFTW,
//     src/fft.f:69-93); other edges sum the pruned DFT directly
//     (`fft_pair_zy_kernel`);
//   * pair x pass and gather (K5c, `fft_pair_x_kernel`): one CTA per pair sums
//     over x for exactly the (kx, ky, kz) of each G_M and adds the result into
//     cprod's column.
// All arithmetic is FP64; the twiddles are a table of exp(+-2 pi i m / nfft).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "spx_common.cuh"

namespace spx {

constexpr int FFT_NMAX = 64;   // largest grid edge
constexpr int FFT_KMAX = 16;   // largest number of distinct G_M - g values per axis
constexpr int FFT_NP = 4;      // unoccupied bands per K5b CTA
constexpr int FFT_XC = 8;      // x planes staged per K5c step

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ void cfma(double2& acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x));
  acc.y = fma(a.x, b.y, fma(a.y, b.x, acc.y));
}

// One separable DFT pass along one axis, G (box index i, value lo + i) -> r (j):
//   out[b, l1, l2, j] = post( sum_i in[b, l1, l2, i] * tw[(lo+i)*j mod n] ),
// post = optional conj, times scale, times mul[l1, l2, j].
struct DftPass {
  const double2* in;
  double2* out;
  const double2* tw;   // exp(+2 pi i m / n), m < n
  const double2* mul;  // or null
  int nin, lo, n, L1, L2, nb;
  int64_t is_i, is_l1, is_l2, is_b;
  int64_t os_j, os_l1, os_l2, os_b;
  int64_t ms_j, ms_l1, ms_l2;
  double scale;
  int conj_out;
};

__global__ void __launch_bounds__(256) dft_pass_kernel(DftPass p) {
  __shared__ double2 tw[FFT_NMAX];
  for (int i = threadIdx.x; i < p.n; i += blockDim.x) tw[i] = p.tw[i];
  __syncthreads();
  const int64_t total = (int64_t)p.n * p.L1 * p.L2 * p.nb;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int j = (int)(t % p.n);
    int64_t r = t / p.n;
    const int l1 = (int)(r % p.L1);
    r /= p.L1;
    const int l2 = (int)(r % p.L2);
    const int b = (int)(r / p.L2);
    const double2* src = p.in + b * p.is_b + l1 * p.is_l1 + l2 * p.is_l2;
    int m = ((p.lo * j) % p.n + p.n) % p.n;
    double2 acc = make_double2(0.0, 0.0);
    for (int i = 0; i < p.nin; ++i) {
      cfma(acc, src[i * p.is_i], tw[m]);
      m += j;
      if (m >= p.n) m -= p.n;
    }
    if (p.conj_out) acc.y = -acc.y;
    acc.x *= p.scale;
    acc.y *= p.scale;
    if (p.mul) acc = cmul(acc, p.mul[l1 * p.ms_l1 + l2 * p.ms_l2 + j * p.ms_j]);
    p.out[b * p.os_b + l1 * p.os_l1 + l2 * p.os_l2 + j * p.os_j] = acc;
  }
}

// box[b*size + gidx[i]] = cpw[b*ngpt + i]; the box is zeroed beforehand.
__global__ void fft_scatter_kernel(const double2* __restrict__ cpw, int ngpt,
                                   const int* __restrict__ gidx, int64_t size,
                                   double2* __restrict__ box) {
  const int64_t b = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ngpt; i += gridDim.x * blockDim.x)
    box[b * size + gidx[i]] = cpw[b * ngpt + i];
}

struct PairParams {
  const double2* A;    // [kl*nocc + n][x][y][z]
  const double2* B;    // [kl*nunocc + n'][x][y][z]
  double2* T2;         // [pairc][x][kz][ky]
  const double2* twf;  // exp(-2 pi i m / n)
  const int* kz;       // distinct kz values (nkz)
  const int* ky;
  int n, nocc, nunocc, nkz, nky;
};

// grid (kl*nocc + n, unoccupied group, x); block (n threads along y, FFT_NP bands)
__global__ void __launch_bounds__(FFT_NMAX * FFT_NP) fft_pair_zy_kernel(PairParams p) {
  extern __shared__ double2 sm[];
  const int n = p.n;
  double2* Apl = sm;                               // [y][z]
  double2* Ez = Apl + n * n;                       // [kk][z]
  double2* Ey = Ez + FFT_KMAX * n;                 // [kk][y]
  double2* T1 = Ey + FFT_KMAX * n;                 // [j][kz][y]
  const int kn = blockIdx.x, grp = blockIdx.y, x = blockIdx.z;
  const int kl = kn / p.nocc;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x, nth = blockDim.x * blockDim.y;
  const double2* a = p.A + ((int64_t)kn * n + x) * n * n;
  for (int i = tid; i < n * n; i += nth) Apl[i] = a[i];
  for (int i = tid; i < FFT_KMAX * n; i += nth) {
    const int kk = i / n, z = i - kk * n;
    Ez[i] = kk < p.nkz ? p.twf[(p.kz[kk] * z) % n] : make_double2(0.0, 0.0);
    Ey[i] = kk < p.nky ? p.twf[(p.ky[kk] * z) % n] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  const int y = threadIdx.x, j = threadIdx.y;
  const int np = grp * FFT_NP + j;
  if (np < p.nunocc) {
    const double2* bl = p.B + (((int64_t)kl * p.nunocc + np) * n + x) * n * n + (int64_t)y * n;
    const double2* al = Apl + y * n;
    double2 acc[FFT_KMAX];
#pragma unroll
    for (int kk = 0; kk < FFT_KMAX; ++kk) acc[kk] = make_double2(0.0, 0.0);
    for (int z = 0; z < n; ++z) {
      const double2 prod = cmul(al[z], __ldg(bl + z));
#pragma unroll
      for (int kk = 0; kk < FFT_KMAX; ++kk)
        if (kk < p.nkz) cfma(acc[kk], Ez[kk * n + z], prod);
    }
    for (int kk = 0; kk < p.nkz; ++kk) T1[(j * FFT_KMAX + kk) * n + y] = acc[kk];
  }
  __syncthreads();
  // y pass: T2[pair][x][kz][ky] = sum_y Ey[ky][y] T1[j][kz][y]
  const int nout = FFT_NP * p.nkz * p.nky;
  for (int o = tid; o < nout; o += nth) {
    const int jj = o / (p.nkz * p.nky);
    const int rem = o - jj * p.nkz * p.nky;
    const int kz = rem / p.nky, ky = rem - kz * p.nky;
    const int npp = grp * FFT_NP + jj;
    if (npp >= p.nunocc) continue;
    const double2* t1 = T1 + (jj * FFT_KMAX + kz) * n;
    const double2* ey = Ey + ky * n;
    double2 s = make_double2(0.0, 0.0);
    for (int yy = 0; yy < n; ++yy) cfma(s, ey[yy], t1[yy]);
    const int64_t pairc = (int64_t)kn * p.nunocc + npp;
    p.T2[((pairc * n + x) * p.nkz + kz) * p.nky + ky] = s;
  }
}

// ---------------------------------------------------------------------------
// K5b as a line FFT, for grid edges n = 16 r (r = 1..4): the 48-point transform of
// the 48^3 grid is radix 16 x 3. With z = r n1 + n2 and k = k1 + 16 k2,
//   X[k] = sum_{n2<r} W_n^{n2 k1} W_r^{n2 k2} F_{n2}[k1],
//   F_{n2}[k1] = sum_{n1<16} x[r n1 + n2] W_16^{n1 k1},
// so thread (line, n2) transforms its 16 decimated points in registers (radix 4 x 4),
// applies W_n^{n2 k1}, and the r partial spectra of a line are combined, through
// shared memory, only at the k the gather needs. W = exp(-2 pi i / n) (forward).

// 4-point forward DFT in place: (x0, x1, x2, x3) -> (X0, X1, X2, X3), W_4 = -i.
__device__ __forceinline__ void dft4_fwd(double2& x0, double2& x1, double2& x2, double2& x3) {
  const double2 t0 = make_double2(x0.x + x2.x, x0.y + x2.y), t1 = make_double2(x0.x - x2.x, x0.y - x2.y);
  const double2 t2 = make_double2(x1.x + x3.x, x1.y + x3.y), t3 = make_double2(x1.x - x3.x, x1.y - x3.y);
  x0 = make_double2(t0.x + t2.x, t0.y + t2.y);
  x2 = make_double2(t0.x - t2.x, t0.y - t2.y);
  x1 = make_double2(t1.x + t3.y, t1.y - t3.x);  // t1 - i t3
  x3 = make_double2(t1.x - t3.y, t1.y + t3.x);  // t1 + i t3
}

// 16-point forward DFT of v (natural order in): n1 = 4a + b, k1 = c + 4d; 4-point
// transforms over a, twiddles W_16^{bc} (w16[m] = W_16^m), 4-point transforms over b.
// The output is left digit-reversed: X[k1] is v[fft16_pos(k1)].
__host__ __device__ constexpr int fft16_pos(int k1) { return 4 * (k1 & 3) + (k1 >> 2); }
__device__ __forceinline__ void fft16_fwd(double2 (&v)[16], const double2* __restrict__ w16) {
#pragma unroll
  for (int b = 0; b < 4; ++b) dft4_fwd(v[b], v[4 + b], v[8 + b], v[12 + b]);  // v[4c + b] = Y_b[c]
#pragma unroll
  for (int b = 1; b < 4; ++b)
#pragma unroll
    for (int c = 1; c < 4; ++c) v[4 * c + b] = cmul(v[4 * c + b], w16[b * c]);
#pragma unroll
  for (int c = 0; c < 4; ++c) dft4_fwd(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);  // v[4c + d] = X[c + 4d]
}

// Shared-memory row strides of the line FFT: 17 complex per (line, phase) spectrum and
// n + 1 per kz row, so that lanes walking lines hit distinct banks.
constexpr int FFTR_LD = 17;

struct PairFftParams {
  const double2* A;    // [kl*nocc + n][x][y][z]
  const double2* B;    // [kl*nunocc + n'][x][y][z]
  double2* T2;         // [pairc][x][kz][ky]
  const double2* twf;  // W_n^m = exp(-2 pi i m / n), m < n
  const int* kz;       // distinct kz values (nkz)
  const int* ky;
  int n, r, bpc, nocc, nunocc, nkz, nky;
};

// grid (kl*nocc + n, group of bpc unoccupied bands, x); block bpc * n * r threads:
// thread t of band j is line t / r, decimation phase t % r.
__global__ void __launch_bounds__(512) fft_pair_zy_radix_kernel(PairFftParams p) {
  extern __shared__ double2 smr[];
  const int n = p.n, r = p.r, per = n * r;
  double2* tw = smr;                                 // [n]
  double2* w16 = tw + n;                             // [16]
  double2* Fb = w16 + 16;                            // [bpc][n lines][r][FFTR_LD]
  double2* T1 = Fb + (size_t)p.bpc * n * r * FFTR_LD;  // [bpc][FFT_KMAX][n + 1]
  const int kn = blockIdx.x, grp = blockIdx.y, x = blockIdx.z;
  const int kl = kn / p.nocc;
  for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = p.twf[i];
  for (int i = threadIdx.x; i < 16; i += blockDim.x) w16[i] = p.twf[i * r];
  __syncthreads();
  const int j = threadIdx.x / per, t = threadIdx.x - j * per;
  const int np = grp * p.bpc + j;
  const bool live = j < p.bpc && np < p.nunocc;
  double2* F = Fb + (size_t)j * n * r * FFTR_LD;
  double2* T = T1 + (size_t)j * FFT_KMAX * (n + 1);
  const int tl = n + 1;
  // z pass: line y = t / r of the product plane A(x, y, .) B(x, y, .)
  if (live) {
    const int y = t / r, n2 = t - (t / r) * r;
    const double2* a = p.A + (((int64_t)kn * n + x) * n + y) * n;
    const double2* bl = p.B + ((((int64_t)kl * p.nunocc + np) * n + x) * n + y) * n;
    double2 v[16];
#pragma unroll
    for (int n1 = 0; n1 < 16; ++n1) {
      const int z = r * n1 + n2;
      v[n1] = cmul(__ldg(a + z), __ldg(bl + z));
    }
    fft16_fwd(v, w16);
    double2* f = F + ((size_t)y * r + n2) * FFTR_LD;
#pragma unroll
    for (int k1 = 0; k1 < 16; ++k1) f[k1] = n2 ? cmul(v[fft16_pos(k1)], tw[n2 * k1]) : v[fft16_pos(k1)];
  }
  __syncthreads();
  // combine at the needed kz: T[kk][y]
  if (live) {
    for (int o = t; o < p.nkz * n; o += per) {
      const int kk = o / n, y = o - kk * n;
      const int k = p.kz[kk], k1 = k & 15, k2 = k >> 4;
      const double2* f = F + (size_t)y * r * FFTR_LD + k1;
      double2 acc = f[0];
      for (int n2 = 1; n2 < r; ++n2) cfma(acc, f[n2 * FFTR_LD], tw[(16 * n2 * k2) % n]);
      T[kk * tl + y] = acc;
    }
  }
  __syncthreads();
  // y pass: line kk of T along y
  if (live && t < p.nkz * r) {
    const int kk = t / r, n2 = t - (t / r) * r;
    double2 v[16];
#pragma unroll
    for (int n1 = 0; n1 < 16; ++n1) v[n1] = T[kk * tl + r * n1 + n2];
    fft16_fwd(v, w16);
    double2* f = F + ((size_t)kk * r + n2) * FFTR_LD;
#pragma unroll
    for (int k1 = 0; k1 < 16; ++k1) f[k1] = n2 ? cmul(v[fft16_pos(k1)], tw[n2 * k1]) : v[fft16_pos(k1)];
  }
  __syncthreads();
  if (live) {
    const int64_t pairc = (int64_t)kn * p.nunocc + np;
    double2* out = p.T2 + (pairc * n + x) * p.nkz * p.nky;
    for (int o = t; o < p.nkz * p.nky; o += per) {
      const int kk = o / p.nky, kyi = o - kk * p.nky;
      const int k = p.ky[kyi], k1 = k & 15, k2 = k >> 4;
      const double2* f = F + (size_t)kk * r * FFTR_LD + k1;
      double2 acc = f[0];
      for (int n2 = 1; n2 < r; ++n2) cfma(acc, f[n2 * FFTR_LD], tw[(16 * n2 * k2) % n]);
      out[o] = acc;
    }
  }
}

struct GatherParams {
  const double2* T2;   // [pairc][x][kz][ky]
  const double2* twf;
  const int* kx;       // distinct kx values
  const int* gmap;     // per ig: ix | iy << 8 | iz << 16
  double2* cprod;      // already offset to (first pair of the chunk, column col0)
  int64_t ldc;
  int n, nkx, nky, nkz, ngptm;
};

// grid: one CTA per pair of the chunk
__global__ void __launch_bounds__(256) fft_pair_x_kernel(GatherParams p) {
  extern __shared__ double2 sm[];
  const int n = p.n, plane = p.nkz * p.nky;
  double2* Ex = sm;                        // [kk][x]
  double2* F = Ex + FFT_KMAX * n;          // [ig]
  double2* Ts = F + p.ngptm;               // [xc][kz][ky]
  const int64_t pairc = blockIdx.x;
  for (int i = threadIdx.x; i < FFT_KMAX * n; i += blockDim.x) {
    const int kk = i / n, x = i - kk * n;
    Ex[i] = kk < p.nkx ? p.twf[(p.kx[kk] * x) % n] : make_double2(0.0, 0.0);
  }
  for (int i = threadIdx.x; i < p.ngptm; i += blockDim.x) F[i] = make_double2(0.0, 0.0);
  const double2* t2 = p.T2 + pairc * n * plane;
  for (int x0 = 0; x0 < n; x0 += FFT_XC) {
    const int xc = min(FFT_XC, n - x0);
    __syncthreads();
    for (int i = threadIdx.x; i < xc * plane; i += blockDim.x) Ts[i] = t2[(int64_t)x0 * plane + i];
    __syncthreads();
    for (int ig = threadIdx.x; ig < p.ngptm; ig += blockDim.x) {
      const int g = p.gmap[ig];
      const int ix = g & 255, iy = (g >> 8) & 255, iz = (g >> 16) & 255;
      double2 acc = F[ig];
      for (int xx = 0; xx < xc; ++xx) cfma(acc, Ex[ix * n + x0 + xx], Ts[xx * plane + iz * p.nky + iy]);
      F[ig] = acc;
    }
  }
  for (int ig = threadIdx.x; ig < p.ngptm; ig += blockDim.x) {
    double2* o = p.cprod + pairc + p.ldc * ig;
    double2 v = *o;
    v.x += F[ig].x;
    v.y += F[ig].y;
    *o = v;
  }
}

// ---------------------------------------------------------------------------
// host

struct Box3 {
  int lo[3] = {0, 0, 0}, dim[3] = {1, 1, 1};
  int64_t size() const { return (int64_t)dim[0] * dim[1] * dim[2]; }
};

static Box3 box_of(const int* g, int n) {
  Box3 b;
  if (n == 0) return b;
  int hi[3];
  for (int c = 0; c < 3; ++c) b.lo[c] = hi[c] = g[c];
  for (int i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) {
      b.lo[c] = std::min(b.lo[c], g[3 * i + c]);
      hi[c] = std::max(hi[c], g[3 * i + c]);
    }
  for (int c = 0; c < 3; ++c) b.dim[c] = hi[c] - b.lo[c] + 1;
  return b;
}

struct FftPlan {
  int n = 0;
  Box3 b1, b2, bs;
  std::vector<int> gidx1, gidx2, ks[3], gmap;
  std::vector<double2> twb, twf;
};

static int plan_fft(spx_ctx* ctx, const spx_pw_desc* d, FftPlan* pl) {
  const int n = d->nfft;
  if (n < 2 || n > FFT_NMAX)
    return set_error(ctx, SPX_EINVAL, "nfft must be in 2..64 for the FFT branch");
  if (d->ngptm > 4096) return set_error(ctx, SPX_EINVAL, "FFT branch supports ngptm <= 4096");
  if (d->step_radius < 0 || d->step_radius > 4 || d->vol <= 0.0)
    return set_error(ctx, SPX_EINVAL, "bad plane-wave descriptor (step_radius must be 0..4)");
  if ((d->ngpt1 > 0 && !d->gpt1) || (d->ngpt2 > 0 && !d->gpt2) || (d->ngptm > 0 && !d->gptm) || !d->cstep)
    return set_error(ctx, SPX_EINVAL, "null plane-wave descriptor array");
  pl->n = n;
  pl->b1 = box_of(d->gpt1, d->ngpt1);
  pl->b2 = box_of(d->gpt2, d->ngpt2);
  for (int c = 0; c < 3; ++c) {
    pl->bs.lo[c] = -d->step_radius;
    pl->bs.dim[c] = 2 * d->step_radius + 1;
  }
  auto lin = [](const Box3& b, const int* g) {
    return (int)((g[0] - b.lo[0]) + (int64_t)b.dim[0] * ((g[1] - b.lo[1]) + (int64_t)b.dim[1] * (g[2] - b.lo[2])));
  };
  if (pl->b1.size() > (1 << 26) || pl->b2.size() > (1 << 26))
    return set_error(ctx, SPX_EINVAL, "plane-wave G boxes too large");
  pl->gidx1.resize(d->ngpt1);
  for (int i = 0; i < d->ngpt1; ++i) pl->gidx1[i] = lin(pl->b1, d->gpt1 + 3 * i);
  pl->gidx2.resize(d->ngpt2);
  for (int i = 0; i < d->ngpt2; ++i) pl->gidx2[i] = lin(pl->b2, d->gpt2 + 3 * i);
  // distinct (G_M - g) mod n per axis, and each ig's position in them
  std::vector<int> idx[3];
  for (int c = 0; c < 3; ++c) {
    std::vector<int> v(d->ngptm);
    for (int i = 0; i < d->ngptm; ++i) v[i] = (((d->gptm[3 * i + c] - d->gshift[c]) % n) + n) % n;
    pl->ks[c] = v;
    std::sort(pl->ks[c].begin(), pl->ks[c].end());
    pl->ks[c].erase(std::unique(pl->ks[c].begin(), pl->ks[c].end()), pl->ks[c].end());
    if ((int)pl->ks[c].size() > FFT_KMAX)
      return set_error(ctx, SPX_ENOTSUP,
                       "FFT branch: more than 16 distinct mixed-basis G components per axis; "
                       "use the explicit convolution (nfft = 0)");
    idx[c].resize(d->ngptm);
    for (int i = 0; i < d->ngptm; ++i)
      idx[c][i] = (int)(std::lower_bound(pl->ks[c].begin(), pl->ks[c].end(), v[i]) - pl->ks[c].begin());
  }
  pl->gmap.resize(d->ngptm);
  for (int i = 0; i < d->ngptm; ++i) pl->gmap[i] = idx[0][i] | (idx[1][i] << 8) | (idx[2][i] << 16);
  pl->twb.resize(n);
  pl->twf.resize(n);
  for (int m = 0; m < n; ++m) {
    const long double ang = 2.0L * 3.14159265358979323846264338327950288L * m / n;
    const double c = (double)cosl(ang), s = (double)sinl(ang);
    pl->twb[m] = make_double2(c, s);
    pl->twf[m] = make_double2(c, -s);
  }
  return SPX_OK;
}

static size_t fft_perk_bytes(const FftPlan& pl, int nocc, int nunocc, int nkzky) {
  const int64_t n = pl.n, n3 = n * n * n;
  const int64_t nb = std::max(nocc, nunocc);
  const Box3& bm = pl.b1.size() > pl.b2.size() ? pl.b1 : pl.b2;
  const int64_t box = nb * std::max(pl.b1.size(), pl.b2.size());
  const int64_t ta = nb * n * std::max(pl.b1.dim[1] * pl.b1.dim[2], pl.b2.dim[1] * pl.b2.dim[2]);
  const int64_t tb = nb * n * n * std::max(pl.b1.dim[2], pl.b2.dim[2]);
  (void)bm;
  return align_up(16 * (size_t)box, 256) + align_up(16 * (size_t)ta, 256) + align_up(16 * (size_t)tb, 256) +
         align_up(16 * (size_t)(nocc + nunocc) * n3, 256) +
         align_up(16 * (size_t)nocc * nunocc * n * nkzky, 256) + 16 * (size_t)n * n * 9 * 2 + 2048;
}

size_t wfprod_pw_fft_workspace(const spx_pw_desc* d, int nk, int nocc, int nunocc) {
  spx_ctx dummy;
  FftPlan pl;
  if (plan_fft(&dummy, d, &pl)) return 0;
  const size_t perk = fft_perk_bytes(pl, nocc, nunocc, (int)(pl.ks[1].size() * pl.ks[2].size()));
  const size_t fixed = 16 * (size_t)pl.n * pl.n * pl.n + 64 * 1024 +
                       4 * (size_t)(d->ngpt1 + d->ngpt2 + 2 * d->ngptm) + 16 * 1024;
  const size_t budget = (size_t)6 << 30;
  const size_t kchunk = std::max<size_t>(1, std::min<size_t>((size_t)nk, budget / perk));
  return fixed + kchunk * perk;
}

// Three passes G box -> r grid for nb bands: box [b][gz][gy][gx] -> out [b][x][y][z].
static int band_grids(spx_ctx* ctx, const Box3& bx, int nb, const double2* box, double2* ta,
                      double2* tb, double2* out, const double2* twb, int n, int conj_out,
                      double scale, const double2* mul, cudaStream_t s, int* launches) {
  if (nb == 0) return SPX_OK;
  auto run = [&](DftPass p) -> int {
    const int64_t total = (int64_t)p.n * p.L1 * p.L2 * p.nb;
    const int grid = (int)std::min<int64_t>((total + 255) / 256, (int64_t)ctx->num_sms * 16);
    dft_pass_kernel<<<grid, 256, 0, s>>>(p);
    ++*launches;
    return check_cuda(ctx, cudaGetLastError(), "dft_pass_kernel launch");
  };
  const int64_t X = bx.dim[0], Y = bx.dim[1], Z = bx.dim[2];
  DftPass p{};
  p.tw = twb;
  p.n = n;
  p.nb = nb;
  p.scale = 1.0;
  // x: box[b][gz][gy][gx] -> ta[b][gz][gy][x]
  p.in = box; p.out = ta; p.nin = (int)X; p.lo = bx.lo[0]; p.L1 = (int)Y; p.L2 = (int)Z;
  p.is_i = 1; p.is_l1 = X; p.is_l2 = X * Y; p.is_b = X * Y * Z;
  p.os_j = 1; p.os_l1 = n; p.os_l2 = (int64_t)n * Y; p.os_b = (int64_t)n * Y * Z;
  int rc = run(p);
  if (rc) return rc;
  // y: ta[b][gz][gy][x] -> tb[b][x][y][gz]
  p.in = ta; p.out = tb; p.nin = (int)Y; p.lo = bx.lo[1]; p.L1 = n; p.L2 = (int)Z;
  p.is_i = n; p.is_l1 = 1; p.is_l2 = (int64_t)n * Y; p.is_b = (int64_t)n * Y * Z;
  p.os_j = Z; p.os_l1 = (int64_t)n * Z; p.os_l2 = 1; p.os_b = (int64_t)n * n * Z;
  if ((rc = run(p))) return rc;
  // z: tb[b][x][y][gz] -> out[b][x][y][z], with the post-operation
  p.in = tb; p.out = out; p.nin = (int)Z; p.lo = bx.lo[2]; p.L1 = n; p.L2 = n;
  p.is_i = 1; p.is_l1 = Z; p.is_l2 = (int64_t)n * Z; p.is_b = (int64_t)n * n * Z;
  p.os_j = 1; p.os_l1 = n; p.os_l2 = (int64_t)n * n; p.os_b = (int64_t)n * n * n;
  p.conj_out = conj_out; p.scale = scale; p.mul = mul;
  p.ms_j = 1; p.ms_l1 = n; p.ms_l2 = (int64_t)n * n;
  return run(p);
}

int wfprod_pw_fft_run(spx_ctx* ctx, const spx_pw_desc* d, int nk, int nocc, int nunocc,
                      const double2* c1, const double2* c2, double2* cprod, int64_t ldc, int col0,
                      void* ws, size_t ws_bytes, cudaStream_t s, int* launches) {
  FftPlan pl;
  int rc = plan_fft(ctx, d, &pl);
  if (rc) return rc;
  if (d->ngptm == 0 || nk == 0 || nocc == 0 || nunocc == 0 || !ws) return SPX_OK;
  if ((nunocc + FFT_NP - 1) / FFT_NP > 65535)
    return set_error(ctx, SPX_EINVAL, "too many unoccupied bands for the FFT branch");
  const int n = pl.n, nkx = (int)pl.ks[0].size(), nky = (int)pl.ks[1].size(), nkz = (int)pl.ks[2].size();
  const int64_t n3 = (int64_t)n * n * n;
  Carve cv{(char*)ws, ws_bytes};
  int* d_g1 = cv.take<int>(d->ngpt1);
  int* d_g2 = cv.take<int>(d->ngpt2);
  int* d_ks[3];
  for (int c = 0; c < 3; ++c) d_ks[c] = cv.take<int>(pl.ks[c].size());
  int* d_gmap = cv.take<int>(d->ngptm);
  double2* d_twb = cv.take<double2>(n);
  double2* d_twf = cv.take<double2>(n);
  double2* d_cs = cv.take<double2>((size_t)pl.bs.size());
  double2* theta = cv.take<double2>((size_t)n3);
  const size_t perk = fft_perk_bytes(pl, nocc, nunocc, nky * nkz);
  if (!cv.ok || cv.left < perk) return set_error(ctx, SPX_ENOMEM, "FFT-branch scratch too small");
  // grid limit of K5c: one CTA per pair of a chunk along x
  const size_t pairs_k = (size_t)nocc * nunocc;
  if (pairs_k > 2147483647u) return set_error(ctx, SPX_EINVAL, "too many band pairs per k point");
  const int kchunk = (int)std::min<size_t>({(size_t)nk, cv.left / perk, 2147483647u / pairs_k});
  const int nbmax = std::max(nocc, nunocc) * kchunk;
  // per-chunk buffers sized for kchunk k points
  double2* box = cv.take<double2>((size_t)nbmax * std::max(pl.b1.size(), pl.b2.size()));
  // pass buffers: the bands of a chunk, or the step-function box for theta
  const size_t ta_n = std::max<size_t>(
      (size_t)nbmax * n * std::max(pl.b1.dim[1] * pl.b1.dim[2], pl.b2.dim[1] * pl.b2.dim[2]),
      (size_t)n * pl.bs.dim[1] * pl.bs.dim[2]);
  const size_t tb_n = std::max<size_t>((size_t)nbmax * n * n * std::max(pl.b1.dim[2], pl.b2.dim[2]),
                                       (size_t)n * n * pl.bs.dim[2]);
  double2* ta = cv.take<double2>(ta_n);
  double2* tb = cv.take<double2>(tb_n);
  double2* A = cv.take<double2>((size_t)kchunk * nocc * n3);
  double2* Bg = cv.take<double2>((size_t)kchunk * nunocc * n3);
  double2* T2 = cv.take<double2>((size_t)kchunk * nocc * nunocc * n * nky * nkz);
  if (!cv.ok) return set_error(ctx, SPX_ENOMEM, "FFT-branch scratch too small");
  auto up = [&](void* dst, const void* src, size_t bytes) {
    return bytes ? check_cuda(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s), "copy plan") : SPX_OK;
  };
  if ((rc = up(d_g1, pl.gidx1.data(), 4 * pl.gidx1.size())) || (rc = up(d_g2, pl.gidx2.data(), 4 * pl.gidx2.size())) ||
      (rc = up(d_ks[0], pl.ks[0].data(), 4 * nkx)) || (rc = up(d_ks[1], pl.ks[1].data(), 4 * nky)) ||
      (rc = up(d_ks[2], pl.ks[2].data(), 4 * nkz)) || (rc = up(d_gmap, pl.gmap.data(), 4 * pl.gmap.size())) ||
      (rc = up(d_twb, pl.twb.data(), 16 * n)) || (rc = up(d_twf, pl.twf.data(), 16 * n)) ||
      (rc = up(d_cs, d->cstep, 16 * (size_t)pl.bs.size())))
    return rc;
  if ((rc = check_cuda(ctx, cudaStreamSynchronize(s), "copy plan"))) return rc;
  // theta(r) from the step-function box (already laid out x fastest)
  if ((rc = band_grids(ctx, pl.bs, 1, d_cs, ta, tb, theta, d_twb, n, 0, 1.0, nullptr, s, launches)))
    return rc;
  const size_t zy_smem = sizeof(double2) * ((size_t)n * n + 2 * FFT_KMAX * n + (size_t)FFT_NP * FFT_KMAX * n);
  const size_t x_smem = sizeof(double2) * ((size_t)FFT_KMAX * n + d->ngptm + (size_t)FFT_XC * nky * nkz);
  cudaFuncSetAttribute(fft_pair_zy_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zy_smem);
  // grid edges 16 r (r <= 4) take the line FFT; bpc bands per CTA within 108 KB of
  // shared memory and 512 threads
  const bool radix = n % 16 == 0 && n / 16 >= 1 && n / 16 <= 4;
  const size_t band_smem = sizeof(double2) * ((size_t)n * (n / 16) * FFTR_LD + (size_t)FFT_KMAX * (n + 1));
  const int bpc = radix ? std::max(1, std::min({4, 512 / (n * (n / 16)), (int)((108 << 10) / band_smem)})) : 1;
  const size_t radix_smem = sizeof(double2) * ((size_t)n + 16) + bpc * band_smem;
  if (radix)
    cudaFuncSetAttribute(fft_pair_zy_radix_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)radix_smem);
  cudaFuncSetAttribute(fft_pair_x_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)x_smem);
  for (int k0 = 0; k0 < nk; k0 += kchunk) {
    const int kn = std::min(kchunk, nk - k0);
    // occupied: conj(phi)/sqrt(vol) * theta; unoccupied: phi / nnfft
    const int nb1 = kn * nocc, nb2 = kn * nunocc;
    if ((rc = check_cuda(ctx, cudaMemsetAsync(box, 0, 16 * (size_t)nb1 * pl.b1.size(), s), "zero box"))) return rc;
    if (d->ngpt1 > 0) {
      dim3 g((d->ngpt1 + 255) / 256, nb1);
      fft_scatter_kernel<<<g, 256, 0, s>>>(c1 + (int64_t)k0 * nocc * d->ngpt1, d->ngpt1, d_g1, pl.b1.size(), box);
      ++*launches;
    }
    if ((rc = band_grids(ctx, pl.b1, nb1, box, ta, tb, A, d_twb, n, 1, 1.0 / std::sqrt(d->vol), theta, s, launches)))
      return rc;
    if ((rc = check_cuda(ctx, cudaMemsetAsync(box, 0, 16 * (size_t)nb2 * pl.b2.size(), s), "zero box"))) return rc;
    if (d->ngpt2 > 0) {
      dim3 g((d->ngpt2 + 255) / 256, nb2);
      fft_scatter_kernel<<<g, 256, 0, s>>>(c2 + (int64_t)k0 * nunocc * d->ngpt2, d->ngpt2, d_g2, pl.b2.size(), box);
      ++*launches;
    }
    if ((rc = band_grids(ctx, pl.b2, nb2, box, ta, tb, Bg, d_twb, n, 0, 1.0 / (double)n3, nullptr, s, launches)))
      return rc;
    if (radix) {
      PairFftParams pr{A, Bg, T2, d_twf, d_ks[2], d_ks[1], n, n / 16, bpc, nocc, nunocc, nkz, nky};
      dim3 gz(nb1, (nunocc + bpc - 1) / bpc, n);
      fft_pair_zy_radix_kernel<<<gz, bpc * n * (n / 16), radix_smem, s>>>(pr);
      if ((rc = check_cuda(ctx, cudaGetLastError(), "fft_pair_zy_radix_kernel launch"))) return rc;
    } else {
      PairParams pp{A, Bg, T2, d_twf, d_ks[2], d_ks[1], n, nocc, nunocc, nkz, nky};
      dim3 gz(nb1, (nunocc + FFT_NP - 1) / FFT_NP, n), bz(n, FFT_NP);
      fft_pair_zy_kernel<<<gz, bz, zy_smem, s>>>(pp);
      if ((rc = check_cuda(ctx, cudaGetLastError(), "fft_pair_zy_kernel launch"))) return rc;
    }
    ++*launches;
    GatherParams gp{T2, d_twf, d_ks[0], d_gmap, cprod + (int64_t)k0 * nocc * nunocc + ldc * col0, ldc,
                    n, nkx, nky, nkz, d->ngptm};
    fft_pair_x_kernel<<<(unsigned)((int64_t)kn * nocc * nunocc), 256, x_smem, s>>>(gp);
    if ((rc = check_cuda(ctx, cudaGetLastError(), "fft_pair_x_kernel launch"))) return rc;
    ++*launches;
  }
  return SPX_OK;
}

}  // namespace spx
