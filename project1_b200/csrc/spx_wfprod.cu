// K4: mixed-product-basis projections M_I,nn'k of SPEX (wavefproducts2_mt and the
// explicit-convolution branch of wavefproducts2_pw), complex FP64.
//
// Muffin tin (src/wavefproducts.f:95-431). For every atom a, k point and occupied
// band n the reference builds
//   mat_n(lm1, I) = sum_lm cmt1(lm, n) * integral(ln, ln1, lln) * gaunt1(l1, l, LL, m, MM)
// and then cprod(n', n, k, I_a) += cexp_a * sum_lm1 cmt2(lm1, n') * conj(mat_n(lm1, I)).
// The first step is a fixed sparse linear map T (Gaunt x radial integral) applied
// to cmt1: the host flattens T into CSR rows over the outputs (I, lm1) once per
// call and K4a applies it with one CTA per (k, a, n). The second step is a
// complex GEMM for every (a, k): K4c with B = mat (K-contiguous rows lm1) and
// the atom phase as the complex scale.
//
// Interstitial (src/wavefproducts.f:760-997). cpw0(G0) = sum_G1 cstep(G0 - G1)
// cpw1(G1) is a 3-D stencil: K4b scatters the occupied coefficients to a dense
// G box and applies the (2 sr + 1)^3 step-function stencil over the box of all
// G2 - G_M + g. The gathered matrix cpw3(ig2, ig) = cpw0(G2 - G_M + g) is never
// stored: its element address is linear in G, base(n, ig) + off(ig2), so K4c
// reads it through two index vectors while staging the B tile.
//
// K4c: C(m, col) += alpha * sum_k A(m, k) * conj(B(col, k)), A rows and B rows
// K-contiguous (B possibly gathered), on the FP64 DMMA path (mma.sync
// m16n8k8 f64): 64x64 complex tiles, four warps of 32x32, two-stage cp.async
// pipeline with zero fill at the edges, output rows m contiguous in cprod.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "spx_common.cuh"
#include "spx_zgemm.h"

namespace spx {

// ---------------------------------------------------------------------------
// K4c: batched complex GEMM with a gathered B operand

constexpr int ZG_B = 64;             // tile edge (rows m and columns col)
constexpr int ZG_KC = 16;            // K per pipeline stage
constexpr int ZG_ROW = ZG_KC + 4;    // padded shared row, double2 units
constexpr int ZG_THREADS = 128;

// ZgParams: see spx_zgemm.h

__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
               "r"(valid ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ void dmma8(double (&d)[4], const double* a, const double* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

struct __align__(16) ZgSmem {
  double2 a[2][ZG_B][ZG_ROW];
  double2 b[2][ZG_B][ZG_ROW];
};

__global__ void __launch_bounds__(ZG_THREADS, 2) zgemm_gather_kernel(ZgParams prm) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  ZgSmem& sm = *reinterpret_cast<ZgSmem*>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tile = blockIdx.x;
  const int tm = tile % prm.mtiles, tn = tile / prm.mtiles;
  const int b = blockIdx.y;
  const int b1 = b % prm.nb1, b2 = b / prm.nb1;
  const int m0 = tm * ZG_B, c0 = tn * ZG_B;
  const int Kb = (prm.K_last > 0 && b == (int)gridDim.y - 1) ? prm.K_last : prm.K;

  // loader role: thread -> (row r, 8 consecutive k); rows of A are m, rows of B col
  const int lr = threadIdx.x >> 1, lk = (threadIdx.x & 1) * 8;
  const bool a_ok = m0 + lr < prm.M;
  const int64_t a_mstride = prm.a_mcontig ? 1 : prm.lda, a_kstride = prm.a_mcontig ? prm.lda : 1;
  const double2* a_row = prm.A + b1 * prm.sA1 + b2 * prm.sA2 + (int64_t)(a_ok ? m0 + lr : 0) * a_mstride;
  const int col = c0 + lr;
  const bool b_ok = col < prm.ncol;
  const double2* b_row;
  {
    const int cc = b_ok ? col : 0;
    const int n = cc / prm.ncin, c = cc - n * prm.ncin;
    b_row = prm.B + b1 * prm.sB1 + b2 * prm.sB2 + (int64_t)n * prm.sBn +
            (prm.cOff ? prm.cOff[c] : (int64_t)c * prm.sBc);
  }
  auto issue = [&](int st, int k0) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int k = k0 + lk + j;
      const bool kin = k < Kb;
      const int kk = kin ? k : 0;
      cp_async16(&sm.a[st][lr][lk + j], a_row + kk * a_kstride, a_ok && kin);
      const int64_t ko = prm.kOff ? (int64_t)__ldg(prm.kOff + kk) : (int64_t)kk;
      cp_async16(&sm.b[st][lr][lk + j], b_ok && kin ? b_row + ko : prm.B, b_ok && kin);
    }
    cp_async_commit();
  };

  const int nst = (Kb + ZG_KC - 1) / ZG_KC;
  issue(0, 0);

  const int wi = warp & 1, wj = warp >> 1;
  const int g = lane >> 2, t = lane & 3;
  double accR[2][4][4], accI[2][4][4];
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int r = 0; r < 4; ++r) accR[mt][nt][r] = accI[mt][nt][r] = 0.0;

  for (int s = 0; s < nst; ++s) {
    const int st = s & 1;
    if (s + 1 < nst) {
      issue(st ^ 1, (s + 1) * ZG_KC);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < ZG_KC / 8; ++ks) {
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        double ar[4], ai[4];
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const double2 v = sm.a[st][32 * wi + 16 * mt + g + 8 * h][ks * 8 + t + 4 * q];
            ar[2 * q + h] = v.x;
            ai[2 * q + h] = v.y;
          }
#pragma unroll
        for (int np = 0; np < 2; ++np) {
          double br[2][2], bim[2][2], bneg[2][2];
#pragma unroll
          for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int q = 0; q < 2; ++q) {
              const double2 v = sm.b[st][32 * wj + 8 * (2 * np + h) + g][ks * 8 + t + 4 * q];
              br[h][q] = v.x;
              bim[h][q] = v.y;
              bneg[h][q] = -v.y;
            }
          // A conj(B): re += ar br + ai bi, im += ai br - ar bi
          dmma8(accR[mt][2 * np], ar, br[0]);
          dmma8(accR[mt][2 * np + 1], ar, br[1]);
          dmma8(accI[mt][2 * np], ai, br[0]);
          dmma8(accI[mt][2 * np + 1], ai, br[1]);
          dmma8(accR[mt][2 * np], ai, bim[0]);
          dmma8(accR[mt][2 * np + 1], ai, bim[1]);
          dmma8(accI[mt][2 * np], ar, bneg[0]);
          dmma8(accI[mt][2 * np + 1], ar, bneg[1]);
        }
      }
    }
    __syncthreads();  // stage st is refilled by the next iteration's issue
  }

  const double2 al = prm.alpha ? prm.alpha[b1] : prm.alpha_v;
  double2* ob = prm.O + b1 * prm.sO1 + b2 * prm.sO2;
#pragma unroll
  for (int nt = 0; nt < 4; ++nt)
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int cl = c0 + 32 * wj + 8 * nt + 2 * t + e;
      if (cl >= prm.ncol) continue;
      const int n = cl / prm.ncin, c = cl - n * prm.ncin;
      double2* oc = ob + (int64_t)n * prm.sOn + (int64_t)c * prm.sOc;
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int m = m0 + 32 * wi + 16 * mt + g + 8 * h;
          if (m >= prm.M) continue;
          const int r = 2 * h + e;
          const double re = accR[mt][nt][r], im = accI[mt][nt][r];
          double2 v = oc[m];
          v.x += al.x * re - al.y * im;
          v.y += al.x * im + al.y * re;
          oc[m] = v;
        }
    }
}

int launch_zgemm(spx_ctx* ctx, ZgParams prm, int nbatch, cudaStream_t s) {
  if (prm.M <= 0 || prm.ncol <= 0 || prm.K <= 0 || nbatch <= 0) return SPX_OK;
  prm.mtiles = (prm.M + ZG_B - 1) / ZG_B;
  prm.ntiles = (prm.ncol + ZG_B - 1) / ZG_B;
  const int64_t tiles = (int64_t)prm.mtiles * prm.ntiles;
  if (tiles > 0x7fffffff || nbatch > 65535)
    return set_error(ctx, SPX_EINVAL, "product GEMM grid too large");
  const size_t smem = sizeof(ZgSmem);
  cudaFuncSetAttribute(zgemm_gather_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  dim3 grid((unsigned)tiles, (unsigned)nbatch);
  zgemm_gather_kernel<<<grid, ZG_THREADS, smem, s>>>(prm);
  return check_cuda(ctx, cudaGetLastError(), "zgemm_gather_kernel launch");
}

// ---------------------------------------------------------------------------
// K4a: sparse Gaunt x radial map applied to the occupied MT coefficients

// matT[((k*natom + a)*nocc + n)*nrow + r] = sum_{e in row r} val[e] * c1(k, n, a, col[e]),
// r = I*maxlm + lm1. One CTA per (n, a, k); the coefficient vector sits in shared memory.
__global__ void __launch_bounds__(256) mt_expand_kernel(const double2* __restrict__ c1, int natom,
                                                        int maxlm, int nocc, int nrow,
                                                        const int* __restrict__ rp,
                                                        const int* __restrict__ ci,
                                                        const double* __restrict__ cv,
                                                        double2* __restrict__ matT) {
  extern __shared__ double2 cvec[];
  const int n = blockIdx.x, a = blockIdx.y, k = blockIdx.z;
  const double2* src = c1 + ((int64_t)(k * nocc + n) * natom + a) * maxlm;
  for (int i = threadIdx.x; i < maxlm; i += blockDim.x) cvec[i] = src[i];
  __syncthreads();
  double2* dst = matT + ((int64_t)(k * natom + a) * nocc + n) * nrow;
  for (int r = threadIdx.x; r < nrow; r += blockDim.x) {
    double sr = 0.0, si = 0.0;
    const int e1 = rp[r + 1];
    for (int e = rp[r]; e < e1; ++e) {
      const double v = cv[e];
      const double2 c = cvec[ci[e]];
      sr = fma(v, c.x, sr);
      si = fma(v, c.y, si);
    }
    dst[r] = make_double2(sr, si);
  }
}

// Host: CSR of the map T over the outputs r = I*maxlm + lm1, following the loop
// nest of src/wavefproducts.f:299-337 (running indices ln, ln1, lm, lln, llm).
struct MtMap {
  std::vector<int> rp, ci;
  std::vector<double> cv;
  int maxlm = 0, maxllm = 0;
};

static int build_mt_map(spx_ctx* ctx, const spx_mt_desc* d, MtMap* out) {
  const int lcut = d->lcut, lcutm = d->lcutm, nrad = d->nrad, nradm = d->nradm;
  if (lcut < 0 || lcutm < 0 || nrad <= 0 || nradm <= 0 || lcut > 30 || d->natom <= 0)
    return set_error(ctx, SPX_EINVAL, "bad muffin-tin descriptor");
  const int maxlm = (lcut + 1) * (lcut + 1) * nrad;
  const int maxllm = (lcutm + 1) * (lcutm + 1) * nradm;
  const int nln = (lcut + 1) * nrad;
  const int64_t nrow = (int64_t)maxlm * maxllm;
  if (nrow > 0x7fffffff) return set_error(ctx, SPX_EINVAL, "muffin-tin basis too large");
  std::vector<int> lmstart((lcut + 1) * (2 * lcut + 1), 0);
  {
    int lm = 0;
    for (int l = 0; l <= lcut; ++l)
      for (int m = -l; m <= l; ++m) {
        lmstart[l * (2 * lcut + 1) + m + lcut] = lm;
        lm += nrad;
      }
  }
  auto gaunt = [&](int l1, int l, int LL, int m, int MM) {
    const int64_t n0 = lcut + 1, n1 = lcut + 1, n2 = lcutm + 1, n3 = 2 * lcut + 1;
    return d->gaunt[l1 + n0 * (l + n1 * (LL + n2 * ((m + lcut) + n3 * (MM + lcutm))))];
  };
  struct Ent {
    int row, col;
    double v;
  };
  std::vector<Ent> ents;
  int llm = 0, lln = 0;
  for (int LL = 0; LL <= lcutm; ++LL) {
    for (int MM = -LL; MM <= LL; ++MM) {
      int lm = 0, ln = 0;
      for (int l = 0; l <= lcut; ++l) {
        for (int m = -l; m <= l; ++m) {
          const int m1 = m + MM;
          int ln1 = 0;
          const int l1lo = std::abs(l - LL), l1hi = std::min(l + LL, lcut);
          for (int l1 = l1lo; l1 <= l1hi; l1 += 2) {
            if (l1 >= std::abs(m1)) {
              const double gnt = gaunt(l1, l, LL, m, MM);
              if (gnt != 0.0) {
                const int lm1 = lmstart[l1 * (2 * lcut + 1) + m1 + lcut];
                for (int nn = 0; nn < nradm; ++nn)
                  for (int j = 0; j < nrad; ++j)
                    for (int i = 0; i < nrad; ++i) {
                      if (ln1 + j >= d->ld1) continue;
                      const double v =
                          d->integral[(ln + i) + (int64_t)nln * ((ln1 + j) + (int64_t)d->ld1 * (lln + nn))];
                      ents.push_back({(llm + nn) * maxlm + lm1 + j, lm + i, v * gnt});
                    }
              }
            }
            ln1 += nrad;
          }
          lm += nrad;
        }
        ln += nrad;
      }
      llm += nradm;
    }
    lln += nradm;
  }
  out->maxlm = maxlm;
  out->maxllm = maxllm;
  out->rp.assign(nrow + 1, 0);
  for (const Ent& e : ents) ++out->rp[e.row + 1];
  for (int64_t r = 0; r < nrow; ++r) out->rp[r + 1] += out->rp[r];
  out->ci.resize(ents.size());
  out->cv.resize(ents.size());
  std::vector<int> fill(out->rp.begin(), out->rp.end() - 1);
  for (const Ent& e : ents) {
    const int p = fill[e.row]++;
    out->ci[p] = e.col;
    out->cv[p] = e.v;
  }
  return SPX_OK;
}

// ---------------------------------------------------------------------------
// K4b: interstitial step-function convolution on a dense G box

struct GBox {
  int lo[3] = {0, 0, 0}, dim[3] = {1, 1, 1};
  __host__ __device__ int64_t size() const { return (int64_t)dim[0] * dim[1] * dim[2]; }
  int64_t lin(int x, int y, int z) const {
    return (int64_t)(x - lo[0]) + (int64_t)dim[0] * ((y - lo[1]) + (int64_t)dim[1] * (z - lo[2]));
  }
};

// grid1[(kn)*size1 + box1(G1)] = cpw1(kn, ig1); the grid is zeroed beforehand.
__global__ void pw_scatter_kernel(const double2* __restrict__ cpw, int ngpt,
                                  const int* __restrict__ gidx, int64_t size1,
                                  double2* __restrict__ grid1) {
  const int64_t kn = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ngpt; i += gridDim.x * blockDim.x)
    grid1[kn * size1 + gidx[i]] = cpw[kn * ngpt + i];
}

// grid0(kn, G0) = sum_{|d|_inf <= sr} cstep(d) * grid1(kn, G0 - d) over box0.
__global__ void __launch_bounds__(256) pw_stencil_kernel(const double2* __restrict__ grid1, GBox b1,
                                                         GBox b0, const double2* __restrict__ cstep,
                                                         int sr, double2* __restrict__ grid0) {
  __shared__ double2 st[9 * 9 * 9];
  const int ns = 2 * sr + 1, nst = ns * ns * ns;
  for (int i = threadIdx.x; i < nst; i += blockDim.x) st[i] = cstep[i];
  __syncthreads();
  const int64_t kn = blockIdx.y;
  const double2* g1 = grid1 + kn * b1.size();
  const int64_t n0 = b0.size();
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n0;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int x = b0.lo[0] + (int)(p % b0.dim[0]);
    const int y = b0.lo[1] + (int)((p / b0.dim[0]) % b0.dim[1]);
    const int z = b0.lo[2] + (int)(p / ((int64_t)b0.dim[0] * b0.dim[1]));
    double sr_ = 0.0, si = 0.0;
    for (int dz = -sr; dz <= sr; ++dz) {
      const int z1 = z - dz - b1.lo[2];
      if (z1 < 0 || z1 >= b1.dim[2]) continue;
      for (int dy = -sr; dy <= sr; ++dy) {
        const int y1 = y - dy - b1.lo[1];
        if (y1 < 0 || y1 >= b1.dim[1]) continue;
        const double2* row = g1 + (int64_t)b1.dim[0] * (y1 + (int64_t)b1.dim[1] * z1);
        const double2* srow = st + ns * ((dy + sr) + ns * (dz + sr));
        for (int dx = -sr; dx <= sr; ++dx) {
          const int x1 = x - dx - b1.lo[0];
          if (x1 < 0 || x1 >= b1.dim[0]) continue;
          const double2 c = srow[dx + sr];
          const double2 v = __ldg(row + x1);
          sr_ += c.x * v.x - c.y * v.y;
          si += c.x * v.y + c.y * v.x;
        }
      }
    }
    grid0[kn * n0 + p] = make_double2(sr_, si);
  }
}

static GBox bounding_box(const int* g, int n) {
  GBox b;
  int hi[3];
  for (int c = 0; c < 3; ++c) {
    b.lo[c] = n > 0 ? g[c] : 0;
    hi[c] = b.lo[c];
  }
  for (int i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) {
      b.lo[c] = std::min(b.lo[c], g[3 * i + c]);
      hi[c] = std::max(hi[c], g[3 * i + c]);
    }
  for (int c = 0; c < 3; ++c) b.dim[c] = hi[c] - b.lo[c] + 1;
  return b;
}

// ---------------------------------------------------------------------------
// workspace planning shared by the entry points



static size_t mt_fixed_bytes(const MtMap& mp) {
  return align_up(sizeof(int) * mp.rp.size(), 256) + align_up(sizeof(int) * std::max<size_t>(mp.ci.size(), 1), 256) +
         align_up(sizeof(double) * std::max<size_t>(mp.cv.size(), 1), 256) + 256;
}
static size_t mt_bytes_per_k(const MtMap& mp, int natom, int nocc) {
  return align_up(sizeof(double2) * (size_t)natom * nocc * mp.maxlm * mp.maxllm, 256);
}

// Runs the MT products for k points [0, nk) with the scratch [ws, ws+bytes).
int wfprod_mt_run(spx_ctx* ctx, const spx_mt_desc* d, int nk, int nocc, int nunocc,
                  const double2* c1, const double2* c2, double2* cprod, int64_t ldc, void* ws,
                  size_t ws_bytes, cudaStream_t s, int* launches) {
  MtMap mp;
  int rc = build_mt_map(ctx, d, &mp);
  if (rc) return rc;
  const size_t fixed = mt_fixed_bytes(mp), perk = mt_bytes_per_k(mp, d->natom, nocc);
  if (ws_bytes < fixed + perk) return set_error(ctx, SPX_ENOMEM, "muffin-tin scratch too small");
  // grid limits: (nocc, natom, k) for K4a, natom*k batches for K4c
  if (nocc > 65535 || d->natom > 65535) return set_error(ctx, SPX_EINVAL, "too many bands or atoms");
  const int kchunk = (int)std::min<size_t>({(size_t)nk, (ws_bytes - fixed) / perk,
                                            (size_t)(65535 / d->natom)});
  Carve cv{(char*)ws, ws_bytes};
  int* d_rp = cv.take<int>(mp.rp.size());
  int* d_ci = cv.take<int>(mp.ci.size());
  double* d_cv = cv.take<double>(mp.cv.size());
  double2* d_alpha = cv.take<double2>(d->natom);
  double2* matT = cv.take<double2>((size_t)kchunk * d->natom * nocc * mp.maxlm * mp.maxllm);
  if (!cv.ok) return set_error(ctx, SPX_ENOMEM, "muffin-tin scratch too small");
  if ((rc = check_cuda(ctx, cudaMemcpyAsync(d_rp, mp.rp.data(), sizeof(int) * mp.rp.size(), cudaMemcpyHostToDevice, s), "copy map")) ||
      (!mp.ci.empty() && (rc = check_cuda(ctx, cudaMemcpyAsync(d_ci, mp.ci.data(), sizeof(int) * mp.ci.size(), cudaMemcpyHostToDevice, s), "copy map"))) ||
      (!mp.cv.empty() && (rc = check_cuda(ctx, cudaMemcpyAsync(d_cv, mp.cv.data(), sizeof(double) * mp.cv.size(), cudaMemcpyHostToDevice, s), "copy map"))) ||
      (rc = check_cuda(ctx, cudaMemcpyAsync(d_alpha, d->cexp, sizeof(double2) * d->natom, cudaMemcpyHostToDevice, s), "copy phases")))
    return rc;
  // the host vectors die with this call: make sure the copies have left them
  if ((rc = check_cuda(ctx, cudaStreamSynchronize(s), "copy map"))) return rc;
  const int nrow = mp.maxlm * mp.maxllm;
  for (int k0 = 0; k0 < nk; k0 += kchunk) {
    const int kn = std::min(kchunk, nk - k0);
    dim3 g1(nocc, d->natom, kn);
    mt_expand_kernel<<<g1, 256, sizeof(double2) * mp.maxlm, s>>>(
        c1 + (int64_t)k0 * nocc * d->natom * mp.maxlm, d->natom, mp.maxlm, nocc, nrow, d_rp, d_ci,
        d_cv, matT);
    if ((rc = check_cuda(ctx, cudaGetLastError(), "mt_expand_kernel launch"))) return rc;
    ++*launches;
    // batches b = a + natom*k: A = cmt2(k, :, a, :), B = matT(k, a), O = cprod block (k, a)
    ZgParams prm{};
    prm.A = c2 + (int64_t)k0 * nunocc * d->natom * mp.maxlm;
    prm.lda = (int64_t)d->natom * mp.maxlm;
    prm.sA1 = mp.maxlm;
    prm.sA2 = (int64_t)nunocc * d->natom * mp.maxlm;
    prm.B = matT;
    prm.sB1 = (int64_t)nocc * nrow;
    prm.sB2 = (int64_t)d->natom * nocc * nrow;
    prm.sBn = nrow;
    prm.sBc = mp.maxlm;
    prm.cOff = nullptr;
    prm.kOff = nullptr;
    prm.O = cprod + (int64_t)k0 * nocc * nunocc;
    prm.sO1 = ldc * mp.maxllm;
    prm.sO2 = (int64_t)nocc * nunocc;
    prm.sOn = nunocc;
    prm.sOc = ldc;
    prm.alpha = d_alpha;
    prm.M = nunocc;
    prm.ncol = nocc * mp.maxllm;
    prm.ncin = mp.maxllm;
    prm.K = mp.maxlm;
    prm.nb1 = d->natom;
    if ((rc = launch_zgemm(ctx, prm, d->natom * kn, s))) return rc;
    ++*launches;
  }
  return SPX_OK;
}

size_t wfprod_mt_workspace(const spx_mt_desc* d, int nk, int nocc) {
  const int maxlm = (d->lcut + 1) * (d->lcut + 1) * d->nrad;
  const int maxllm = (d->lcutm + 1) * (d->lcutm + 1) * d->nradm;
  const size_t perk = align_up(sizeof(double2) * (size_t)d->natom * nocc * maxlm * maxllm, 256);
  // the CSR holds at most maxlm*maxllm*nrad entries per row group; bound it loosely
  const size_t nrow = (size_t)maxlm * maxllm;
  const size_t nnz_bound = nrow * (size_t)d->nrad * (d->lcut + 1);
  const size_t fixed = align_up(sizeof(int) * (nrow + 1), 256) + align_up(12 * nnz_bound, 256) + 1024;
  const size_t budget = (size_t)4 << 30;  // k points per chunk: as many as fit in 4 GiB
  const size_t kchunk = std::max<size_t>(1, std::min<size_t>((size_t)nk, budget / perk));
  return fixed + kchunk * perk;
}

struct PwPlan {
  GBox b1, b0;
  std::vector<int> gidx1, koff;
  std::vector<int64_t> coff;
  int ns = 1;
};

static int plan_pw(spx_ctx* ctx, const spx_pw_desc* d, PwPlan* pl) {
  if (d->ngpt1 < 0 || d->ngpt2 < 0 || d->ngptm < 0 || d->step_radius < 0 || d->step_radius > 4 ||
      d->vol <= 0.0)
    return set_error(ctx, SPX_EINVAL, "bad plane-wave descriptor (step_radius must be 0..4)");
  if ((d->ngpt1 > 0 && !d->gpt1) || (d->ngpt2 > 0 && !d->gpt2) || (d->ngptm > 0 && !d->gptm) || !d->cstep)
    return set_error(ctx, SPX_EINVAL, "null plane-wave descriptor array");
  pl->b1 = bounding_box(d->gpt1, d->ngpt1);
  // box of all G2 - G_M + g
  GBox b2 = bounding_box(d->gpt2, d->ngpt2), bm = bounding_box(d->gptm, d->ngptm);
  for (int c = 0; c < 3; ++c) {
    const int hi2 = b2.lo[c] + b2.dim[c] - 1, him = bm.lo[c] + bm.dim[c] - 1;
    pl->b0.lo[c] = b2.lo[c] - him + d->gshift[c];
    pl->b0.dim[c] = (hi2 - bm.lo[c] + d->gshift[c]) - pl->b0.lo[c] + 1;
  }
  if (pl->b0.size() > ((int64_t)1 << 30) || pl->b1.size() > ((int64_t)1 << 30))
    return set_error(ctx, SPX_EINVAL, "plane-wave G boxes too large");
  pl->gidx1.resize(d->ngpt1);
  for (int i = 0; i < d->ngpt1; ++i)
    pl->gidx1[i] = (int)pl->b1.lin(d->gpt1[3 * i], d->gpt1[3 * i + 1], d->gpt1[3 * i + 2]);
  // address of cpw0(G2(ig2) - GM(ig) + g) in box0 = koff[ig2] + coff[ig]
  const GBox& b0 = pl->b0;
  pl->koff.resize(d->ngpt2);
  for (int i = 0; i < d->ngpt2; ++i)
    pl->koff[i] = d->gpt2[3 * i] + b0.dim[0] * (d->gpt2[3 * i + 1] + b0.dim[1] * d->gpt2[3 * i + 2]);
  pl->coff.resize(d->ngptm);
  const int64_t base = (int64_t)b0.lo[0] + (int64_t)b0.dim[0] * (b0.lo[1] + (int64_t)b0.dim[1] * b0.lo[2]);
  for (int i = 0; i < d->ngptm; ++i) {
    const int64_t x = d->gshift[0] - d->gptm[3 * i], y = d->gshift[1] - d->gptm[3 * i + 1],
                  z = d->gshift[2] - d->gptm[3 * i + 2];
    pl->coff[i] = x + (int64_t)b0.dim[0] * (y + (int64_t)b0.dim[1] * z) - base;
  }
  pl->ns = 2 * d->step_radius + 1;
  return SPX_OK;
}

size_t wfprod_pw_fft_workspace(const spx_pw_desc* d, int nk, int nocc, int nunocc);
size_t sgemm_workspace_bytes(int nbatch, int M, int ncol, int K);
int sgemm_products(spx_ctx* ctx, int nbatch, int M, int ncol, int K, const double2* A,
                   int64_t lda, int64_t a_bstride, const double2* grid, int64_t g_bstride,
                   int64_t g_nstride, const int64_t* coff, const int* koff, int ncin,
                   double2* out, int64_t sO2, int64_t sOn, int64_t sOc, double alpha, void* ws,
                   size_t ws_bytes, cudaStream_t s, int* launches, bool overwrite);
int wfprod_pw_fft_run(spx_ctx* ctx, const spx_pw_desc* d, int nk, int nocc, int nunocc,
                      const double2* c1, const double2* c2, double2* cprod, int64_t ldc, int col0,
                      void* ws, size_t ws_bytes, cudaStream_t s, int* launches);

size_t wfprod_pw_workspace(const spx_pw_desc* d, int nk, int nocc, int nunocc, bool split) {
  if (d->nfft > 0) return wfprod_pw_fft_workspace(d, nk, nocc, nunocc);
  spx_ctx dummy;
  PwPlan pl;
  if (plan_pw(&dummy, d, &pl)) return 0;
  size_t perk = align_up(sizeof(double2) * nocc * (size_t)(pl.b1.size() + pl.b0.size()), 256);
  if (split) perk += sgemm_workspace_bytes(1, nunocc, nocc * d->ngptm, d->ngpt2);
  const size_t fixed = align_up(sizeof(int) * std::max(d->ngpt1, 1), 256) +
                       align_up(sizeof(int) * std::max(d->ngpt2, 1), 256) +
                       align_up(sizeof(int64_t) * std::max(d->ngptm, 1), 256) + 4096;
  const size_t budget = (size_t)2 << 30;
  const size_t kchunk = std::max<size_t>(1, std::min<size_t>((size_t)nk, budget / perk));
  return fixed + kchunk * perk;
}

// Runs the explicit-convolution PW products into cprod columns [col0, col0+ngptm).
// split: the product GEMM on int8 digit slices (K4s) instead of FP64 (K4c);
// overwrite: those columns hold nothing yet, so K4s stores instead of adding.
int wfprod_pw_run(spx_ctx* ctx, const spx_pw_desc* d, int nk, int nocc, int nunocc,
                  const double2* c1, const double2* c2, double2* cprod, int64_t ldc, int col0,
                  void* ws, size_t ws_bytes, cudaStream_t s, int* launches, bool split,
                  bool overwrite) {
  if (d->nfft > 0)
    return wfprod_pw_fft_run(ctx, d, nk, nocc, nunocc, c1, c2, cprod, ldc, col0, ws, ws_bytes, s,
                             launches);
  PwPlan pl;
  int rc = plan_pw(ctx, d, &pl);
  if (rc) return rc;
  if (d->ngptm == 0 || nk == 0 || nocc == 0 || nunocc == 0) return SPX_OK;
  const size_t sg_perk = split ? sgemm_workspace_bytes(1, nunocc, nocc * d->ngptm, d->ngpt2) : 0;
  const size_t perk =
      align_up(sizeof(double2) * nocc * (size_t)(pl.b1.size() + pl.b0.size()), 256) + 512 + sg_perk;
  Carve cv{(char*)ws, ws_bytes};
  int* d_gidx = cv.take<int>(d->ngpt1);
  int* d_koff = cv.take<int>(d->ngpt2);
  int64_t* d_coff = cv.take<int64_t>(d->ngptm);
  double2* d_cstep = cv.take<double2>((size_t)pl.ns * pl.ns * pl.ns);
  double2* d_alpha = cv.take<double2>(1);
  if (!cv.ok || cv.left < perk) return set_error(ctx, SPX_ENOMEM, "plane-wave scratch too small");
  if (nocc > 65535) return set_error(ctx, SPX_EINVAL, "too many occupied bands");
  // grid limit: k*nocc grids per launch of K4b
  const int kchunk = (int)std::min<size_t>({(size_t)nk, cv.left / perk, (size_t)(65535 / nocc)});
  double2* grid1 = cv.take<double2>((size_t)kchunk * nocc * pl.b1.size());
  double2* grid0 = cv.take<double2>((size_t)kchunk * nocc * pl.b0.size());
  const size_t sg_bytes = split ? sgemm_workspace_bytes(kchunk, nunocc, nocc * d->ngptm, d->ngpt2) + 1024 : 0;
  void* sg_ws = split ? (void*)cv.take<uint8_t>(sg_bytes) : nullptr;
  if (!cv.ok) return set_error(ctx, SPX_ENOMEM, "plane-wave scratch too small");
  const double2 alpha = make_double2(1.0 / std::sqrt(d->vol), 0.0);
  if ((d->ngpt1 && (rc = check_cuda(ctx, cudaMemcpyAsync(d_gidx, pl.gidx1.data(), sizeof(int) * d->ngpt1, cudaMemcpyHostToDevice, s), "copy plan"))) ||
      (d->ngpt2 && (rc = check_cuda(ctx, cudaMemcpyAsync(d_koff, pl.koff.data(), sizeof(int) * d->ngpt2, cudaMemcpyHostToDevice, s), "copy plan"))) ||
      (rc = check_cuda(ctx, cudaMemcpyAsync(d_coff, pl.coff.data(), sizeof(int64_t) * d->ngptm, cudaMemcpyHostToDevice, s), "copy plan")) ||
      (rc = check_cuda(ctx, cudaMemcpyAsync(d_cstep, d->cstep, sizeof(double2) * pl.ns * pl.ns * pl.ns, cudaMemcpyHostToDevice, s), "copy step")) ||
      (rc = check_cuda(ctx, cudaMemcpyAsync(d_alpha, &alpha, sizeof(double2), cudaMemcpyHostToDevice, s), "copy scale")))
    return rc;
  if ((rc = check_cuda(ctx, cudaStreamSynchronize(s), "copy plan"))) return rc;
  for (int k0 = 0; k0 < nk; k0 += kchunk) {
    const int kn = std::min(kchunk, nk - k0);
    const int nkn = kn * nocc;
    if ((rc = check_cuda(ctx, cudaMemsetAsync(grid1, 0, sizeof(double2) * nkn * pl.b1.size(), s), "zero grid")))
      return rc;
    if (d->ngpt1 > 0) {
      dim3 gs((d->ngpt1 + 255) / 256, nkn);
      pw_scatter_kernel<<<gs, 256, 0, s>>>(c1 + (int64_t)k0 * nocc * d->ngpt1, d->ngpt1, d_gidx,
                                           pl.b1.size(), grid1);
      if ((rc = check_cuda(ctx, cudaGetLastError(), "pw_scatter_kernel launch"))) return rc;
      ++*launches;
    }
    {
      const int64_t blocks = std::min<int64_t>((pl.b0.size() + 255) / 256, 4096);
      dim3 gs((unsigned)blocks, nkn);
      pw_stencil_kernel<<<gs, 256, 0, s>>>(grid1, pl.b1, pl.b0, d_cstep, d->step_radius, grid0);
      if ((rc = check_cuda(ctx, cudaGetLastError(), "pw_stencil_kernel launch"))) return rc;
      ++*launches;
    }
    if (d->ngpt2 == 0) continue;
    if (split) {
      rc = sgemm_products(ctx, kn, nunocc, nocc * d->ngptm, d->ngpt2,
                          c2 + (int64_t)k0 * nunocc * d->ngpt2, d->ngpt2,
                          (int64_t)nunocc * d->ngpt2, grid0, (int64_t)nocc * pl.b0.size(),
                          pl.b0.size(), d_coff, d_koff, d->ngptm,
                          cprod + (int64_t)k0 * nocc * nunocc + ldc * col0,
                          (int64_t)nocc * nunocc, nunocc, ldc, 1.0 / std::sqrt(d->vol), sg_ws,
                          sg_bytes, s, launches, overwrite);
      if (rc) return rc;
      continue;
    }
    // batches b = k: A = cpw2(k, :, :), B(col = n*ngptm + ig, ig2) = grid0(k, n)[coff[ig] + koff[ig2]]
    ZgParams prm{};
    prm.A = c2 + (int64_t)k0 * nunocc * d->ngpt2;
    prm.lda = d->ngpt2;
    prm.sA1 = 0;
    prm.sA2 = (int64_t)nunocc * d->ngpt2;
    prm.B = grid0;
    prm.sB1 = 0;
    prm.sB2 = (int64_t)nocc * pl.b0.size();
    prm.sBn = pl.b0.size();
    prm.sBc = 0;
    prm.cOff = d_coff;
    prm.kOff = d_koff;
    prm.O = cprod + (int64_t)k0 * nocc * nunocc + ldc * col0;
    prm.sO1 = 0;
    prm.sO2 = (int64_t)nocc * nunocc;
    prm.sOn = nunocc;
    prm.sOc = ldc;
    prm.alpha = d_alpha;
    prm.M = nunocc;
    prm.ncol = nocc * d->ngptm;
    prm.ncin = d->ngptm;
    prm.K = d->ngpt2;
    prm.nb1 = 1;
    if ((rc = launch_zgemm(ctx, prm, kn, s))) return rc;
    ++*launches;
  }
  return SPX_OK;
}

}  // namespace spx

using namespace spx;

static int check_band_args(spx_ctx* ctx, int nk, int nocc, int nunocc, const void* c1,
                           const void* c2, const void* cprod, int64_t ldc) {
  if (!ctx) return SPX_EINVAL;
  if (nk < 0 || nocc < 0 || nunocc < 0) return set_error(ctx, SPX_EINVAL, "negative size");
  if ((int64_t)nk * nocc * nunocc > 0) {
    if (!c1 || !c2 || !cprod) return set_error(ctx, SPX_EINVAL, "null array argument");
    if (ldc < (int64_t)nk * nocc * nunocc) return set_error(ctx, SPX_EINVAL, "ldc < nk*nocc*nunocc");
  }
  return SPX_OK;
}

extern "C" int spx_wfprod_mt_dev(spx_ctx* ctx, const spx_mt_desc* mt, int32_t nk, int32_t nocc,
                                 int32_t nunocc, const double* cmt_occ, const double* cmt_unocc,
                                 double* cprod, int64_t ldc, void* stream) {
  int rc = check_band_args(ctx, nk, nocc, nunocc, cmt_occ, cmt_unocc, cprod, ldc);
  if (rc) return rc;
  if (!mt || !mt->gaunt || !mt->integral || !mt->cexp)
    return set_error(ctx, SPX_EINVAL, "null muffin-tin descriptor array");
  if ((int64_t)nk * nocc * nunocc == 0) return SPX_OK;
  cudaSetDevice(ctx->device);
  const size_t need = wfprod_mt_workspace(mt, nk, nocc);
  if ((rc = ensure_workspace(ctx, need))) return rc;
  int launches = 0;
  cudaStream_t s = pick_stream(ctx, stream);
  return wfprod_mt_run(ctx, mt, nk, nocc, nunocc, reinterpret_cast<const double2*>(cmt_occ),
                       reinterpret_cast<const double2*>(cmt_unocc), reinterpret_cast<double2*>(cprod),
                       ldc, ctx->ws, ctx->ws_bytes, s, &launches);
}

extern "C" int spx_wfprod_pw_dev(spx_ctx* ctx, const spx_pw_desc* pw, int32_t nk, int32_t nocc,
                                 int32_t nunocc, const double* cpw_occ, const double* cpw_unocc,
                                 double* cprod, int64_t ldc, int32_t col0, void* stream) {
  int rc = check_band_args(ctx, nk, nocc, nunocc, cpw_occ, cpw_unocc, cprod, ldc);
  if (rc) return rc;
  if (!pw) return set_error(ctx, SPX_EINVAL, "null plane-wave descriptor");
  if (col0 < 0) return set_error(ctx, SPX_EINVAL, "negative col0");
  if ((int64_t)nk * nocc * nunocc == 0) return SPX_OK;
  cudaSetDevice(ctx->device);
  const bool split = ctx->opt.products == SPX_PRODUCTS_SPLIT;
  const size_t need = wfprod_pw_workspace(pw, nk, nocc, nunocc, split);
  if (need == 0) {
    // the plan is invalid: run it once more to report why
    if (pw->nfft > 0)
      return wfprod_pw_fft_run(ctx, pw, nk, nocc, nunocc, nullptr, nullptr, nullptr, ldc, col0,
                               nullptr, 0, nullptr, nullptr);
    PwPlan pl;
    return plan_pw(ctx, pw, &pl);
  }
  if ((rc = ensure_workspace(ctx, need))) return rc;
  int launches = 0;
  cudaStream_t s = pick_stream(ctx, stream);
  return wfprod_pw_run(ctx, pw, nk, nocc, nunocc, reinterpret_cast<const double2*>(cpw_occ),
                       reinterpret_cast<const double2*>(cpw_unocc), reinterpret_cast<double2*>(cprod),
                       ldc, col0, ctx->ws, ctx->ws_bytes, s, &launches, split, false);
}

// ---------------------------------------------------------------------------
// Transform to the Coulomb eigenbasis (src/susceptibility.f:806-832, FULLPW branch of
// the complex build): cprod(:, :dim) = conj(conj(cprod) ctrafo), i.e.
//   out(p, j) = sum_i cprod(p, i) conj(ctrafo(i, j)),
// which is K4c with the p-contiguous cprod panel as A and the columns of ctrafo as
// the rows of B. In place (out == cprod), rows go through a scratch panel in chunks,
// as the reference's row blocks do, so that no output overwrites an input still read.

// The transform with the in-place chunk buffer at byte offset `ws_off` of the workspace
// (anything the caller keeps in the workspace lies below it).
static int trafo_run(spx_ctx* ctx, const double* cprod, int64_t ldc, int64_t npair, int32_t nbas,
                     const double* ctrafo, int64_t ldt, int32_t dim, double* out, int64_t ldo,
                     void* stream, size_t ws_off) {
  if (!ctx) return SPX_EINVAL;
  if (npair < 0 || nbas < 0 || dim < 0) return set_error(ctx, SPX_EINVAL, "negative size");
  if (npair == 0 || dim == 0) return SPX_OK;
  if (!cprod || !out || (nbas > 0 && !ctrafo)) return set_error(ctx, SPX_EINVAL, "null array argument");
  if (ldc < npair || ldo < npair || ldt < nbas) return set_error(ctx, SPX_EINVAL, "leading dimension too small");
  if (out == cprod && ldo != ldc) return set_error(ctx, SPX_EINVAL, "in place needs ldo == ldc");
  if (out != cprod) {
    // a partial overlap of the two panels would let outputs overwrite inputs
    const char* a0 = (const char*)cprod;
    const char* a1 = a0 + 16 * (size_t)(ldc * (nbas - 1) + npair);
    const char* b0 = (const char*)out;
    const char* b1 = b0 + 16 * (size_t)(ldo * (dim - 1) + npair);
    if (nbas > 0 && a0 < b1 && b0 < a1) return set_error(ctx, SPX_EINVAL, "cprod and out overlap");
  }
  cudaSetDevice(ctx->device);
  cudaStream_t s = pick_stream(ctx, stream);
  int rc;
  ZgParams prm{};
  prm.a_mcontig = 1;
  prm.lda = ldc;
  prm.B = reinterpret_cast<const double2*>(ctrafo);
  prm.sBc = ldt;
  prm.ncin = dim;
  prm.alpha_v = make_double2(1.0, 0.0);
  prm.ncol = dim;
  prm.K = nbas;
  prm.nb1 = 1;
  if (out != cprod) {
    if ((rc = check_cuda(ctx, cudaMemset2DAsync(out, 16 * ldo, 0, 16 * npair, dim, s), "zero out")))
      return rc;
    if (nbas == 0) return SPX_OK;
    prm.A = reinterpret_cast<const double2*>(cprod);
    prm.O = reinterpret_cast<double2*>(out);
    prm.sOc = ldo;
    prm.M = (int)std::min<int64_t>(npair, 2147483647);
    if (npair > 2147483647) return set_error(ctx, SPX_EINVAL, "npair too large");
    return launch_zgemm(ctx, prm, 1, s);
  }
  // in place: row chunks through the workspace
  const int64_t chunk = std::min<int64_t>(npair, 65536);
  if ((rc = ensure_workspace(ctx, ws_off + 16 * (size_t)chunk * std::max(dim, 1) + 256))) return rc;
  double2* tmp = reinterpret_cast<double2*>((char*)ctx->ws + ws_off);
  for (int64_t r0 = 0; r0 < npair; r0 += chunk) {
    const int64_t len = std::min<int64_t>(chunk, npair - r0);
    if ((rc = check_cuda(ctx, cudaMemsetAsync(tmp, 0, 16 * (size_t)len * dim, s), "zero chunk")))
      return rc;
    if (nbas > 0) {
      prm.A = reinterpret_cast<const double2*>(cprod) + r0;
      prm.O = tmp;
      prm.sOc = len;
      prm.M = (int)len;
      if ((rc = launch_zgemm(ctx, prm, 1, s))) return rc;
    }
    if ((rc = check_cuda(ctx, cudaMemcpy2DAsync(out + 2 * r0, 16 * ldo, tmp, 16 * len, 16 * len, dim,
                                                cudaMemcpyDeviceToDevice, s), "copy chunk")))
      return rc;
  }
  return SPX_OK;
}

extern "C" int spx_trafo_dev(spx_ctx* ctx, const double* cprod, int64_t ldc, int64_t npair,
                             int32_t nbas, const double* ctrafo, int64_t ldt, int32_t dim,
                             double* out, int64_t ldo, void* stream) {
  return trafo_run(ctx, cprod, ldc, npair, nbas, ctrafo, ldt, dim, out, ldo, stream, 0);
}

// olapvec (src/overlap.f:298-316) forms out(i) = zdotc(row, vec) with
// row(j) = cstep(G_j - G_i), i.e. out = O vec with O(i, j) = conj(cstep(G_j - G_i)).
// This kernel writes conj(O)(i, j) = cstep(G_j - G_i) for the MPB plane waves
// (0 outside the box of cstep), column-major (ngptm, ngptm).
__global__ void olap_conj_kernel(const int* __restrict__ gptm, int ngptm, const double2* __restrict__ cstep,
                                 int sr, double2* __restrict__ O) {
  const int ns = 2 * sr + 1;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < (int64_t)ngptm * ngptm;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % ngptm), j = (int)(t / ngptm);
    const int d0 = gptm[3 * j] - gptm[3 * i], d1 = gptm[3 * j + 1] - gptm[3 * i + 1],
              d2 = gptm[3 * j + 2] - gptm[3 * i + 2];
    double2 v = make_double2(0.0, 0.0);
    if (abs(d0) <= sr && abs(d1) <= sr && abs(d2) <= sr)
      v = cstep[(d0 + sr) + ns * ((d1 + sr) + ns * (d2 + sr))];
    O[t] = v;
  }
}

// In place: z = conj(z) for rows [0, rows) of `cols` columns (leading dimension ld).
__global__ void conj_rows_kernel(double2* z, int64_t ld, int rows, int cols) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < (int64_t)rows * cols;
       t += (int64_t)gridDim.x * blockDim.x) {
    double2* p = z + (t / rows) * ld + t % rows;
    p->y = -p->y;
  }
}

extern "C" int spx_trafo_olap_dev(spx_ctx* ctx, const double* cprod, int64_t ldc, int64_t npair,
                                  int32_t nbas, int32_t nbasp, const double* ctrafo, int64_t ldt,
                                  int32_t dim, const spx_pw_desc* pw, double* out, int64_t ldo,
                                  void* stream) {
  if (!ctx) return SPX_EINVAL;
  if (!pw || nbasp < 0 || nbasp + pw->ngptm != nbas || pw->step_radius < 0 || pw->step_radius > 4 ||
      (pw->ngptm > 0 && (!pw->gptm || !pw->cstep)))
    return set_error(ctx, SPX_EINVAL, "bad plane-wave descriptor (nbas must be nbasp + ngptm)");
  if (npair < 0 || nbas < 0 || dim < 0) return set_error(ctx, SPX_EINVAL, "negative size");
  if (npair == 0 || dim == 0) return SPX_OK;
  if (!ctrafo || ldt < nbas) return set_error(ctx, SPX_EINVAL, "ctrafo NULL or ldt < nbas");
  cudaSetDevice(ctx->device);
  cudaStream_t s = pick_stream(ctx, stream);
  const int ng = pw->ngptm, sr = pw->step_radius, ns = 2 * sr + 1;
  // workspace: ctrafo1 (nbas, dim), conj(O) (ng, ng), the G list and cstep
  const size_t t1_b = align_up(16 * (size_t)nbas * dim, 256);
  const size_t o_b = align_up(16 * (size_t)ng * ng, 256);
  const size_t g_b = align_up(sizeof(int) * 3 * (size_t)std::max(ng, 1), 256);
  const size_t c_b = align_up(16 * (size_t)ns * ns * ns, 256);
  const size_t keep = t1_b + o_b + g_b + c_b;
  int rc = ensure_workspace(ctx, keep + 256);
  if (rc) return rc;
  char* w = (char*)ctx->ws;
  double2* T1 = (double2*)w;
  double2* O = (double2*)(w + t1_b);
  int* G = (int*)(w + t1_b + o_b);
  double2* CS = (double2*)(w + t1_b + o_b + g_b);
  // ctrafo1(:nbasp) = ctrafo(:nbasp); ctrafo1(nbasp:) = O ctrafo(nbasp:) (olapvec per column)
  if ((rc = check_cuda(ctx, cudaMemcpy2DAsync(T1, 16 * (size_t)nbas, ctrafo, 16 * (size_t)ldt,
                                              16 * (size_t)nbasp, dim, cudaMemcpyDeviceToDevice, s),
                       "copy MT rows")))
    return rc;
  if (ng > 0) {
    if ((rc = check_cuda(ctx, cudaMemcpyAsync(G, pw->gptm, sizeof(int) * 3 * ng, cudaMemcpyHostToDevice, s),
                         "copy G list")) ||
        (rc = check_cuda(ctx, cudaMemcpyAsync(CS, pw->cstep, 16 * (size_t)ns * ns * ns, cudaMemcpyHostToDevice, s),
                         "copy step function")) ||
        0)
      return rc;
    if ((rc = check_cuda(ctx, cudaMemset2DAsync(T1 + nbasp, 16 * (size_t)nbas, 0, 16 * (size_t)ng, dim, s),
                         "zero PW rows")))
      return rc;
    olap_conj_kernel<<<std::min<int64_t>(((int64_t)ng * ng + 255) / 256, (int64_t)ctx->num_sms * 16), 256, 0, s>>>(
        G, ng, CS, sr, O);
    if ((rc = check_cuda(ctx, cudaGetLastError(), "olap_conj_kernel launch"))) return rc;
    // conj(ctrafo1_pw)(i, c) = sum_j conj(O(i, j)) conj(ctrafo(nbasp + j, c))
    ZgParams prm{};
    prm.A = O;
    prm.a_mcontig = 1;
    prm.lda = ng;
    prm.B = reinterpret_cast<const double2*>(ctrafo) + nbasp;
    prm.sBc = ldt;
    prm.ncin = dim;
    prm.O = T1 + nbasp;
    prm.sOc = nbas;
    prm.alpha_v = make_double2(1.0, 0.0);
    prm.M = ng;
    prm.ncol = dim;
    prm.K = ng;
    prm.nb1 = 1;
    if ((rc = launch_zgemm(ctx, prm, 1, s))) return rc;
    conj_rows_kernel<<<std::min<int64_t>(((int64_t)ng * dim + 255) / 256, (int64_t)ctx->num_sms * 16), 256, 0, s>>>(
        T1 + nbasp, nbas, ng, dim);
    if ((rc = check_cuda(ctx, cudaGetLastError(), "conj_rows_kernel launch"))) return rc;
  }
  return trafo_run(ctx, cprod, ldc, npair, nbas, reinterpret_cast<const double*>(T1), nbas, dim, out,
                   ldo, stream, keep);
}

// ---------------------------------------------------------------------------
// q -> 0 head and wings (src/susceptibility.f:1092-1157, HILBERT NONE), FP64:
//   head(ij(k1,k2), f) += sum_p dcprod(p,k1) conj(dcprod(p,k2)) w(p,f),  k1 <= k2,
//   wing(k2, i, f)     += sum_p cprod(p,i)  conj(dcprod(p,k2)) w(p,f).
// Both are the rows k < 3 of the weighted Gram of X = [dcprod | cprod]: with the
// 3 nw rows D(a,f; p) = dcprod(p,a) w(p,f) it is one complex GEMM D conj(X)^T with a
// long K = P, run as K4c over K chunks into per-chunk partials that a second kernel
// sums in a fixed order and scatters into head and wing.

constexpr int HW_KC = 16384;   // pairs per K chunk

__global__ void hw_rows_kernel(const double2* __restrict__ dc, int64_t ldd, const double* __restrict__ w,
                               int64_t ldw, int64_t p0, int64_t len, int nw, double2* __restrict__ D,
                               int64_t ldD) {
  const int64_t total = (int64_t)3 * nw * len;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = t % len;
    const int m = (int)(t / len), a = m / nw, f = m - a * nw;
    const double2 v = dc[a * ldd + p0 + p];
    const double ww = w[f * ldw + p0 + p];
    D[m * ldD + p] = make_double2(v.x * ww, v.y * ww);
  }
}

// out(m, col) = sum over chunks of part[c][m + M*col]; then scatter
__global__ void hw_reduce_kernel(const double2* __restrict__ part, int nchunk, int nw, int ncol,
                                 int dim, double2* __restrict__ head, double2* __restrict__ wing) {
  const int M = 3 * nw;
  const int64_t total = (int64_t)M * ncol;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    double sx = 0.0, sy = 0.0;
    for (int c = 0; c < nchunk; ++c) {
      const double2 v = part[(int64_t)c * total + t];
      sx += v.x;
      sy += v.y;
    }
    const int m = (int)(t % M), col = (int)(t / M);
    const int a = m / nw, f = m - a * nw;
    if (col < 3) {
      if (a <= col) {
        double2* o = head + (col * (col + 1) / 2 + a) + 6 * (int64_t)f;
        o->x += sx;
        o->y += sy;
      }
    } else {
      const int i = col - 3;
      double2* o = wing + a + 3 * ((int64_t)i + (int64_t)dim * f);
      o->x += sx;
      o->y -= sy;   // wing = conj of the Gram's (k2, 3 + i) element
    }
  }
}

extern "C" int spx_headwings_dev(spx_ctx* ctx, const double* cprod, int64_t ldc, int64_t npair,
                                 int32_t dim, const double* dcprod, int64_t ldd, const double* w,
                                 int64_t ldw, int32_t nw, double* head, double* wing, void* stream) {
  if (!ctx) return SPX_EINVAL;
  if (npair < 0 || dim < 0 || nw < 0) return set_error(ctx, SPX_EINVAL, "negative size");
  if (npair == 0 || nw == 0) return SPX_OK;
  if (!dcprod || !w || !head || (dim > 0 && (!cprod || !wing)))
    return set_error(ctx, SPX_EINVAL, "null array argument");
  if (ldd < npair || ldw < npair || (dim > 0 && ldc < npair))
    return set_error(ctx, SPX_EINVAL, "leading dimension too small");
  if (nw > 1024) return set_error(ctx, SPX_EINVAL, "nw > 1024");
  cudaSetDevice(ctx->device);
  cudaStream_t s = pick_stream(ctx, stream);
  const int M = 3 * nw, ncol = 3 + dim;
  // pair ranges of at most 64 chunks per pass: D (M x range) and the chunk partials
  const int64_t range = std::min<int64_t>(npair, (int64_t)64 * HW_KC);
  const int64_t ldD = (int64_t)align_up((size_t)range, 2);
  const int maxchunk = (int)((range + HW_KC - 1) / HW_KC);
  const size_t d_bytes = align_up(sizeof(double2) * (size_t)M * ldD, 256);
  const size_t p_bytes = align_up(sizeof(double2) * (size_t)maxchunk * M * ncol, 256);
  int rc;
  if ((rc = ensure_workspace(ctx, d_bytes + p_bytes + 256))) return rc;
  double2* D = reinterpret_cast<double2*>(ctx->ws);
  double2* part = reinterpret_cast<double2*>((char*)ctx->ws + d_bytes);
  const double2* dc = reinterpret_cast<const double2*>(dcprod);
  const double2* cp = reinterpret_cast<const double2*>(cprod);
  for (int64_t p0 = 0; p0 < npair; p0 += range) {
    const int64_t len = std::min<int64_t>(range, npair - p0);
    const int nchunk = (int)((len + HW_KC - 1) / HW_KC);
    const int64_t tot = (int64_t)M * len;
    hw_rows_kernel<<<(unsigned)std::min<int64_t>((tot + 255) / 256, (int64_t)ctx->num_sms * 16), 256, 0, s>>>(
        dc, ldd, w, ldw, p0, len, nw, D, ldD);
    if ((rc = check_cuda(ctx, cudaGetLastError(), "hw_rows_kernel launch"))) return rc;
    if ((rc = check_cuda(ctx, cudaMemsetAsync(part, 0, sizeof(double2) * (size_t)nchunk * M * ncol, s),
                         "zero partials")))
      return rc;
    // chunk b2 of the K4c launch: A = D[:, b2 KC ...], B rows = columns of [dcprod | cprod]
    // (the two panels differ in leading dimension: one launch each)
    for (int panel = 0; panel < 2; ++panel) {
      const int pcols = panel == 0 ? 3 : dim;
      if (pcols == 0) continue;
      ZgParams prm{};
      prm.A = D;
      prm.lda = ldD;
      prm.sA2 = HW_KC;
      prm.B = panel == 0 ? dc + p0 : cp + p0;
      prm.sBc = panel == 0 ? ldd : ldc;
      prm.sB2 = HW_KC;
      prm.ncin = pcols;
      prm.O = part + (panel == 0 ? 0 : (int64_t)M * 3);
      prm.sOc = M;
      prm.sO2 = (int64_t)M * ncol;
      prm.alpha_v = make_double2(1.0, 0.0);
      prm.M = M;
      prm.ncol = pcols;
      prm.K = (int)std::min<int64_t>(HW_KC, len);
      prm.K_last = (int)(len - (int64_t)(nchunk - 1) * HW_KC);
      prm.nb1 = 1;
      if ((rc = launch_zgemm(ctx, prm, nchunk, s))) return rc;
    }
    const int64_t tot2 = (int64_t)M * ncol;
    hw_reduce_kernel<<<(unsigned)std::min<int64_t>((tot2 + 255) / 256, (int64_t)ctx->num_sms * 8), 256, 0, s>>>(
        part, nchunk, nw, ncol, dim, reinterpret_cast<double2*>(head), reinterpret_cast<double2*>(wing));
    if ((rc = check_cuda(ctx, cudaGetLastError(), "hw_reduce_kernel launch"))) return rc;
  }
  return SPX_OK;
}

// ---------------------------------------------------------------------------
// q -> 0 momentum matrix: momentum_matrix (src/dwavefproducts.f:89-330, the non-SOC
// branch without storeibz) and the dcprod scaling of src/susceptibility.f:848-870.
//
// MT part: per atom and occupied band, the reference builds cvec1/2/3 from cmt1 with
// the F / G coefficients (:135-146) times the radial integrals qmat2 (l -> l+1,
// :215-219) and qmat1 (l -> l-1, :233-238); cvec(x) = zdotc(cvec_x, cmt2) / i and
//   momentum(1) += (cvec(1) - cvec(3)) / sqrt 2,  momentum(2) -= (cvec(1) + cvec(3)) i / sqrt 2,
//   momentum(3) += cvec(2).
// Here the linear map cmt1 -> v_x with v_1 = (cvec1 - cvec3)/sqrt 2, v_2 = i (cvec1 +
// cvec3)/sqrt 2, v_3 = cvec2 is a complex sparse matrix (CSR, built on the host from
// the same index nest), applied per (k, atom, band), and
//   momentum(n', n, k, x) += -i sum_idx cmt2(n', idx) conj(v_x(n, idx))
// is a batched complex DMMA GEMM (K4c), one launch per atom.
// PW part (:269-283): vec1 = olapvec(cpw(:, n)) = O cpw_n with O(i, j) =
// conj(cstep(G_j - G_i)), and momentum(n', n, k, x) += sum_G conj(vec1(G)) cpw(G, n')
// qg(G, x), qg = rlat (k + G): two K4c GEMMs (conj(O) conj(cpw) gives conj(vec1), then
// cpw_unocc against vec1 qg).

struct MomMap {
  int maxlm;
  std::vector<int> rp, ci;
  std::vector<double2> cv;
};

static int build_mom_map(spx_ctx* ctx, const spx_mom_desc* d, MomMap* mp) {
  const int L = d->lcut, nr = d->nrad;
  if (L < 0 || L > 16 || nr <= 0 || nr > 16 || !d->qmat1 || !d->qmat2)
    return set_error(ctx, SPX_EINVAL, "bad momentum descriptor (lcut 0..16, nrad 1..16, qmat1/2)");
  const int maxlm = (L + 1) * (L + 1) * nr;
  mp->maxlm = maxlm;
  auto off = [&](int l) { return l * l * nr; };           // first index of block l
  auto q1 = [&](int n1, int n2, int l) { return d->qmat1[n1 + nr * (n2 + nr * l)]; };
  auto q2 = [&](int n1, int n2, int l) { return d->qmat2[n1 + nr * (n2 + nr * l)]; };
  // c[x][out] : list of (in, real coefficient) for cvec_{x+1}
  std::vector<std::vector<std::pair<int, double>>> c(3 * maxlm);
  for (int l = 0; l <= L; ++l)
    for (int m = -l; m <= l; ++m) {
      const double fl = (double)l, fm = (double)m;
      const double f[3] = {-std::sqrt((fl + fm + 1) * (fl + fm + 2) / (2 * (2 * fl + 1) * (2 * fl + 3))),
                           std::sqrt((fl - fm + 1) * (fl + fm + 1) / ((2 * fl + 1) * (2 * fl + 3))),
                           -std::sqrt((fl - fm + 1) * (fl - fm + 2) / (2 * (2 * fl + 1) * (2 * fl + 3)))};
      const double g[3] = {std::sqrt((fl - fm) * (fl - fm - 1) / (2 * (2 * fl - 1) * (2 * fl + 1))),
                           std::sqrt((fl - fm) * (fl + fm) / ((2 * fl - 1) * (2 * fl + 1))),
                           std::sqrt((fl + fm) * (fl + fm - 1) / (2 * (2 * fl - 1) * (2 * fl + 1)))};
      const int out = off(l) + (m + l) * nr;
      for (int x = 0; x < 3; ++x) {
        const int mp_ = m + 1 - x;                         // m+1, m, m-1 for cvec1, 2, 3
        if (l < L) {                                       // from l+1 (:211-219)
          const int src = off(l + 1) + (mp_ + l + 1) * nr;
          for (int n2 = 0; n2 < nr; ++n2)
            for (int n1 = 0; n1 < nr; ++n1)
              c[x * maxlm + out + n2].push_back({src + n1, f[x] * q2(n1, n2, l)});
        }
        if (l >= 1 && std::abs(mp_) <= l - 1) {            // from l-1 (:222-238)
          const int src = off(l - 1) + (mp_ + l - 1) * nr;
          for (int n2 = 0; n2 < nr; ++n2)
            for (int n1 = 0; n1 < nr; ++n1)
              c[x * maxlm + out + n2].push_back({src + n1, g[x] * q1(n1, n2, l)});
        }
      }
    }
  // v_1 = (c1 - c3)/sqrt2, v_2 = i (c1 + c3)/sqrt2, v_3 = c2
  const double r2 = 1.0 / std::sqrt(2.0);
  mp->rp.assign(1, 0);
  for (int x = 0; x < 3; ++x)
    for (int o = 0; o < maxlm; ++o) {
      std::vector<double2> row(maxlm, make_double2(0.0, 0.0));
      std::vector<char> used(maxlm, 0);
      auto add = [&](const std::vector<std::pair<int, double>>& v, double2 s) {
        for (auto& e : v) {
          row[e.first].x += s.x * e.second;
          row[e.first].y += s.y * e.second;
          used[e.first] = 1;
        }
      };
      if (x == 0) {
        add(c[0 * maxlm + o], make_double2(r2, 0.0));
        add(c[2 * maxlm + o], make_double2(-r2, 0.0));
      } else if (x == 1) {
        add(c[0 * maxlm + o], make_double2(0.0, r2));
        add(c[2 * maxlm + o], make_double2(0.0, r2));
      } else {
        add(c[1 * maxlm + o], make_double2(1.0, 0.0));
      }
      for (int i = 0; i < maxlm; ++i)
        if (used[i]) {
          mp->ci.push_back(i);
          mp->cv.push_back(row[i]);
        }
      mp->rp.push_back((int)mp->ci.size());
    }
  return SPX_OK;
}

// v[k][n][atom][x][idx] = sum_in T(x*maxlm + idx, in) cmt1[k][n][atom][in], one CTA per
// (band, atom, k); the band's coefficients are staged in shared memory.
__global__ void __launch_bounds__(256) mom_expand_kernel(const double2* __restrict__ c1, int natom,
                                                         int maxlm, int nocc, const int* __restrict__ rp,
                                                         const int* __restrict__ ci,
                                                         const double2* __restrict__ cv,
                                                         double2* __restrict__ v) {
  extern __shared__ double2 cm[];
  const int n = blockIdx.x, a = blockIdx.y, k = blockIdx.z;
  const double2* src = c1 + (((int64_t)k * nocc + n) * natom + a) * maxlm;
  for (int i = threadIdx.x; i < maxlm; i += blockDim.x) cm[i] = src[i];
  __syncthreads();
  double2* dst = v + (((int64_t)k * nocc + n) * natom + a) * 3 * maxlm;
  for (int r = threadIdx.x; r < 3 * maxlm; r += blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int e = rp[r]; e < rp[r + 1]; ++e) {
      const double2 t = cv[e], x = cm[ci[e]];
      re += t.x * x.x - t.y * x.y;
      im += t.x * x.y + t.y * x.x;
    }
    dst[r] = make_double2(re, im);
  }
}

struct Mat3 {
  double r[9];  // column-major 3 x 3
};

// Bq[((k n) 3 + x) ngpt + G] = conj(R(G, k n)) qg_k(G, x), qg = rlat (k + G) with
// kc[3k + x] = (rlat k)_x.
__global__ void mom_pw_rhs_kernel(const double2* __restrict__ R, int ngpt, int nkn, int nocc,
                                  const int* __restrict__ gpt, const double* __restrict__ kc, Mat3 rl,
                                  double2* __restrict__ Bq) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < (int64_t)ngpt * nkn;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int G = (int)(t % ngpt), kn = (int)(t / ngpt), k = kn / nocc;
    const double2 r = R[(int64_t)kn * ngpt + G];
    const double g0 = gpt[3 * G], g1 = gpt[3 * G + 1], g2 = gpt[3 * G + 2];
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      const double q = kc[3 * k + x] + rl.r[x] * g0 + rl.r[x + 3] * g1 + rl.r[x + 6] * g2;
      Bq[((int64_t)kn * 3 + x) * ngpt + G] = make_double2(r.x * q, -r.y * q);
    }
  }
}

// dcprod(p, x) /= sqrt(vol) e(p), and 0 where |e(p)| <= 1e-8 (src/susceptibility.f:858-869);
// only the volume factor when e is NULL.
__global__ void mom_scale_kernel(double2* __restrict__ dc, int64_t ldd, int64_t npair,
                                 const double* __restrict__ e, double rsv) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < 3 * npair;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = t % npair;
    const int x = (int)(t / npair);
    double f = rsv;
    if (e) {
      const double r = e[p];
      f = fabs(r) > 1e-8 ? rsv / r : 0.0;
    }
    double2* z = dc + x * ldd + p;
    z->x *= f;
    z->y *= f;
  }
}

extern "C" int spx_dcprod_dev(spx_ctx* ctx, const spx_mom_desc* d, int32_t nk, int32_t nocc,
                              int32_t nunocc, const double* cmt_occ, const double* cmt_unocc,
                              const double* cpw_occ, const double* cpw_unocc, const double* ediff,
                              double* dcprod, int64_t ldd, void* stream) {
  if (!ctx) return SPX_EINVAL;
  if (!d || nk < 0 || nocc < 0 || nunocc < 0) return set_error(ctx, SPX_EINVAL, "bad arguments");
  const int64_t npair = (int64_t)nk * nocc * nunocc;
  if (npair == 0) return SPX_OK;
  if (!dcprod || ldd < npair) return set_error(ctx, SPX_EINVAL, "dcprod NULL or ldd < nk*nocc*nunocc");
  if (d->natom > 0 && (!cmt_occ || !cmt_unocc)) return set_error(ctx, SPX_EINVAL, "MT coefficients missing");
  if (d->ngpt > 0 && (!cpw_occ || !cpw_unocc || !d->gpt || !d->kpt || !d->rlat || !d->cstep ||
                      d->step_radius < 0 || d->step_radius > 4))
    return set_error(ctx, SPX_EINVAL, "plane-wave part of the momentum descriptor incomplete");
  if (!(d->vol > 0)) return set_error(ctx, SPX_EINVAL, "vol must be positive");
  if (nocc > 65535 || d->natom > 65535 || nk > 65535) return set_error(ctx, SPX_EINVAL, "too many bands");
  cudaSetDevice(ctx->device);
  cudaStream_t s = pick_stream(ctx, stream);
  int rc;
  MomMap mp{};
  if (d->natom > 0 && (rc = build_mom_map(ctx, d, &mp))) return rc;
  const int ng = d->ngpt, sr = d->step_radius, ns = 2 * sr + 1;
  const int64_t nkn = (int64_t)nk * nocc;
  size_t need = 0;
  auto add = [&](size_t b) { need += align_up(b, 256); };
  if (d->natom > 0) {
    add(sizeof(int) * mp.rp.size());
    add(sizeof(int) * std::max<size_t>(mp.ci.size(), 1));
    add(sizeof(double2) * std::max<size_t>(mp.cv.size(), 1));
    add(sizeof(double2) * (size_t)nkn * d->natom * 3 * mp.maxlm);
  }
  if (ng > 0) {
    add(sizeof(double2) * (size_t)ng * ng);
    add(sizeof(double2) * (size_t)ng * nkn);
    add(sizeof(double2) * (size_t)ng * nkn * 3);
    add(sizeof(int) * 3 * (size_t)ng);
    add(sizeof(double2) * (size_t)ns * ns * ns);
    add(sizeof(double) * 3 * (size_t)nk);
  }
  if ((rc = ensure_workspace(ctx, need + 4096))) return rc;
  Carve cv{(char*)ctx->ws, ctx->ws_bytes};
  if ((rc = check_cuda(ctx, cudaMemset2DAsync(dcprod, 16 * ldd, 0, 16 * npair, 3, s), "zero dcprod"))) return rc;
  double2* out = reinterpret_cast<double2*>(dcprod);
  if (ng > 0) {
    double2* O = cv.take<double2>((size_t)ng * ng);
    double2* R = cv.take<double2>((size_t)ng * nkn);
    double2* Bq = cv.take<double2>((size_t)ng * nkn * 3);
    int* G = cv.take<int>(3 * (size_t)ng);
    double2* CS = cv.take<double2>((size_t)ns * ns * ns);
    double* kc = cv.take<double>(3 * (size_t)nk);
    if (!cv.ok) return set_error(ctx, SPX_ENOMEM, "momentum scratch");
    std::vector<double> kch(3 * (size_t)nk);
    for (int k = 0; k < nk; ++k)
      for (int x = 0; x < 3; ++x)
        kch[3 * k + x] = d->rlat[x] * d->kpt[3 * k] + d->rlat[x + 3] * d->kpt[3 * k + 1] +
                         d->rlat[x + 6] * d->kpt[3 * k + 2];
    if ((rc = check_cuda(ctx, cudaMemcpyAsync(G, d->gpt, sizeof(int) * 3 * ng, cudaMemcpyHostToDevice, s), "copy G")) ||
        (rc = check_cuda(ctx, cudaMemcpyAsync(CS, d->cstep, 16 * (size_t)ns * ns * ns, cudaMemcpyHostToDevice, s), "copy cstep")) ||
        (rc = check_cuda(ctx, cudaMemcpyAsync(kc, kch.data(), sizeof(double) * 3 * nk, cudaMemcpyHostToDevice, s), "copy k")) ||
        (rc = check_cuda(ctx, cudaStreamSynchronize(s), "copy k")) ||
        (rc = check_cuda(ctx, cudaMemsetAsync(R, 0, sizeof(double2) * (size_t)ng * nkn, s), "zero R")))
      return rc;
    olap_conj_kernel<<<std::min<int64_t>(((int64_t)ng * ng + 255) / 256, (int64_t)ctx->num_sms * 16), 256, 0, s>>>(
        G, ng, CS, sr, O);
    if ((rc = check_cuda(ctx, cudaGetLastError(), "olap_conj_kernel launch"))) return rc;
    // R(i, kn) = conj(vec1_kn(i)) = sum_j conj(O)(i, j) conj(cpw_occ(kn, j))
    ZgParams p1{};
    p1.A = O;
    p1.a_mcontig = 1;
    p1.lda = ng;
    p1.B = reinterpret_cast<const double2*>(cpw_occ);
    p1.sBc = ng;
    p1.ncin = (int)nkn;
    p1.O = R;
    p1.sOc = ng;
    p1.alpha_v = make_double2(1.0, 0.0);
    p1.M = ng;
    p1.ncol = (int)nkn;
    p1.K = ng;
    p1.nb1 = 1;
    if ((rc = launch_zgemm(ctx, p1, 1, s))) return rc;
    Mat3 rl;
    for (int i = 0; i < 9; ++i) rl.r[i] = d->rlat[i];
    mom_pw_rhs_kernel<<<std::min<int64_t>(((int64_t)ng * nkn + 255) / 256, (int64_t)ctx->num_sms * 16), 256, 0, s>>>(
        R, ng, (int)nkn, nocc, G, kc, rl, Bq);
    if ((rc = check_cuda(ctx, cudaGetLastError(), "mom_pw_rhs_kernel launch"))) return rc;
    // momentum(n', n, k, x) += sum_G cpw_unocc(k, n', G) conj(Bq(k, n, x, G))
    ZgParams p2{};
    p2.A = reinterpret_cast<const double2*>(cpw_unocc);
    p2.lda = ng;
    p2.sA1 = (int64_t)nunocc * ng;
    p2.B = Bq;
    p2.sB1 = (int64_t)nocc * 3 * ng;
    p2.sBn = 3 * (int64_t)ng;
    p2.sBc = ng;
    p2.ncin = 3;
    p2.O = out;
    p2.sO1 = (int64_t)nocc * nunocc;
    p2.sOn = nunocc;
    p2.sOc = ldd;
    p2.alpha_v = make_double2(1.0, 0.0);
    p2.M = nunocc;
    p2.ncol = 3 * nocc;
    p2.K = ng;
    p2.nb1 = nk;
    if ((rc = launch_zgemm(ctx, p2, nk, s))) return rc;
  }
  if (d->natom > 0) {
    int* d_rp = cv.take<int>(mp.rp.size());
    int* d_ci = cv.take<int>(std::max<size_t>(mp.ci.size(), 1));
    double2* d_cv = cv.take<double2>(std::max<size_t>(mp.cv.size(), 1));
    double2* V = cv.take<double2>((size_t)nkn * d->natom * 3 * mp.maxlm);
    if (!cv.ok) return set_error(ctx, SPX_ENOMEM, "momentum scratch");
    if ((rc = check_cuda(ctx, cudaMemcpyAsync(d_rp, mp.rp.data(), sizeof(int) * mp.rp.size(), cudaMemcpyHostToDevice, s), "copy map")) ||
        (!mp.ci.empty() && (rc = check_cuda(ctx, cudaMemcpyAsync(d_ci, mp.ci.data(), sizeof(int) * mp.ci.size(), cudaMemcpyHostToDevice, s), "copy map"))) ||
        (!mp.cv.empty() && (rc = check_cuda(ctx, cudaMemcpyAsync(d_cv, mp.cv.data(), sizeof(double2) * mp.cv.size(), cudaMemcpyHostToDevice, s), "copy map"))) ||
        (rc = check_cuda(ctx, cudaStreamSynchronize(s), "copy map")))
      return rc;
    mom_expand_kernel<<<dim3(nocc, d->natom, nk), 256, sizeof(double2) * mp.maxlm, s>>>(
        reinterpret_cast<const double2*>(cmt_occ), d->natom, mp.maxlm, nocc, d_rp, d_ci, d_cv, V);
    if ((rc = check_cuda(ctx, cudaGetLastError(), "mom_expand_kernel launch"))) return rc;
    // one launch per atom (the atoms add into the same outputs)
    for (int a = 0; a < d->natom; ++a) {
      ZgParams p3{};
      p3.A = reinterpret_cast<const double2*>(cmt_unocc) + (int64_t)a * mp.maxlm;
      p3.lda = (int64_t)d->natom * mp.maxlm;
      p3.sA1 = (int64_t)nunocc * d->natom * mp.maxlm;
      p3.B = V + (int64_t)a * 3 * mp.maxlm;
      p3.sB1 = (int64_t)nocc * d->natom * 3 * mp.maxlm;
      p3.sBn = (int64_t)d->natom * 3 * mp.maxlm;
      p3.sBc = mp.maxlm;
      p3.ncin = 3;
      p3.O = out;
      p3.sO1 = (int64_t)nocc * nunocc;
      p3.sOn = nunocc;
      p3.sOc = ldd;
      p3.alpha_v = make_double2(0.0, -1.0);   // 1 / i
      p3.M = nunocc;
      p3.ncol = 3 * nocc;
      p3.K = mp.maxlm;
      p3.nb1 = nk;
      if ((rc = launch_zgemm(ctx, p3, nk, s))) return rc;
    }
  }
  mom_scale_kernel<<<std::min<int64_t>((3 * npair + 255) / 256, (int64_t)ctx->num_sms * 16), 256, 0, s>>>(
      out, ldd, npair, ediff, 1.0 / std::sqrt(d->vol));
  return check_cuda(ctx, cudaGetLastError(), "mom_scale_kernel launch");
}
