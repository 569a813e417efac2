// K7: the split-precision polarisation of many q points as ONE persistent launch.
//
// The reference computes one q point per call of `susceptibility`
// (src/correlation.f:293-339), each q with its own mixed basis and band window and
// its pairs split into packets (src/susceptibility.f:632-642). Here the whole batch
// is one kernel: one CTA per SM, each CTA running two independent workers over
// two device work queues.
//
//   * The accumulation pipeline (warp 0 TMA, warp 1 tcgen05 MMA, warps 2-5
//     epilogue) takes items (slab k, tile, frequency) from the accumulation queue:
//     the same 6-product int8 accumulation of the folded digit planes as the
//     one-call kernel, 64 complex rows x BN complex columns per item.
//   * Six preparation warps take items from the preparation queue: for slab k
//     (a) generate M (or read the caller's) and take the column maxima, (b) the
//     HILBERT NONE weights of one frequency, their maximum, sign and folded
//     factors, (c) the digit planes of 8 columns.
//
// Slabs are ordered q by q, the q with most work first, and live in a ring of
// NSLOT operand buffers. Dependencies are counters in device memory, each waited
// on with a bounded spin: an accumulation item waits until its slab's planes are
// ready; a preparation item waits until the slab that last used its buffer has
// been fully accumulated, and a quantizer item until its slab's maxima and
// factors exist. Every wait is on items already handed to a running CTA (a queue
// hands items out only to CTAs that run), so the schedule cannot deadlock, whether
// or not all CTAs are resident. The epilogue of slab s of a q adds into an output
// tile only after slab s-1 has added into it (a per-(q, tile, frequency) counter),
// so the sums happen in the same order as per-q calls and give the same bits.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "spx_philox.h"
#include "spx_split.cuh"

namespace spx {

constexpr int PB_EPI = 4;         // epilogue warps (one per TMEM lane quarter)
constexpr int PB_THREADS = 384;   // warps 0-5 accumulation, 6-11 preparation
constexpr int PB_PREP0 = 192;     // first preparation thread
constexpr int PB_NPREP = 192;
constexpr int PB_RING = 4;        // item descriptors in flight between the pipeline roles
constexpr int PB_ACOLS = 6;       // columns per (a) item: one per preparation warp
constexpr int PB_QCOLS = 8;       // columns per (c) item

struct PbQ {            // one q point
  int N, nblk, ntile, npad, S, nslab;
  int64_t P, npack, R;
  const double2* M;     // caller's cprod (ldc) or NULL: generated
  int64_t ldc;
  uint64_t seed;
  uint32_t sid;
  double mscale;
  const double* ediff;
  const double* wscale;
  double scale_all;
  double* out;
  int* seq;             // ntile * nw ordering counters
};

struct PbSlab {         // one slab of one q, in queue order
  int q, s, slot;
  int len, lenp, nk;
  int64_t p0;
  int64_t g0;           // first accumulation item
  int64_t r0;           // first preparation item
  int na, nb, nc;       // preparation items of kinds a, b, c
  int ngram;
};

struct PbSlot {         // one operand buffer of the ring
  int8_t* F;
  double* G;
  double* sA;
  double* wmax;
  int* wsgn;
  double2* Mbuf;
};

struct PbParams {
  const PbQ* q;
  const PbSlab* slab;
  const PbSlot* slot;
  const CUtensorMap* maps;   // per (q, slot): A box (128 rows), B box (2 BN rows)
  int nslab, nslot, nw;
  int64_t ngram, nprep;
  const double* omega;
  unsigned long long* heads;  // [0] accumulation queue, [1] preparation queue
  int* ab;                    // per slab: finished (a) + (b) items
  int* ready;                 // per slab: finished (c) items
  int* gdone;                 // per slab: finished accumulation items
  int* status;
  uint64_t timeout_ns;
  unsigned long long* prof;   // SPX_PB_PROF_N role counters, or NULL
};

#if defined(__CUDACC__)
__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void red_release_add(int* p, int v) {
  asm volatile("red.release.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}
// Bounded wait until *ctr >= target (acquire). False on timeout (status set) or
// when another worker has already given up. The first look is inline (the counter is
// usually there already); the spinning is a call, so its code exists once.
__device__ __noinline__ bool gwait_spin(const int* ctr, int target, uint64_t timeout_ns, int* status) {
  const uint64_t t0 = global_ns();
  uint32_t nap = 64;  // doubling up to 2 us: long waits (a buffer, a slab) poll rarely
  for (uint32_t n = 1;; ++n) {
    __nanosleep(nap);
    if (nap < 2048) nap <<= 1;
    if (ld_acquire(ctr) >= target) return true;
    if ((n & 31) == 0) {
      if (global_ns() - t0 > timeout_ns) {
        atomicCAS(status, 0, (int)kStatusTimeout);
        return false;
      }
      if (*((volatile int*)status) != 0) return false;
    }
  }
}
__device__ __forceinline__ bool gwait(const int* ctr, int target, uint64_t timeout_ns, int* status) {
  return ld_acquire(ctr) >= target || gwait_spin(ctr, target, timeout_ns, status);
}
// The last index k with key(k) <= v over a nondecreasing array (first entry <= v).
__device__ __forceinline__ int pb_find(const PbSlab* sl, int n, int64_t v, bool prep) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if ((prep ? sl[mid].r0 : sl[mid].g0) <= v) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}
#endif

// Tiles of the upper region for 64-row x BN-column tiles, column-major (column block
// bj holds the row blocks that reach its last column, at most the last of N's).
template <int BN>
inline int pb_ntile(int N) {
  const int nb = (N + BN - 1) / BN, nbr = (N + 63) / 64;
  int c = 0;
  for (int j = 0; j < nb; ++j) c += split_rows_of(j, BN, nbr);
  return c;
}

// Columns of a tile the epilogue stages in shared memory: all of them, except for the
// 64 x 80 tile, whose second half stays in registers (three pipeline stages then fit).
constexpr int pb_sbn(int bn) { return bn == 80 ? 40 : bn; }

// An accumulation item as the pipeline roles read it (taken from the queue and
// decoded ahead of use, so that no role waits on global memory between items).
struct PbItem {
  int k;                // slab (-1: the queue is empty)
  int tile, f, bi, bj;  // tile (round-aware order), frequency, its row / column blocks
  int nk, jr;           // 64-pair stages, K direction of the round
  int qi, slot, nc;     // q point, operand buffer, digit items that make the planes ready
  int same;             // set by the TMA producer: A doubles as B (diagonal 64 x 64 tile)
  int pad;
  const int* wsgn;      // the buffer's per-frequency weight signs
};

template <int BN, int ST>
struct __align__(1024) PbSmem {
  uint8_t a[ST][SP_SF][SP_PLANE];
  uint8_t b[ST][SP_SF][2 * BN * SP_KB];
  double stage[SP_ROWS][pb_sbn(BN) + 1];  // epilogue: the tile's values (the first
                                         // pb_sbn(BN) columns; the rest in registers)
  uint64_t full[ST], empty[ST];
  uint64_t tfull, tempty, mdone;
  uint64_t ifull[PB_RING];
  PbItem item[PB_RING];                 // accumulation items taken ahead, decoded
  long long prep_item;
  int ecount[PB_RING];                  // epilogue warps done with a ring entry's item
  double red[PB_NPREP / 32];
  int redi[2][PB_NPREP / 32];
  uint32_t tmem_base;
};

#if defined(__CUDACC__)
// ---------------- preparation workers (192 threads) ----------------
__device__ __forceinline__ void pb_prep_bar() { named_bar_sync(1, PB_NPREP); }

// Adds a role's cycle counts to the launch's profile (prm.prof, when given).
__device__ __forceinline__ void pb_prof_add(const PbParams& prm, int k, unsigned long long v) {
  if (prm.prof && v) atomicAdd(prm.prof + k, v);
}

template <int BN, int ST>
__device__ void pb_prep(PbSmem<BN, ST>& sm, const PbParams& prm, int pt) {
  const int pw = pt >> 5, lane = pt & 31;
  unsigned long long c_wait = 0, c_kind[3] = {0, 0, 0}, n_items = 0;
  for (;;) {
    if (pt == 0) sm.prep_item = (long long)atomicAdd(&prm.heads[1], 1ull);
    pb_prep_bar();
    const int64_t item = sm.prep_item;
    pb_prep_bar();  // everyone has read it before thread 0 may overwrite it
    if (item >= prm.nprep) break;
    const int k = pb_find(prm.slab, prm.nslab, item, true);
    const PbSlab& sl = prm.slab[k];
    const PbQ& q = prm.q[sl.q];
    const PbSlot& slot = prm.slot[sl.slot];
    int64_t local = item - sl.r0;
    const int kind = local < sl.na ? 0 : (local < sl.na + sl.nb ? 1 : 2);
    local -= kind == 0 ? 0 : (kind == 1 ? sl.na : sl.na + sl.nb);
    // the buffer must be free (the slab that used it last fully accumulated), and a
    // quantizer item needs its slab's maxima and factors
    int ok = 1;
    const long long t0 = clock64();
    if (pt == 0) {
      if (k >= prm.nslot) {
        const PbSlab& prev = prm.slab[k - prm.nslot];
        ok = gwait(&prm.gdone[k - prm.nslot], prev.ngram, prm.timeout_ns, prm.status);
      }
      if (ok && kind == 2) ok = gwait(&prm.ab[k], sl.na + sl.nb, prm.timeout_ns, prm.status);
      sm.redi[0][0] = ok;
    }
    pb_prep_bar();
    ok = sm.redi[0][0];
    pb_prep_bar();
    if (!ok) break;
    const long long t1 = clock64();

    if (kind == 0) {
      // (a) column i: M values of the slab (generated into the buffer, or the
      // caller's) and their largest |Re|, |Im|
      const int i = (int)local * PB_ACOLS + pw;
      if (i < q.N) {
        double m = 0.0;
        if (q.M) {
          const double2* col = q.M + (int64_t)i * q.ldc + sl.p0;
          for (int p = lane; p < sl.len; p += 32) {
            const double2 v = col[p];
            m = fmax(m, fmax(fabs(v.x), fabs(v.y)));
          }
        } else {
          double2* dst = slot.Mbuf + (int64_t)i * sl.lenp;
          for (int p = lane; p < sl.len; p += 32) {
            double z0, z1;
            normal_pair(q.seed, q.sid, (uint64_t)(q.P * i + sl.p0 + p), &z0, &z1);
            const double2 v = make_double2(__dmul_rn(q.mscale, z0), __dmul_rn(q.mscale, z1));
            dst[p] = v;
            m = fmax(m, fmax(fabs(v.x), fabs(v.y)));
          }
        }
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 0) slot.sA[i] = m;
      }
    } else if (kind == 1) {
      // (b) frequency f: weights, their maximum and sign, the folded factors
      const int f = (int)local;
      const double om = prm.omega[f];
      double m = 0.0;
      int pos = 0, neg = 0;
      for (int p = pt; p < sl.len; p += PB_NPREP) {
        const double s = (q.wscale ? q.wscale[sl.p0 + p] : 1.0) * q.scale_all;
        const double w = hilbert_none_weight(q.ediff[sl.p0 + p], om, s);
        m = fmax(m, fabs(w));
        pos |= w > 0.0;
        neg |= w < 0.0;
      }
      for (int o = 16; o > 0; o >>= 1) {
        m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        pos |= __shfl_xor_sync(0xffffffffu, pos, o);
        neg |= __shfl_xor_sync(0xffffffffu, neg, o);
      }
      if (lane == 0) sm.red[pw] = m, sm.redi[0][pw] = pos, sm.redi[1][pw] = neg;
      pb_prep_bar();
      m = 0.0;
      pos = neg = 0;
#pragma unroll
      for (int w = 0; w < PB_NPREP / 32; ++w)
        m = fmax(m, sm.red[w]), pos |= sm.redi[0][w], neg |= sm.redi[1][w];
      pb_prep_bar();
      if (pt == 0) {
        slot.wmax[f] = m;
        slot.wsgn[f] = (pos && neg) ? 0 : (neg ? -1 : 1);
      }
      double* gf = slot.G + (int64_t)f * sl.lenp;
      for (int p = pt; p < sl.lenp; p += PB_NPREP) {
        double g = 0.0;
        if (p < sl.len) {
          const double s = (q.wscale ? q.wscale[sl.p0 + p] : 1.0) * q.scale_all;
          g = fold_factor(hilbert_none_weight(q.ediff[sl.p0 + p], om, s), m);
        }
        gf[p] = g;
      }
    } else {
      // (c) digit planes of 8 columns: tasks (column, 16 pairs), a warp = 8 columns x
      // the 4 quarters of one 64-pair block
      const int nchunk = sl.lenp / 16;
      const int64_t nkb = q.S / SP_KB;
      const int64_t pstride = nkb * q.R * SP_KB;
      for (int t = pt; t < PB_QCOLS * nchunk; t += PB_NPREP) {
        const int lane8 = t & 7, quarter = (t >> 3) & 3, kb = t >> 5;
        const int i = (int)local * PB_QCOLS + lane8;
        const int p = kb * SP_KB + quarter * 16;
        const bool col_ok = i < q.N;
        const int ic = col_ok ? i : 0;
        const double2* col =
            q.M ? q.M + (int64_t)ic * q.ldc + sl.p0 : slot.Mbuf + (int64_t)ic * sl.lenp;
        const int64_t o_re = ((int64_t)kb * q.R + split_row_re(i)) * SP_KB + quarter * 16;
        quantize_task(col, col_ok, sl.len, p, col_ok ? slot.sA[i] : 0.0, o_re, pstride, prm.nw,
                      slot.wsgn, slot.G, sl.lenp, slot.F);
      }
    }
    // publish: generic stores become visible to the TMA (async proxy) and to the
    // other CTAs before the counter moves
    fence_proxy_async_global();
    __threadfence();
    pb_prep_bar();
    if (pt == 0) red_release_add(kind == 2 ? &prm.ready[k] : &prm.ab[k], 1);
    c_wait += (unsigned long long)(t1 - t0);
    c_kind[kind] += (unsigned long long)(clock64() - t1);
    ++n_items;
  }
  if (pt == 0) {
    pb_prof_add(prm, 8, c_wait);
    for (int k = 0; k < 3; ++k) pb_prof_add(prm, 9 + k, c_kind[k]);
    pb_prof_add(prm, 13, n_items);
  }
}

// Takes the next accumulation item from the queue into `it`. A CTA's items come in
// increasing order, so the slab is searched forward from `kprev` (the slab of the
// CTA's previous item), with a binary search when it lies further on.
template <int BN>
__device__ __forceinline__ void pb_take_item(const PbParams& prm, int kprev, PbItem* it) {
  const int64_t g = kprev < 0 ? prm.ngram : (int64_t)atomicAdd(&prm.heads[0], 1ull);
  if (g >= prm.ngram) {
    it->k = -1;
    return;
  }
  int k = kprev, n = 0;
  while (k + 1 < prm.nslab && prm.slab[k + 1].g0 <= g && ++n <= 8) ++k;
  if (n > 8) k = pb_find(prm.slab, prm.nslab, g, false);
  const PbSlab& sl = prm.slab[k];
  const PbQ& q = prm.q[sl.q];
  const int local = (int)(g - sl.g0);
  const int tile = split_round_tile(local % q.ntile, q.ntile, g - local % q.ntile, gridDim.x);
  int bi, bj;
  split_decode_tile_bn<BN>(tile, q.nblk, &bi, &bj);
  it->k = k;
  it->tile = tile;
  it->f = local / q.ntile;
  it->bi = bi;
  it->bj = bj;
  it->nk = sl.nk;
  it->jr = (int)((g / gridDim.x) & 1);
  it->qi = sl.q;
  it->slot = sl.slot;
  it->nc = sl.nc;
  it->same = 0;
  it->wsgn = prm.slot[sl.slot].wsgn;
}

template <int BN, int ST>
__global__ void __launch_bounds__(PB_THREADS, 1) pb_kernel(PbParams prm) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  using Smem = PbSmem<BN, ST>;
  Smem& sm = *reinterpret_cast<Smem*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                      ~(uintptr_t)1023);
  constexpr int BROWS = 2 * BN;                  // B rows (N of the MMA)
  constexpr uint32_t IDESC = sp_idesc(BROWS);
  constexpr uint32_t OSTRIDE = BROWS;            // TMEM columns per order
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long t_start = clock64();

  if (threadIdx.x == 0) {
    for (int s = 0; s < ST; ++s) {
      mbar_init(&sm.full[s], 1);
      mbar_init(&sm.empty[s], 1);
    }
    for (int r = 0; r < PB_RING; ++r) {
      mbar_init(&sm.ifull[r], 1);
      sm.ecount[r] = 0;
    }
    mbar_init(&sm.tfull, 1);
    mbar_init(&sm.tempty, PB_EPI);
    mbar_init(&sm.mdone, 1);
    fence_barrier_init();
  }
  if (warp == 1) tmem_alloc(&sm.tmem_base, SP_TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sm.tmem_base;

  if (threadIdx.x >= PB_PREP0) {
    pb_prep<BN, ST>(sm, prm, threadIdx.x - PB_PREP0);
  } else if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      int st = 0;
      uint32_t ph = 0;
      bool issued[ST];
      uint32_t last_ph[ST];
      unsigned long long c_ready = 0, c_empty = 0, n_items = 0;
      for (int s = 0; s < ST; ++s) issued[s] = false, last_ph[s] = 0;
      for (int j = 0;; ++j) {
        const int r = j % PB_RING;
        if (!mbar_wait(&sm.ifull[r], (uint32_t)((j / PB_RING) & 1), prm.timeout_ns, prm.status)) break;
        const PbItem it = sm.item[r];
        if (it.k < 0) break;
        // the slab's planes must be ready before the first copy
        long long tw = clock64();
        const bool okr = gwait(&prm.ready[it.k], it.nc, prm.timeout_ns, prm.status);
        c_ready += (unsigned long long)(clock64() - tw);
        ++n_items;
        if (!okr) break;
        const int sg = it.wsgn[it.f];
        const bool same = BN == SP_TILE && sg != 0 && it.bi == it.bj;
        // read by the MMA issuer once the item's first stage has landed (the stage's
        // barrier orders this store before that read)
        sm.item[r].same = same ? 1 : 0;
        fence_proxy_async_global();
        const CUtensorMap* mA = prm.maps + 2 * ((int64_t)it.qi * prm.nslot + it.slot);
        const CUtensorMap* mB = mA + 1;
        const int za = it.f * SP_SLOT, zb = za + (sg == 0 ? SP_SF : 0);
        bool ok = true;
        for (int ks = 0; ks < it.nk; ++ks) {
          tw = clock64();
          if (!mbar_wait(&sm.empty[st], ph ^ 1u, prm.timeout_ns, prm.status)) {
            ok = false;
            break;
          }
          c_empty += (unsigned long long)(clock64() - tw);
          mbar_arrive_expect_tx(&sm.full[st], (uint32_t)(SP_SF * (SP_PLANE + (same ? 0 : BROWS * SP_KB))));
          const int kc = split_k_order(it.jr, ks, it.nk);
          tma_load_4d(&sm.a[st][0][0], mA, 0, it.bi * SP_ROWS, kc, za, &sm.full[st]);
          if (!same) tma_load_4d(&sm.b[st][0][0], mB, 0, it.bj * BROWS, kc, zb, &sm.full[st]);
          issued[st] = true;
          last_ph[st] = ph;
          if (++st == ST) st = 0, ph ^= 1u;
        }
        if (!ok) break;
      }
      for (int s = 0; s < ST; ++s)
        if (issued[s]) mbar_drain(&sm.full[s], last_ph[s], prm.timeout_ns);
      pb_prof_add(prm, 1, c_ready);
      pb_prof_add(prm, 2, c_empty);
      pb_prof_add(prm, 12, n_items);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      int st = 0;
      uint32_t ph = 0;
      bool committed = false;
      unsigned long long c_item = 0, c_acc = 0, c_full = 0;
      for (int j = 0;; ++j) {
        const int r = j % PB_RING;
        long long tw = clock64();
        if (!mbar_wait_idle(&sm.ifull[r], (uint32_t)((j / PB_RING) & 1), prm.timeout_ns, prm.status)) break;
        c_item += (unsigned long long)(clock64() - tw);
        const int kslab = sm.item[r].k;
        if (kslab < 0) break;
        const int nk = sm.item[r].nk;
        bool same = false;
        tw = clock64();
        if (!mbar_wait(&sm.tempty, (uint32_t)(j & 1) ^ 1u, prm.timeout_ns, prm.status)) break;
        c_acc += (unsigned long long)(clock64() - tw);
        tc_fence_after();
        bool ok = true;
        for (int ks = 0; ks < nk; ++ks) {
          tw = clock64();
          if (!mbar_wait(&sm.full[st], ph, prm.timeout_ns, prm.status)) {
            ok = false;
            break;
          }
          c_full += (unsigned long long)(clock64() - tw);
          tc_fence_after();
          if (ks == 0) same = sm.item[r].same != 0;
#pragma unroll
          for (int kk = 0; kk < SP_NKS; ++kk) {
            uint64_t da[SP_SF], db[SP_SF];
#pragma unroll
            for (int t = 0; t < SP_SF; ++t) {
              da[t] = desc_sw64(&sm.a[st][t][0]) + (uint64_t)(kk * 2);
              db[t] = same ? da[t] : desc_sw64(&sm.b[st][t][0]) + (uint64_t)(kk * 2);
            }
            const uint32_t k0 = (ks > 0 || kk > 0);
            mma_i8<1>(tmem + 0 * OSTRIDE, da[0], db[0], IDESC, k0);
            mma_i8<2>(tmem + 1 * OSTRIDE, da[0], db[1], IDESC, k0);
            mma_i8<3>(tmem + 2 * OSTRIDE, da[0], db[2], IDESC, k0);
            mma_i8<1>(tmem + 1 * OSTRIDE, da[1], db[0], IDESC, 1u);
            mma_i8<3>(tmem + 2 * OSTRIDE, da[1], db[1], IDESC, 1u);
            mma_i8<0>(tmem + 2 * OSTRIDE, da[2], db[0], IDESC, 1u);
          }
          tc_commit(&sm.empty[st]);
          committed = true;
          if (++st == ST) st = 0, ph ^= 1u;
        }
        if (!ok) break;
        tc_commit(&sm.tfull);
      }
      if (committed) {
        tc_commit(&sm.mdone);
        mbar_drain(&sm.mdone, 0u, prm.timeout_ns);
      }
      pb_prof_add(prm, 3, c_full);
      pb_prof_add(prm, 4, c_acc);
      pb_prof_add(prm, 5, c_item);
    }
  } else {
    // ---------------- epilogue: warps 2-5, TMEM lane quarter warp % 4 ----------------
    const int qd = warp & 3;
    const int row = 32 * qd + lane;          // TMEM lane = real-stacked row of the tile
    const int c = lane & 1;
    const uint32_t tl = tmem + ((uint32_t)(32 * qd) << 16);
    unsigned long long c_tile = 0, c_seq = 0;
    if (threadIdx.x == 64) {
      // the first PB_RING items; afterwards each entry is refilled by the warp that
      // retires its item
      int kprev = pb_find(prm.slab, prm.nslab, 0, false);
      for (int r = 0; r < PB_RING; ++r) {
        pb_take_item<BN>(prm, kprev, &sm.item[r]);
        kprev = sm.item[r].k;
        mbar_arrive(&sm.ifull[r]);
      }
    }
    for (int j = 0;; ++j) {
      const int r = j % PB_RING;
      long long tw = clock64();
      if (!mbar_wait_idle(&sm.ifull[r], (uint32_t)((j / PB_RING) & 1), prm.timeout_ns, prm.status)) break;
      const int kslab = sm.item[r].k;
      if (kslab < 0) break;
      const int tile = sm.item[r].tile, f = sm.item[r].f, bi = sm.item[r].bi, bj = sm.item[r].bj;
      if (!mbar_wait_idle(&sm.tfull, (uint32_t)(j & 1), prm.timeout_ns, prm.status)) break;
      c_tile += (unsigned long long)(clock64() - tw);
      tc_fence_after();
      const PbSlab& sl = prm.slab[kslab];
      const PbQ& q = prm.q[sl.q];
      const PbSlot& slot = prm.slot[sl.slot];
      // the accumulator, combined into complex values, into shared memory (columns
      // below SBN) and registers (the rest)
      constexpr int SBN = pb_sbn(BN);
      double o[BN > SBN ? BN - SBN : 1];
#pragma unroll 1
      for (int cc = 0; cc < SBN / 8; ++cc) {
        double T[16];
        load_fold16(tl + (uint32_t)(16 * cc), OSTRIDE, T);
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) {
          const double pb = __shfl_xor_sync(0xffffffffu, T[2 * jj + 1], 1);
          sm.stage[row][8 * cc + jj] = c == 0 ? T[2 * jj] + pb : T[2 * jj] - pb;
        }
      }
      if constexpr (BN > SBN) {
#pragma unroll
        for (int cc = SBN / 8; cc < BN / 8; ++cc) {
          double T[16];
          load_fold16(tl + (uint32_t)(16 * cc), OSTRIDE, T);
#pragma unroll
          for (int jj = 0; jj < 8; ++jj) {
            const double pb = __shfl_xor_sync(0xffffffffu, T[2 * jj + 1], 1);
            o[8 * cc + jj - SBN] = c == 0 ? T[2 * jj] + pb : T[2 * jj] - pb;
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&sm.tempty);  // the MMAs of the next item may start
      // slab s of this q adds into the tile after slab s-1 did (the order of per-q calls);
      // each warp adds only its own rows (its staged values), so the warps need no
      // barrier among themselves
      int* seq = q.seq + (int64_t)f * q.ntile + tile;
      int ok = 1;
      tw = clock64();
      if (lane == 0 && sl.s > 0) ok = gwait(seq, sl.s, prm.timeout_ns, prm.status);
      ok = __shfl_sync(0xffffffffu, ok, 0);
      c_seq += (unsigned long long)(clock64() - tw);
      const int gil = bi * SP_TILE + row / 2;
      if (ok && gil < q.N) {
        const double fac = fold_row_factor(slot.wsgn[f], slot.sA[gil], slot.wmax[f]);
        double* ob = q.out + 2 * (int64_t)f * q.npack + 2 * gil + c;
        for (int jj = 0; jj < SBN; ++jj) {
          const int gj = bj * BN + jj;
          if (gil <= gj && gj < q.N)
            atomicAdd(ob + (int64_t)gj * (gj + 1), fac * slot.sA[gj] * sm.stage[row][jj]);
        }
        if constexpr (BN > SBN) {
#pragma unroll
          for (int jj = SBN; jj < BN; ++jj) {
            const int gj = bj * BN + jj;
            if (gil <= gj && gj < q.N)
              atomicAdd(ob + (int64_t)gj * (gj + 1), fac * slot.sA[gj] * o[jj - SBN]);
          }
        }
      }
      // the last warp done with the item publishes it (the tile's order counter, the
      // slab's count) and refills the ring entry with the item PB_RING further on (no
      // CTA barrier, so a warp that gave up on a wait cannot hold the others)
      __threadfence();
      __syncwarp();
      if (lane == 0 && atomicAdd(&sm.ecount[r], 1) % PB_EPI == PB_EPI - 1) {
        __threadfence();
        red_release_add(seq, 1);
        red_release_add(&prm.gdone[kslab], 1);
        pb_take_item<BN>(prm, sm.item[(r + PB_RING - 1) % PB_RING].k, &sm.item[r]);
        mbar_arrive(&sm.ifull[r]);
      }
      if (!ok) break;
    }
    if (warp == 2 && lane == 0) {
      pb_prof_add(prm, 6, c_tile);
      pb_prof_add(prm, 7, c_seq);
    }
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1) tmem_dealloc(tmem, SP_TMEM_COLS);
  if (threadIdx.x == 0) pb_prof_add(prm, 0, (unsigned long long)(clock64() - t_start));
}
#endif

// ---------------------------------------------------------------------------
// host side

int make_tmap_u8_4d(spx_ctx* ctx, CUtensorMap* map, const void* base, const uint64_t dims[4],
                    const uint64_t strides[3], const uint32_t box[4], CUtensorMapSwizzle swz);

struct PbConfig {
  int bn, stages;
};

static size_t pb_smem(PbConfig c) {
  if (c.bn == 64) return sizeof(PbSmem<64, 3>) + 1024;
  if (c.bn == 80) return sizeof(PbSmem<80, 3>) + 1024;
  return c.stages == 4 ? sizeof(PbSmem<32, 4>) + 1024 : sizeof(PbSmem<32, 3>) + 1024;
}

// The schedule of one batch on the device: descriptors, ring buffers, counters.
struct PbPlan {
  std::vector<PbQ> q;
  std::vector<PbSlab> slab;
  std::vector<PbSlot> slot;
  std::vector<CUtensorMap> maps;
  int64_t ngram = 0, nprep = 0;
  size_t slot_bytes = 0, ctr_bytes = 0, seq_ints = 0;
};

// Bytes of the ring and the device descriptors for `nq` q points at slab sizes S_q.
size_t pb_plan_bytes(int nq, const spx_q_desc* qd, const int* S, int nw, int nslot) {
  size_t per_slot = 0, seq = 0;
  int64_t nslab = 0;
  for (int i = 0; i < nq; ++i) {
    const int N = qd[i].nbas;
    if (N <= 0 || qd[i].npair <= 0) continue;
    const int nblk = (N + 63) / 64;
    const int64_t R = (int64_t)((nblk + 1) / 2 * 2) * SP_ROWS;
    size_t b = align_up((size_t)SP_SLOT * nw * R * S[i], 1024) + align_up(sizeof(double) * (size_t)nw * S[i], 256) +
               align_up(sizeof(double) * (size_t)R, 256) + 2 * align_up(sizeof(double) * (size_t)nw, 256) +
               (qd[i].cprod ? 0 : align_up(sizeof(double2) * (size_t)N * S[i], 256));
    per_slot = std::max(per_slot, b);
    seq += (size_t)pb_ntile<32>(N) * nw;   // the largest of the tilings (32, 64, 80 columns)
    nslab += (qd[i].npair + S[i] - 1) / S[i];
  }
  const size_t desc = align_up(sizeof(PbQ) * nq, 256) + align_up(sizeof(PbSlab) * nslab, 256) +
                      align_up(sizeof(PbSlot) * nslot, 256) +
                      align_up(sizeof(CUtensorMap) * 2 * (size_t)nq * nslot, 256);
  const size_t ctr = align_up(sizeof(unsigned long long) * 2 + sizeof(int) * (3 * nslab + seq), 256);
  return per_slot * nslot + desc + ctr + 4096;
}

// Builds the schedule into `mem` (device, pb_plan_bytes large): the descriptors are
// copied there in order on `s`, after whatever `s` already runs (a previous launch
// on the same scratch still reads its own); the counters (the first `*ctr_bytes`
// bytes at *ctr) must be zeroed before every launch.
int pb_build(spx_ctx* ctx, int nq, const spx_q_desc* qd, const int* S, int nw, int nslot,
             PbConfig cfg, const double* omega, char* mem, size_t mem_bytes, PbParams* out,
             void** ctr, size_t* ctr_bytes, cudaStream_t s) {
  (void)mem_bytes;
  // q order: most work first
  std::vector<int> order;
  for (int i = 0; i < nq; ++i)
    if (qd[i].nbas > 0 && qd[i].npair > 0) order.push_back(i);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    return (double)qd[a].nbas * qd[a].nbas * (double)qd[a].npair >
           (double)qd[b].nbas * qd[b].nbas * (double)qd[b].npair;
  });
  std::vector<PbQ> q(nq);
  std::vector<PbSlab> slabs;
  int64_t g0 = 0, r0 = 0;
  size_t seq_total = 0;
  std::vector<size_t> seq_off(nq, 0);
  for (int i = 0; i < nq; ++i) {
    const spx_q_desc& d = qd[i];
    PbQ& x = q[i];
    std::memset(&x, 0, sizeof(x));
    x.N = d.nbas;
    x.P = d.npair;
    if (x.N <= 0 || x.P <= 0) continue;
    x.nblk = (x.N + 63) / 64;
    x.ntile = cfg.bn == 64 ? pb_ntile<64>(x.N) : (cfg.bn == 80 ? pb_ntile<80>(x.N) : pb_ntile<32>(x.N));
    x.R = (int64_t)((x.nblk + 1) / 2 * 2) * SP_ROWS;
    x.npad = (int)(x.R / 2);
    x.S = S[i];
    x.nslab = (int)((x.P + x.S - 1) / x.S);
    x.npack = (int64_t)x.N * (x.N + 1) / 2;
    x.M = reinterpret_cast<const double2*>(d.cprod);
    x.ldc = d.ldc;
    x.seed = d.seed;
    x.sid = d.stream_id;
    x.mscale = d.m_scale;
    x.ediff = d.ediff;
    x.wscale = d.wscale;
    x.scale_all = d.scale_all;
    x.out = d.susceph;
    seq_off[i] = seq_total;
    seq_total += (size_t)x.ntile * nw;
  }
  for (int i : order) {
    const PbQ& x = q[i];
    for (int s = 0; s < x.nslab; ++s) {
      PbSlab sl;
      std::memset(&sl, 0, sizeof(sl));
      sl.q = i;
      sl.s = s;
      sl.slot = (int)(slabs.size() % nslot);
      sl.p0 = (int64_t)s * x.S;
      sl.len = (int)std::min<int64_t>(x.S, x.P - sl.p0);
      sl.lenp = (int)align_up((size_t)sl.len, SP_KB);
      sl.nk = sl.lenp / SP_KB;
      sl.g0 = g0;
      sl.r0 = r0;
      sl.na = (x.N + PB_ACOLS - 1) / PB_ACOLS;
      sl.nb = nw;
      sl.nc = x.npad / PB_QCOLS;
      sl.ngram = x.ntile * nw;
      g0 += sl.ngram;
      r0 += sl.na + sl.nb + sl.nc;
      slabs.push_back(sl);
    }
  }
  const int nslab = (int)slabs.size();
  Carve cv{mem, mem_bytes};
  // counters first (one memset per launch): heads, ab, ready, gdone, seq
  char* c0 = cv.p;
  unsigned long long* heads = cv.take<unsigned long long>(2);
  int* ab = cv.take<int>(nslab);
  int* ready = cv.take<int>(nslab);
  int* gdone = cv.take<int>(nslab);
  int* seq = cv.take<int>(seq_total);
  *ctr = c0;
  *ctr_bytes = (size_t)(cv.p - c0);
  for (int i = 0; i < nq; ++i) q[i].seq = seq + seq_off[i];
  PbQ* dq = cv.take<PbQ>(nq);
  PbSlab* dsl = cv.take<PbSlab>(nslab);
  PbSlot* dslot = cv.take<PbSlot>(nslot);
  CUtensorMap* dmaps = reinterpret_cast<CUtensorMap*>(cv.take<char>(sizeof(CUtensorMap) * 2 * (size_t)nq * nslot));
  // ring buffers sized for the largest q
  size_t fb = 0, gb = 0, sb = 0, mb = 0;
  for (int i = 0; i < nq; ++i) {
    if (q[i].N <= 0) continue;
    fb = std::max(fb, (size_t)SP_SLOT * nw * q[i].R * q[i].S);
    gb = std::max(gb, (size_t)nw * q[i].S);
    sb = std::max(sb, (size_t)q[i].R);
    if (!q[i].M) mb = std::max(mb, (size_t)q[i].N * q[i].S);
  }
  std::vector<PbSlot> slot(nslot);
  for (int b = 0; b < nslot; ++b) {
    slot[b].F = reinterpret_cast<int8_t*>(cv.take<char>(fb));
    slot[b].G = cv.take<double>(gb);
    slot[b].sA = cv.take<double>(sb);
    slot[b].wmax = cv.take<double>(nw);
    slot[b].wsgn = cv.take<int>(nw);
    slot[b].Mbuf = mb ? cv.take<double2>(mb) : nullptr;
  }
  if (!cv.ok) return set_error(ctx, SPX_ENOMEM, "persistent batch: scratch too small");
  // tensor maps per (q, slot): planes [6 nw][nkb][R][64 B]
  std::vector<CUtensorMap> maps(2 * (size_t)nq * nslot);
  for (int i = 0; i < nq; ++i) {
    if (q[i].N <= 0) continue;
    const uint64_t nkb = (uint64_t)(q[i].S / SP_KB);
    const uint64_t st[3] = {SP_KB, (uint64_t)q[i].R * SP_KB, nkb * q[i].R * SP_KB};
    const uint64_t dims[4] = {SP_KB, (uint64_t)q[i].R, nkb, (uint64_t)SP_SLOT * nw};
    const uint32_t ba[4] = {SP_KB, SP_ROWS, 1, SP_SF};
    const uint32_t bb[4] = {SP_KB, (uint32_t)(2 * cfg.bn), 1, SP_SF};
    for (int b = 0; b < nslot; ++b) {
      int rc = make_tmap_u8_4d(ctx, &maps[2 * ((size_t)i * nslot + b)], slot[b].F, dims, st, ba,
                               CU_TENSOR_MAP_SWIZZLE_64B);
      if (!rc)
        rc = make_tmap_u8_4d(ctx, &maps[2 * ((size_t)i * nslot + b) + 1], slot[b].F, dims, st, bb,
                             CU_TENSOR_MAP_SWIZZLE_64B);
      if (rc) return rc;
    }
  }
  int rc;
  // pageable sources: each copy is staged before the call returns, so the vectors may
  // go; the transfer itself is ordered on `s`
  if ((rc = check_cuda(ctx, cudaMemcpyAsync(dq, q.data(), sizeof(PbQ) * nq, cudaMemcpyHostToDevice, s), "plan copy")) ||
      (rc = check_cuda(ctx, cudaMemcpyAsync(dsl, slabs.data(), sizeof(PbSlab) * nslab, cudaMemcpyHostToDevice, s), "plan copy")) ||
      (rc = check_cuda(ctx, cudaMemcpyAsync(dslot, slot.data(), sizeof(PbSlot) * nslot, cudaMemcpyHostToDevice, s), "plan copy")) ||
      (rc = check_cuda(ctx, cudaMemcpyAsync(dmaps, maps.data(), sizeof(CUtensorMap) * maps.size(), cudaMemcpyHostToDevice, s), "plan copy")))
    return rc;
  PbParams& p = *out;
  std::memset(&p, 0, sizeof(p));
  p.q = dq;
  p.slab = dsl;
  p.slot = dslot;
  p.maps = dmaps;
  p.nslab = nslab;
  p.nslot = nslot;
  p.nw = nw;
  p.ngram = g0;
  p.nprep = r0;
  p.omega = omega;
  p.heads = heads;
  p.ab = ab;
  p.ready = ready;
  p.gdone = gdone;
  p.status = ctx->d_status;
  p.timeout_ns = (uint64_t)(ctx->opt.timeout_ms > 0 ? ctx->opt.timeout_ms : 4000) * 1000000ull;
  p.prof = ctx->prof_on ? ctx->d_prof : nullptr;
  return SPX_OK;
}

// Enqueues one launch of the schedule on `s` (the counters are zeroed first).
int pb_launch(spx_ctx* ctx, const PbParams& prm, PbConfig cfg, void* ctr, size_t ctr_bytes,
              cudaStream_t s) {
  int rc = check_cuda(ctx, cudaMemsetAsync(ctr, 0, ctr_bytes, s), "counters");
  if (rc) return rc;
  const size_t smem = pb_smem(cfg);
  const int grid = ctx->num_sms;
  if (cfg.bn == 64) {
    cudaFuncSetAttribute(pb_kernel<64, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    pb_kernel<64, 3><<<grid, PB_THREADS, smem, s>>>(prm);
  } else if (cfg.bn == 80) {
    // 64 x 80 tiles (N = 160 MMAs), three stages beside half the epilogue's staging
    cudaFuncSetAttribute(pb_kernel<80, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    pb_kernel<80, 3><<<grid, PB_THREADS, smem, s>>>(prm);
  } else if (cfg.stages == 4) {
    cudaFuncSetAttribute(pb_kernel<32, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    pb_kernel<32, 4><<<grid, PB_THREADS, smem, s>>>(prm);
  } else {
    cudaFuncSetAttribute(pb_kernel<32, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    pb_kernel<32, 3><<<grid, PB_THREADS, smem, s>>>(prm);
  }
  return check_cuda(ctx, cudaGetLastError(), "persistent batch launch");
}

// Operand buffers in the ring: four (the preparation runs up to three slabs ahead of
// the accumulation) while they take at most 24 GiB, else three.
static int pb_nslot(int nq, const spx_q_desc* q, const int* S, int nw) {
  return pb_plan_bytes(nq, q, S, nw, 4) <= ((size_t)24 << 30) ? 4 : 3;
}
constexpr int PB_DEFAULT_SLAB = 16384;
constexpr PbConfig PB_DEFAULT_CFG = {80, 3};
constexpr size_t PB_MAX_GRAPHS = 8;

static int pb_nbas_bucket(int N) { return (N + 127) / 128; }
static int pb_npair_bucket(int64_t P) { return P <= 16384 ? 0 : (P <= 32768 ? 1 : 2); }

static const spx_tune_entry* pb_find_tune(const spx_ctx* ctx, int N, int64_t P, int nw) {
  for (const auto& e : ctx->tune)
    if (e.variant == 4 && e.nbas_bucket == pb_nbas_bucket(N) && e.npair_bucket == pb_npair_bucket(P) &&
        e.nw == nw)
      return &e;
  return nullptr;
}

static PbConfig pb_cfg_of(int tile) {
  const int bn = tile & 255, st = tile >> 8;
  if (bn == 32 && (st == 3 || st == 4)) return {32, st};
  if (bn == 80 && st == 3) return {80, 3};
  return PB_DEFAULT_CFG;
}

static uint64_t pb_fnv(uint64_t h, const void* p, size_t n) {
  const unsigned char* b = (const unsigned char*)p;
  for (size_t i = 0; i < n; ++i) {
    h ^= b[i];
    h *= 1099511628211ull;
  }
  return h;
}

// One persistent launch for the whole batch (split precision). Slab sizes: the
// descriptor's, else the tuned, else 16384; tile shape: the tuned shape of the q
// with most work, else 64 x 80 with 3 stages (`force` overrides both when set).
int pb_run(spx_ctx* ctx, int nq, const spx_q_desc* q, int nw, const double* omega, int flags,
           cudaStream_t s, int* launches, const PbConfig* force, int force_slab, char* scratch,
           size_t scratch_bytes) {
  std::vector<int> S(nq, PB_DEFAULT_SLAB);
  PbConfig cfg = PB_DEFAULT_CFG;
  double most = -1;
  for (int i = 0; i < nq; ++i) {
    if (q[i].nbas <= 0 || q[i].npair <= 0) continue;
    const spx_tune_entry* t = pb_find_tune(ctx, q[i].nbas, q[i].npair, nw);
    int sl = q[i].slab_pairs > 0 ? q[i].slab_pairs : (t ? t->slab_pairs : PB_DEFAULT_SLAB);
    if (force_slab > 0) sl = force_slab;
    S[i] = std::max(SP_KB, std::min(SP_SLAB, sl / SP_KB * SP_KB));
    const double work = (double)q[i].nbas * q[i].nbas * (double)q[i].npair;
    if (work > most) {
      most = work;
      cfg = t ? pb_cfg_of(t->tile) : PB_DEFAULT_CFG;
    }
  }
  if (force) cfg = *force;
  const int nslot = pb_nslot(nq, q, S.data(), nw);
  const size_t bytes = pb_plan_bytes(nq, q, S.data(), nw, nslot);
  PbParams prm;
  void* ctr = nullptr;
  size_t ctr_bytes = 0;
  int rc;
  if (flags & SPX_BATCH_NOGRAPH) {
    // the caller's scratch, or the workspace from its start
    if (scratch) {
      if (scratch_bytes < bytes) return set_error(ctx, SPX_EINVAL, "persistent schedule: scratch too small");
    } else {
      if ((rc = ensure_workspace(ctx, bytes))) return rc;
      scratch = (char*)ctx->ws;
      scratch_bytes = ctx->ws_bytes;
    }
    if ((rc = pb_build(ctx, nq, q, S.data(), nw, nslot, cfg, omega, scratch, scratch_bytes,
                       &prm, &ctr, &ctr_bytes, s)))
      return rc;
    if ((rc = pb_launch(ctx, prm, cfg, ctr, ctr_bytes, s))) return rc;
    *launches = 1;
    return SPX_OK;
  }
  uint64_t key = 0x9e3779b97f4a7c15ull;
  key = pb_fnv(key, "persistent", 10);
  key = pb_fnv(key, &nq, sizeof(nq));
  key = pb_fnv(key, q, sizeof(spx_q_desc) * nq);
  key = pb_fnv(key, S.data(), sizeof(int) * nq);
  key = pb_fnv(key, &cfg, sizeof(cfg));
  key = pb_fnv(key, &nw, sizeof(nw));
  key = pb_fnv(key, &ctx->prof_on, sizeof(ctx->prof_on));
  key = pb_fnv(key, &omega, sizeof(omega));
  spx_ctx::BatchGraph* hit = nullptr;
  for (auto& g : ctx->graphs)
    if (g.key == key) hit = &g;
  if (!hit) {
    void* mem = nullptr;
    if (cudaMalloc(&mem, bytes) != cudaSuccess) {
      cudaGetLastError();
      return set_error(ctx, SPX_ENOMEM, "persistent batch: cannot allocate " + std::to_string(bytes) + " bytes");
    }
    rc = pb_build(ctx, nq, q, S.data(), nw, nslot, cfg, omega, (char*)mem, bytes, &prm, &ctr, &ctr_bytes,
                  ctx->stream);
    // the graph may be launched on another stream: the plan must have landed first
    if (!rc) rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "plan copy");
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    if (!rc) rc = check_cuda(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed), "begin capture");
    if (!rc) {
      rc = pb_launch(ctx, prm, cfg, ctr, ctr_bytes, ctx->stream);
      cudaError_t ee = cudaStreamEndCapture(ctx->stream, &graph);
      if (!rc) rc = check_cuda(ctx, ee, "end capture");
      if (!rc) rc = check_cuda(ctx, cudaGraphInstantiate(&exec, graph, 0), "graph instantiate");
    }
    if (rc) {
      cudaGetLastError();
      if (graph) cudaGraphDestroy(graph);
      cudaFree(mem);
      return rc;
    }
    if (ctx->graphs.size() >= PB_MAX_GRAPHS) {
      auto old = std::min_element(ctx->graphs.begin(), ctx->graphs.end(),
                                  [](const spx_ctx::BatchGraph& a, const spx_ctx::BatchGraph& b) {
                                    return a.last_use < b.last_use;
                                  });
      cudaGraphExecDestroy(old->exec);
      cudaGraphDestroy(old->graph);
      if (old->mem) cudaFree(old->mem);
      ctx->graphs.erase(old);
    }
    ctx->graphs.push_back({key, graph, exec, 0, mem});
    hit = &ctx->graphs.back();
  }
  hit->last_use = ++ctx->graph_clock;
  *launches = 1;
  return check_cuda(ctx, cudaGraphLaunch(hit->exec, s), "graph launch");
}

// Scratch of one call through the persistent schedule: nbas x npair explicit M,
// slabs of `slab` pairs.
size_t pb_single_bytes(int64_t P, int N, int nw, int slab) {
  spx_q_desc d;
  std::memset(&d, 0, sizeof(d));
  d.nbas = N;
  d.npair = P;
  d.cprod = reinterpret_cast<const double*>(16);   // explicit M: no generation buffer
  const int S = std::max(SP_KB, std::min(SP_SLAB, slab / SP_KB * SP_KB));
  return pb_plan_bytes(1, &d, &S, nw, pb_nslot(1, &d, &S, nw));
}

// One spx_chi0_accumulate_dev-style call (HILBERT NONE weights from ediff, explicit
// M on the device) through the persistent schedule with tile code `tile` and slab
// `slab`, in the caller's scratch.
int pb_single(spx_ctx* ctx, const double2* M, int64_t ldc, int64_t P, int N, const double* ediff,
              const double* wscale, double scale_all, int nw, const double* omega, double2* out,
              int tile, int slab, char* scratch, size_t scratch_bytes, cudaStream_t s, int* launches) {
  spx_q_desc d;
  std::memset(&d, 0, sizeof(d));
  d.nbas = N;
  d.npair = P;
  d.cprod = reinterpret_cast<const double*>(M);
  d.ldc = ldc;
  d.ediff = ediff;
  d.wscale = wscale;
  d.scale_all = scale_all;
  d.susceph = reinterpret_cast<double*>(out);
  const PbConfig cfg = pb_cfg_of(tile);
  int n = 0;
  const int rc = pb_run(ctx, 1, &d, nw, omega, SPX_BATCH_NOGRAPH, s, &n, &cfg, slab > 0 ? slab : PB_DEFAULT_SLAB,
                        scratch, scratch_bytes);
  *launches += n + 1;   // the counters' memset and the kernel
  return rc;
}

}  // namespace spx

using namespace spx;

namespace spx {
int launch_gen_normal(spx_ctx*, uint64_t, uint32_t, int64_t, int64_t, double, double*, cudaStream_t);
int launch_abs(spx_ctx*, int64_t, double*, cudaStream_t);
}

// Times the persistent schedule's tile shapes and slab sizes on a seeded probe of one
// q (M generated on the device), keeps the fastest as a variant-4 entry.
extern "C" int spx_autotune_batched(spx_ctx* ctx, int32_t nbas, int64_t npair, int32_t nw,
                                    spx_tune_entry* out) {
  if (!ctx) return SPX_EINVAL;
  if (nbas <= 0 || npair <= 0 || nw <= 0) return set_error(ctx, SPX_EINVAL, "empty probe");
  if (nbas > 46340) return set_error(ctx, SPX_EINVAL, "nbas too large");
  cudaSetDevice(ctx->device);
  const int slabs[3] = {8192, 16384, 32768};
  const PbConfig cfgs[4] = {{64, 3}, {80, 3}, {32, 4}, {32, 3}};
  const int64_t P = std::min<int64_t>(npair, 4 * (int64_t)SP_SLAB);
  const int64_t npack = (int64_t)nbas * (nbas + 1) / 2;
  // probe arrays in a private allocation (the schedule itself uses the workspace)
  const size_t e_bytes = align_up(sizeof(double) * (size_t)P, 256);
  const size_t o_bytes = align_up(sizeof(double2) * (size_t)npack * nw, 256);
  const size_t om_bytes = align_up(sizeof(double) * (size_t)nw, 256);
  char* buf = nullptr;
  if (cudaMalloc(&buf, e_bytes + o_bytes + om_bytes) != cudaSuccess) {
    cudaGetLastError();
    return set_error(ctx, SPX_ENOMEM, "autotune probe");
  }
  double* E = (double*)buf;
  double* O = (double*)(buf + e_bytes);
  double* OM = (double*)(buf + e_bytes + o_bytes);
  cudaStream_t s = ctx->stream;
  std::vector<double> om(nw);
  for (int f = 0; f < nw; ++f) om[f] = 1.0 + f;
  int rc = launch_gen_normal(ctx, 0x5eed, 78, 0, P, 3.0, E, s);
  if (!rc) rc = launch_abs(ctx, P, E, s);  // positive energies: one-signed weights
  if (!rc) rc = check_cuda(ctx, cudaMemcpyAsync(OM, om.data(), sizeof(double) * nw, cudaMemcpyHostToDevice, s), "probe");
  if (!rc) rc = check_cuda(ctx, cudaStreamSynchronize(s), "probe");
  spx_tune_entry best{};
  best.nbas_bucket = pb_nbas_bucket(nbas);
  best.npair_bucket = pb_npair_bucket(npair);
  best.nw = nw;
  best.variant = 4;
  best.tflops = -1;
  spx_q_desc d;
  std::memset(&d, 0, sizeof(d));
  d.nbas = nbas;
  d.npair = P;
  d.seed = 0x5eed;
  d.stream_id = 77;
  d.m_scale = 1.0 / std::sqrt((double)nbas);
  d.ediff = E;
  d.scale_all = 1.0;
  d.susceph = O;
  const double flops = 8.0 * (double)nbas * nbas * (double)P * nw;
  cudaEvent_t e0 = ctx->ev[8], e1 = ctx->ev[9];
  // rounds interleave the candidates (tile shape x slab) so that clock drift under the
  // power cap favours none of them; round 0 warms up, each keeps its best round
  struct Cand {
    int ci, slab;
    float ms;
  };
  std::vector<Cand> cands;
  // the 64 x 32 tile with 3 stages is kept as a shape (tuning tables may name it) but
  // not probed: it never beat the 4-stage form
  for (int ci = 0; ci < 3; ++ci)
    for (int sl : slabs) {
      if (sl == 32768 && P <= 16384) continue;
      cands.push_back({ci, sl, 1e30f});
    }
  // multi-pass windows, as in the single-call tuner: the clock settles per candidate
  constexpr int kPasses = 2;
  for (int round = 0; round < 2 && !rc; ++round)  // round 0 warms up
    for (auto& c : cands) {
      int launches = 0;
      cudaEventRecord(e0, s);
      for (int pass = 0; pass < kPasses && !rc; ++pass)
        rc = pb_run(ctx, 1, &d, nw, OM, SPX_BATCH_NOGRAPH, s, &launches, &cfgs[c.ci], c.slab, nullptr, 0);
      if (rc) break;
      cudaEventRecord(e1, s);
      if ((rc = collect_status(ctx, s, "batched autotune"))) break;
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (round) c.ms = std::min(c.ms, ms / kPasses);
    }
  if (!rc)
    for (const auto& c : cands) {
      const double tf = flops / (c.ms * 1e-3) / 1e12;
      if (tf > best.tflops) {
        best.tflops = tf;
        best.slab_pairs = c.slab;
        best.tile = cfgs[c.ci].bn + 256 * cfgs[c.ci].stages;
      }
    }
  cudaFree(buf);
  if (rc) return rc;
  bool stored = false;
  for (auto& e : ctx->tune)
    if (e.variant == 4 && e.nbas_bucket == best.nbas_bucket && e.npair_bucket == best.npair_bucket &&
        e.nw == nw) {
      e = best;
      stored = true;
    }
  if (!stored) ctx->tune.push_back(best);
  if (out) *out = best;
  return SPX_OK;
}

extern "C" int spx_pb_profile_enable(spx_ctx* ctx, int32_t on) {
  if (!ctx) return SPX_EINVAL;
  cudaSetDevice(ctx->device);
  if (on) {
    const size_t bytes = sizeof(unsigned long long) * SPX_PB_PROF_N;
    if (!ctx->d_prof && cudaMalloc(&ctx->d_prof, bytes) != cudaSuccess) {
      cudaGetLastError();
      ctx->d_prof = nullptr;
      return set_error(ctx, SPX_ENOMEM, "profile counters");
    }
    int rc = check_cuda(ctx, cudaMemsetAsync(ctx->d_prof, 0, bytes, ctx->stream), "profile counters");
    if (!rc) rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "profile counters");
    if (rc) return rc;
  }
  ctx->prof_on = on != 0;
  return SPX_OK;
}

extern "C" int spx_pb_profile_read(spx_ctx* ctx, double* out, int32_t n) {
  if (!ctx || !out || n < 0) return SPX_EINVAL;
  cudaSetDevice(ctx->device);
  unsigned long long v[SPX_PB_PROF_N] = {};
  if (ctx->d_prof) {
    int rc = check_cuda(ctx, cudaDeviceSynchronize(), "profile read");
    if (!rc) rc = check_cuda(ctx, cudaMemcpy(v, ctx->d_prof, sizeof(v), cudaMemcpyDeviceToHost), "profile read");
    if (rc) return rc;
  }
  for (int k = 0; k < n && k < SPX_PB_PROF_N; ++k) out[k] = (double)v[k];
  return SPX_OK;
}

extern "C" int spx_tune_lookup_batched(const spx_ctx* ctx, int32_t nbas, int64_t npair, int32_t nw,
                                       spx_tune_entry* out) {
  if (!ctx) return SPX_EINVAL;
  const spx_tune_entry* t = pb_find_tune(ctx, nbas, npair, nw);
  if (!t) return SPX_ENOTSUP;
  if (out) *out = *t;
  return SPX_OK;
}
