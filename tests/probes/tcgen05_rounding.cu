// tcgen05 kind::f16 (BF16 in, FP32 accumulate) probe: checks one MMA 128x256x16
// against the CPU, then measures how the accumulator rounds (diagonal tests).
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <cmath>
#include <cuda_runtime.h>

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// SWIZZLE_NONE K-major canonical layout: core matrix = 8 rows x 16 B; K chunks (8 elems)
// at LBO = 128 B, 8-row groups at SBO = 256 B (for K = 16 per tile).
__device__ __forceinline__ uint32_t off_none(int row, int k) {
  return (row >> 3) * 256 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2;
}
__device__ __forceinline__ uint64_t desc_none(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((128 >> 4) & 0x3FFF) << 16;   // LBO
  d |= (uint64_t)((256 >> 4) & 0x3FFF) << 32;   // SBO
  d |= (uint64_t)1 << 46;                       // version (sm100)
  return d;                                     // layout type 0 = SWIZZLE_NONE
}
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((256u >> 3) << 17) | ((128u >> 4) << 24);

template <int S>
__global__ void probe(const uint16_t* A, const uint16_t* B, float* out) {
  __shared__ __align__(1024) uint8_t sa[S][128 * 32];
  __shared__ __align__(1024) uint8_t sb[S][256 * 32];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_base;
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 256;" :: "r"(su32(&tmem_base)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  for (int s = 0; s < S; ++s) {
    for (int t = threadIdx.x; t < 128 * 16; t += blockDim.x) { int r = t / 16, k = t % 16;
      *(uint16_t*)(sa[s] + off_none(r, k)) = A[(s * 128 + r) * 16 + k]; }
    for (int t = threadIdx.x; t < 256 * 16; t += blockDim.x) { int r = t / 16, k = t % 16;
      *(uint16_t*)(sb[s] + off_none(r, k)) = B[(s * 256 + r) * 16 + k]; }
  }
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(su32(&bar)));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  uint32_t tm = tmem_base;
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      uint64_t da = desc_none(su32(sa[s])), db = desc_none(su32(sb[s]));
      uint32_t acc = s > 0;
      asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                   " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
                   :: "r"(tm), "l"(da), "l"(db), "r"(IDESC), "r"(acc));
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" :: "r"(su32(&bar)) : "memory");
  }
  // bounded wait on the commit
  {
    uint32_t ok = 0; long long t0 = clock64();
    while (!ok) {
      asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0,1,0,p;\n}\n" : "=r"(ok) : "r"(su32(&bar)) : "memory");
      if (clock64() - t0 > 4000000000LL) break;
    }
  }
  asm volatile("tcgen05.fence::after_thread_sync;");
  for (int c0 = 0; c0 < 256; c0 += 8) {
    uint32_t r[8];
    uint32_t addr = tm + ((uint32_t)(warp * 32) << 16) + c0;
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]),"=r"(r[1]),"=r"(r[2]),"=r"(r[3]),"=r"(r[4]),"=r"(r[5]),"=r"(r[6]),"=r"(r[7]) : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;");
    for (int j = 0; j < 8; ++j) out[(warp * 32 + lane) * 256 + c0 + j] = __uint_as_float(r[j]);
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 256;" :: "r"(tm));
}

static uint16_t bf(float x) { uint32_t u; memcpy(&u, &x, 4); return (uint16_t)(u >> 16); }
static float fb(uint16_t h) { uint32_t u = (uint32_t)h << 16; float x; memcpy(&x, &u, 4); return x; }

template <int S> int run(uint16_t* hA, uint16_t* hB, float* hD) {
  uint16_t *dA, *dB; float* dD;
  cudaMalloc(&dA, S * 128 * 16 * 2); cudaMalloc(&dB, S * 256 * 16 * 2); cudaMalloc(&dD, 128 * 256 * 4);
  cudaMemcpy(dA, hA, S * 128 * 16 * 2, cudaMemcpyHostToDevice);
  cudaMemcpy(dB, hB, S * 256 * 16 * 2, cudaMemcpyHostToDevice);
  probe<S><<<1, 128>>>(dA, dB, dD);
  cudaError_t e = cudaDeviceSynchronize();
  cudaMemcpy(hD, dD, 128 * 256 * 4, cudaMemcpyDeviceToHost);
  cudaFree(dA); cudaFree(dB); cudaFree(dD);
  if (e != cudaSuccess) { printf("cuda error %s\n", cudaGetErrorString(e)); return 1; }
  return 0;
}

int main() {
  // ---- 1: one MMA against the CPU (small integers, exact) ----
  {
    static uint16_t hA[128 * 16], hB[256 * 16]; static float hD[128 * 256];
    for (int m = 0; m < 128; ++m) for (int k = 0; k < 16; ++k) hA[m * 16 + k] = bf((float)(((m * 7 + k * 3) % 17) - 8));
    for (int n = 0; n < 256; ++n) for (int k = 0; k < 16; ++k) hB[n * 16 + k] = bf((float)(((n * 5 + k * 11) % 13) - 6));
    if (run<1>(hA, hB, hD)) return 1;
    int bad = 0;
    for (int m = 0; m < 128; ++m) for (int n = 0; n < 256; ++n) {
      float s = 0; for (int k = 0; k < 16; ++k) s += fb(hA[m * 16 + k]) * fb(hB[n * 16 + k]);
      if (s != hD[m * 256 + n]) ++bad;
    }
    printf("single MMA 128x256x16 bf16->f32: %s (%d mismatches)\n", bad ? "MISMATCH" : "ok", bad);
    if (bad) return 1;
  }
  // ---- 2: rounding of the accumulator, diagonal tests D[t][t], 4 steps ----
  {
    const int S = 3;
    static uint16_t hA[S * 128 * 16], hB[S * 256 * 16]; static float hD[128 * 256];
    memset(hA, 0, sizeof hA); memset(hB, 0, sizeof hB);
    auto setA = [&](int s, int t, int k, float v) { hA[(s * 128 + t) * 16 + k] = bf(v); };
    auto setB = [&](int s, int t, int k, float v) { hB[(s * 256 + t) * 16 + k] = bf(v); };
    const float U = ldexpf(1.f, -23);  // ulp of 1
    // t0: 1 then +0.75ulp ; t1: +0.25ulp ; t2: +0.5ulp ; t3: (1+ulp) +0.5ulp ; t4: -1 -0.75ulp
    setA(0, 0, 0, 1); setB(0, 0, 0, 1); setA(1, 0, 0, 0.75f * U); setB(1, 0, 0, 1);
    setA(0, 1, 0, 1); setB(0, 1, 0, 1); setA(1, 1, 0, 0.25f * U); setB(1, 1, 0, 1);
    setA(0, 2, 0, 1); setB(0, 2, 0, 1); setA(1, 2, 0, 0.5f * U); setB(1, 2, 0, 1);
    setA(0, 3, 0, 1); setB(0, 3, 0, 1); setA(0, 3, 1, U); setB(0, 3, 1, 1); setA(1, 3, 0, 0.5f * U); setB(1, 3, 0, 1);
    setA(0, 4, 0, -1); setB(0, 4, 0, 1); setA(1, 4, 0, -0.75f * U); setB(1, 4, 0, 1);
    // t5: inside one MMA: 1 + 15 * 0.125ulp (exact 1 + 1.875 ulp)
    setA(0, 5, 0, 1); setB(0, 5, 0, 1); for (int k = 1; k < 16; ++k) { setA(0, 5, k, 0.125f * U); setB(0, 5, k, 1); }
    // t6: 2^20 - 2^20 + 2^-10 inside one MMA
    setA(0, 6, 0, 1048576.f); setB(0, 6, 0, 1); setA(0, 6, 1, -1048576.f); setB(0, 6, 1, 1); setA(0, 6, 2, ldexpf(1, -10)); setB(0, 6, 2, 1);
    // t7: 1 then three times +0.75ulp
    setA(0, 7, 0, 1); setB(0, 7, 0, 1); for (int s = 1; s < 3; ++s) { setA(s, 7, 0, 0.75f * U); setB(s, 7, 0, 1); }
    // t8: 1 then +0.75ulp split over two products inside one MMA (0.375 + 0.375)
    setA(0, 8, 0, 1); setB(0, 8, 0, 1); setA(1, 8, 0, 0.375f * U); setB(1, 8, 0, 1); setA(1, 8, 1, 0.375f * U); setB(1, 8, 1, 1);
    // t9: accumulator 1 + 3 ulp, add -0.75 ulp  (RN -> 1+2ulp, RZ -> 1+2ulp, RD...)
    setA(0, 9, 0, 1); setB(0, 9, 0, 1); setA(0, 9, 1, 3 * U); setB(0, 9, 1, 1); setA(1, 9, 0, -0.75f * U); setB(1, 9, 0, 1);
    // t10: accumulator 1, add -0.25 ulp (below 1: ulp halves) exact 1 - 2^-25 -> RN: 1-2^-24 ... 
    setA(0, 10, 0, 1); setB(0, 10, 0, 1); setA(1, 10, 0, -0.25f * U); setB(1, 10, 0, 1);
    if (run<S>(hA, hB, hD)) return 1;
    const char* names[] = {"1 + 0.75ulp", "1 + 0.25ulp", "1 + 0.5ulp (tie)", "(1+ulp) + 0.5ulp (tie)", "-1 - 0.75ulp",
                           "1 + 15*0.125ulp in one MMA", "2^20 - 2^20 + 2^-10 in one MMA", "1 + 2*(0.75ulp) over 2 MMAs",
                           "1 + (0.375+0.375)ulp in one MMA", "(1+3ulp) - 0.75ulp", "1 - 0.25ulp"};
    for (int t = 0; t < 11; ++t) {
      double v = hD[t * 256 + t];
      printf("t%-2d %-34s -> 1 + %.4f ulp   (raw %.10e)\n", t, names[t], (fabs(v) - 1.0) / U, v);
    }
  }
  return 0;
}
