// sm_100a building blocks: tensor-memory allocation, tcgen05 MMA / commit / load,
// shared-memory matrix descriptors and 3-D TMA tile loads.
#pragma once
#include <cuda.h>
#include <stdint.h>

#include "spx_common.cuh"

namespace spx {

#if defined(__CUDACC__)
__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(dst_smem)),
               "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Arrives on `bar` once every tcgen05 operation issued so far by this thread completes.
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

// D(tmem) (+)= A(smem desc) * B(smem desc)^T, int8 x int8 -> int32. `coll` selects the
// A-collector usage: 0 none, 1 fill, 2 use, 3 lastuse.
template <int COLL>
__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t da, uint64_t db, uint32_t idesc,
                                       uint32_t accumulate) {
  if constexpr (COLL == 1) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::i8.collector::a::fill [%0], %1, %2, %3, p;\n}\n" ::"r"(
            d_tmem),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
  } else if constexpr (COLL == 2) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::i8.collector::a::use [%0], %1, %2, %3, p;\n}\n" ::"r"(
            d_tmem),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
  } else if constexpr (COLL == 3) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::i8.collector::a::lastuse [%0], %1, %2, %3, p;\n}\n" ::"r"(
            d_tmem),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
  } else {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
  }
}

// ---- CTA-pair (cta_group::2) forms: one MMA spans the two SMs of a cluster of 2 ----
__device__ __forceinline__ uint32_t cluster_ctarank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cluster_id_x() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t nclusters_x() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%nclusterid.x;" : "=r"(r));
  return r;
}
__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\nbarrier.cluster.wait.acquire.aligned;" ::
                   : "memory");
}
// shared::cluster address of the same shared variable in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t mapa_shared(uint32_t saddr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(saddr), "r"(rank));
  return r;
}
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr)
               : "memory");
}
__device__ __forceinline__ void tmem_alloc2(uint32_t* dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(dst_smem)),
               "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
}
__device__ __forceinline__ void tmem_dealloc2(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}
// Arrives on the mbarrier at shared::cluster address `bar_cluster` (this CTA's or the
// peer's) once every cta_group::2 tcgen05 operation issued so far has completed.
__device__ __forceinline__ void tc_commit2(uint32_t bar_cluster) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          bar_cluster)
      : "memory");
}
template <int COLL>
__device__ __forceinline__ void mma2_i8(uint32_t d_tmem, uint64_t da, uint64_t db, uint32_t idesc,
                                        uint32_t accumulate) {
  if constexpr (COLL == 1) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::2.kind::i8.collector::a::fill [%0], %1, %2, %3, p;\n}\n" ::"r"(
            d_tmem),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
  } else if constexpr (COLL == 2) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::2.kind::i8.collector::a::use [%0], %1, %2, %3, p;\n}\n" ::"r"(
            d_tmem),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
  } else if constexpr (COLL == 3) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::2.kind::i8.collector::a::lastuse [%0], %1, %2, %3, p;\n}\n" ::"r"(
            d_tmem),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
  } else {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
  }
}
// 4-D TMA load of this CTA's part of a CTA-pair operand; completes on the
// mbarrier at shared::cluster address `bar_cluster` (the leader CTA's).
__device__ __forceinline__ void tma_load_4d_pair(void* dst, const CUtensorMap* map, int x, int y,
                                                 int z, int w, uint32_t bar_cluster) {
  asm volatile(
      "cp.async.bulk.tensor.4d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5, %6}], [%2];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(bar_cluster), "r"(x), "r"(y), "r"(z), "r"(w)
      : "memory");
}

// Pulls a 4-D tile into L2 ahead of its load (no shared memory, no completion).
__device__ __forceinline__ void tma_prefetch_4d(const CUtensorMap* map, int x, int y, int z,
                                                int w) {
  asm volatile("cp.async.bulk.prefetch.tensor.4d.L2.global.tile [%0, {%1, %2, %3, %4}];" ::"l"(map),
               "r"(x), "r"(y), "r"(z), "r"(w)
               : "memory");
}
// 16 consecutive 32-bit TMEM columns of this thread's lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, int32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}

// 32 consecutive 32-bit TMEM columns of this thread's lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, int32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// K-major operand descriptor for a SWIZZLE_32B tile of 32-byte rows:
// 8-row atoms of 256 B (SBO), version 1, layout type 6.
__device__ __forceinline__ uint64_t desc_sw32(const void* smem_tile) {
  const uint32_t a = smem_u32(smem_tile);
  uint64_t d = 0;
  d |= (uint64_t)((a >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;                  // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(256 >> 4) << 32;         // stride byte offset: next 8-row group
  d |= (uint64_t)1 << 46;                  // descriptor version for sm_100
  d |= (uint64_t)6 << 61;                  // SWIZZLE_32B
  return d;
}

// K-major operand descriptor for a SWIZZLE_64B tile of 64-byte rows: 8-row atoms
// of 512 B (SBO), version 1, layout type 4. The second 32-byte K step of a row is
// addressed by advancing the start address by 32 bytes inside the atom.
__device__ __forceinline__ uint64_t desc_sw64(const void* smem_tile) {
  const uint32_t a = smem_u32(smem_tile);
  uint64_t d = 0;
  d |= (uint64_t)((a >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;                  // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(512 >> 4) << 32;         // stride byte offset: next 8-row group
  d |= (uint64_t)1 << 46;                  // descriptor version for sm_100
  d |= (uint64_t)4 << 61;                  // SWIZZLE_64B
  return d;
}

// 3-D tiled TMA load into shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}
// 4-D tiled TMA load into shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            int w, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5, %6}], [%2];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z), "r"(w)
      : "memory");
}
__device__ __forceinline__ void named_bar_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}
#endif

// Host: a tiled tensor map of `rank` dims (dims[0] contiguous, strides[] the byte
// strides of dims 1..rank-1) without a context: 0, -1 (no driver entry), or the
// driver's error code.
int encode_tmap(CUtensorMap* map, CUtensorMapDataType type, int rank, const void* base,
                const uint64_t* dims, const uint64_t* strides, const uint32_t* box,
                CUtensorMapSwizzle swz);
// Host: builds a 3-D uint8 tiled tensor map (dims innermost first, byte strides of
// dims 1 and 2) through the driver entry point. Returns 0 on success.
int make_tmap_u8_3d(spx_ctx* ctx, CUtensorMap* map, const void* base, uint64_t d0, uint64_t d1,
                    uint64_t d2, uint64_t s1, uint64_t s2, uint32_t b0, uint32_t b1, uint32_t b2,
                    CUtensorMapSwizzle swz);
// Host: 4-D uint8 tiled tensor map; dims[0] is contiguous, strides[] are the byte
// strides of dims 1..3 (any order in memory).
int make_tmap_u8_4d(spx_ctx* ctx, CUtensorMap* map, const void* base, const uint64_t dims[4],
                    const uint64_t strides[3], const uint32_t box[4], CUtensorMapSwizzle swz);

}  // namespace spx
