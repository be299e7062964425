// gemm_tc.cu -- FP32 LU trailing update on the 5th-generation tensor cores.
//
// C (complex64, column-major) -= L21 * U12 for one panel step of the FP32 LU,
// with TF32 operands and FP32 accumulation in tensor memory.
//
// Complex as real GEMMs: the panel L21 (m x k complex) is viewed as a real
// matrix Lhat of 2m rows (row 2r = Re L(r,:), row 2r+1 = Im L(r,:)); U12 is
// split into U_re and U_im (k x n each).  Then
//   D1 = Lhat * U_re,   D2 = Lhat * U_im        (2m x n real, FP32)
//   Re C(r,j) -= D1(2r,j) - D2(2r+1,j),  Im C(r,j) -= D2(2r,j) + D1(2r+1,j).
// Both operands are packed K-major (64 FP32 per row, rounded to TF32) once
// per panel step: Lhat by k_pack_l21, U_re/U_im by the row-interchange +
// triangular-solve kernel.
//
// k_gemm_tc: persistent, one CTA per SM, 8 warps, one 64 x 128 complex tile
// of C at a time.  Warp 0 issues TMA loads (128-byte swizzle, no multicast)
// of the operands in 32-wide K chunks through a 3-stage ring, and L2
// prefetches of the C tiles a few tiles ahead.  Warp 1 allocates 512 TMEM
// columns and one elected thread issues tcgen05.mma (M=128, N=128, K=8,
// kind::tf32) into double-buffered accumulators.  Warps 4-7 read the
// accumulators with tcgen05.ld, combine real and imaginary parts with one
// lane shuffle, stage -(L21 U12) in shared memory per 64-column half and
// hand it to a TMA reduce-add (f32), so C is updated in L2 without ever
// being loaded into the SM: C = C + (-D) rounds exactly like C - D.  Every
// mbarrier wait is bounded; on timeout the kernel records ST_TIMEOUT and
// drains.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "bem_internal.h"

namespace bem {

namespace {

constexpr int kTcRows = 64;        // complex rows per tile (UMMA M = 128 real rows)
constexpr int kTcCols = 128;       // columns per tile (UMMA N)
constexpr uint32_t kChunk = 128 * 32 * 4;  // one operand box: 128 rows x 32 floats (K) = 16 KB
constexpr uint32_t kStageBytes = 3 * kChunk;  // Lhat, U_re, U_im for 32 of K
constexpr int kStages = 3;
constexpr uint32_t kHalfBytes = 128 * 64 * 4;  // C staging: 64 complex rows x 64 columns = 32 KB
constexpr uint32_t kTmemCols = 512;
constexpr int kPrefetch = 3;  // C tiles prefetched into L2 ahead of the current one
constexpr int kKPitch = 256;  // floats per packed operand row: K up to 256 (four 64-column panels)
constexpr size_t kTcSmem = (size_t)kStages * kStageBytes + 2 * kHalfBytes + 1024;

// Instruction descriptor, M = 128, N = 256: c_format F32 (bit 4), a/b format
// TF32 = 2 (bits 7, 10), K-major A and B, N >> 3 at bit 17, M >> 4 at bit
// 24.  U_re and U_im of a stage (128 rows each, adjacent in shared memory in
// the same swizzled K-major layout) form one 256-row B, so one MMA per K
// step writes both products into 256 accumulator columns (the U_re part in
// columns 0..127, the U_im part in 128..255).
__device__ __forceinline__ uint32_t idesc_tf32_128x256() {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(2 * kTcCols >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (SBO), version 1.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// L2 prefetch of one C tile (no shared memory, no completion to wait for).
__device__ __forceinline__ void tma_prefetch_3d(const CUtensorMap* map, int x, int y, int z) {
  asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];" ::"l"(map), "r"(x), "r"(y),
               "r"(z)
               : "memory");
}
// C += staged tile, the add done by the TMA unit at L2 (f32 add, the type of
// the tensor map).
__device__ __forceinline__ void tma_reduce_add_3d(const CUtensorMap* map, int x, int y, int z, const void* src) {
  asm volatile(
      "cp.reduce.async.bulk.tensor.3d.global.shared::cta.add.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(map),
      "r"(x), "r"(y), "r"(z), "r"(smem_u32(src))
      : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
__device__ __forceinline__ void tma_wait_read_1() { asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory"); }
__device__ __forceinline__ void tma_store_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void epi_bar_sync() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

__device__ __forceinline__ void umma_tf32(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

// 64 consecutive columns of this warp's 32 lanes (four x16 loads, no wait).
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float (&v)[64]) {
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr + 16u * q));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[16 * q + i] = __uint_as_float(r[i]);
  }
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

struct TcArgs {
  float2* A;        // the systems (complex64), problem b at A + b*bstride
  size_t lda, bstride;
  int nn, r0, c0, ncols, kw;
  int kbase;  // first K slot of the packed operands (a panel's own slot for a narrow update)
  int cend;         // columns >= cend are left unchanged
  int urow_off;     // packed U row of column c0
  int mtiles, ntiles, batch;
  int band;         // m-tiles per band of the tile order (see tile_of)
  int lrows;        // Lhat rows per problem (2*nn)
  int urows;        // U rows per problem (nn+1)
  int* status;
};

// Tile t of a launch -> (problem b, m-tile tm, n-tile tn).  Tiles run in
// bands of a.band m-tiles: every n-tile of one band before the next band, m
// fastest inside a band.  The band's rows of Lhat (a few MB) stay in L2 while
// all of U streams past them once per band; with m fastest over the whole
// height instead, a tall system's Lhat (74 MB at n = 36000) would be read
// from HBM again for every n-tile.
__device__ __forceinline__ void tile_of(int t, const TcArgs& a, int& b, int& tm, int& tn) {
  const int per = a.mtiles * a.ntiles;
  b = t / per;
  const int rem = t % per;
  const int bi = rem / (a.band * a.ntiles);
  const int r2 = rem - bi * a.band * a.ntiles;
  const int bm = min(a.band, a.mtiles - bi * a.band);
  tn = r2 / bm;
  tm = bi * a.band + r2 % bm;
}

// Non-blocking test of an mbarrier phase.
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Bounded wait; on timeout raise the kernel-wide abort flag and the status
// word.  A phase that has already completed is taken by one test, with no
// flag read and no suspend: the single MMA-issuing thread waits once per
// stage, and a blocking wait there cost a large share of the tensor pipe.
__device__ __forceinline__ bool wait_or_abort(uint64_t* bar, uint32_t parity, volatile int* abort_flag, int* status,
                                              unsigned long long limit_ns) {
  if (mbar_test(bar, parity)) return true;
  if (*abort_flag) return false;
  if (mbar_wait(bar, parity, limit_ns)) return true;
  *abort_flag = 1;
  atomicExch(&status[ST_TIMEOUT], 1);
  return false;
}

__global__ void __launch_bounds__(256, 1) k_gemm_tc(const __grid_constant__ CUtensorMap tm_l,
                                                    const __grid_constant__ CUtensorMap tm_ure,
                                                    const __grid_constant__ CUtensorMap tm_uim,
                                                    const __grid_constant__ CUtensorMap tm_c, TcArgs a) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* ring = smem;                                              // kStages x (Lhat, U_re, U_im) chunks
  float* stage_c = reinterpret_cast<float*>(smem + kStages * kStageBytes);  // 2 x [64 cols][128 floats]
  __shared__ uint64_t full[kStages], empty[kStages], t_full[2], t_empty[2];
  __shared__ uint32_t s_tmem;
  __shared__ int s_abort;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int total = a.mtiles * a.ntiles * a.batch;
  const int nchunks = (a.kw + 31) / 32;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int s = 0; s < 2; ++s) {
      mbar_init(&t_full[s], 1);
      mbar_init(&t_empty[s], 4);
    }
    s_abort = 0;
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  volatile int* abort_flag = &s_abort;
  const unsigned long long wlim = wait_limit(a.status);

  if (warp == 0 && lane == 0) {
    // ---- TMA producer: operand K-chunks through a kStages ring; C tiles
    //      kPrefetch ahead are prefetched into L2 for the reduce-adds ----
    auto prefetch_c = [&](int t) {
      if (t >= total) return;
      int b, tm, tn;
      tile_of(t, a, b, tm, tn);
      const int x = 2 * (a.r0 + tm * kTcRows), y = a.c0 + tn * kTcCols;
      tma_prefetch_3d(&tm_c, x, y, b);
      tma_prefetch_3d(&tm_c, x, y + 64, b);
    };
    for (int q = 0; q < kPrefetch; ++q) prefetch_c(blockIdx.x + q * gridDim.x);
    int s = 0;
    uint32_t ph = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < total && ok; t += gridDim.x) {
      prefetch_c(t + kPrefetch * gridDim.x);
      int b, tm, tn;
      tile_of(t, a, b, tm, tn);
      const int ly = b * a.lrows + 2 * tm * kTcRows;
      const int uy = b * a.urows + a.urow_off + tn * kTcCols;
      for (int h = 0; h < nchunks; ++h) {
        if (!wait_or_abort(&empty[s], ph ^ 1u, abort_flag, a.status, wlim)) {
          ok = false;
          break;
        }
        unsigned char* st = ring + (size_t)s * kStageBytes;
        mbar_expect_tx(&full[s], kStageBytes);
        tma_load_2d(st, &tm_l, a.kbase + 32 * h, ly, &full[s]);
        tma_load_2d(st + kChunk, &tm_ure, a.kbase + 32 * h, uy, &full[s]);
        tma_load_2d(st + 2 * kChunk, &tm_uim, a.kbase + 32 * h, uy, &full[s]);
        if (++s == kStages) {
          s = 0;
          ph ^= 1u;
        }
      }
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer ----
    // One thread issues every MMA of the CTA, so its instruction stream is
    // on the critical path: a K = 8 step of both products is 140 tensor
    // cycles, and building three descriptors per step from addresses took
    // about as long.  Descriptors are the stage-0 Lhat descriptor plus
    // constant offsets (the 14-bit start-address field holds addr >> 4 of a
    // shared window below 256 KB, so the adds never carry out of it).
    const uint32_t idesc = idesc_tf32_128x256();
    const uint64_t dbase = sdesc(smem_u32(ring));
    int s = 0;
    uint32_t ph = 0;
    int it = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < total && ok; t += gridDim.x, ++it) {
      const int buf = it & 1;
      if (!wait_or_abort(&t_empty[buf], ((uint32_t)(it >> 1) & 1u) ^ 1u, abort_flag, a.status, wlim)) break;
      tc_fence_after();
      const uint32_t d1 = tmem + (uint32_t)buf * 256u;
      for (int h = 0; h < nchunks; ++h) {
        if (!wait_or_abort(&full[s], ph, abort_flag, a.status, wlim)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint64_t da = dbase + (uint64_t)(((uint32_t)s * kStageBytes) >> 4);
        const uint64_t du = da + (kChunk >> 4);  // U_re then U_im: one N = 256 operand
        const int ks = min(4, (a.kw - 32 * h) / 8);
        const uint32_t acc0 = h > 0 ? 1u : 0u;
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
          if (kk < ks) {
            const uint64_t o = (uint64_t)(2 * kk);  // 32 bytes of K
            umma_tf32(d1, da + o, du + o, idesc, acc0 | (uint32_t)kk);
          }
        }
        umma_commit(&empty[s]);
        if (++s == kStages) {
          s = 0;
          ph ^= 1u;
        }
      }
      if (ok) umma_commit(&t_full[buf]);
    }
  } else if (warp >= 4) {
    // ---- epilogue: stage -(D) per 64-column half, reduce-add it into C ----
    const int e = warp - 4;
    const int rho = 32 * e + lane;  // real row in the tile = float index in the C column
    const int p = lane & 1;
    const bool issuer = (e == 0 && lane == 0);
    int it = 0;
    for (int t = blockIdx.x; t < total; t += gridDim.x, ++it) {
      const int buf = it & 1;
      if (!__all_sync(0xffffffffu, wait_or_abort(&t_full[buf], (uint32_t)(it >> 1) & 1u, abort_flag, a.status, wlim)))
        break;
      tc_fence_after();
      int b, tm, tn;
      tile_of(t, a, b, tm, tn);
      const uint32_t tbase = tmem + (uint32_t)buf * 256u + ((uint32_t)(32 * e) << 16);
      for (int hc = 0; hc < 2; ++hc) {
        float* ct = stage_c + (size_t)hc * (kHalfBytes / 4);
        // the half's 64 columns of both products in one go (one wait), while
        // this half's previous reduce may still be leaving shared memory
        float v1[64], v2[64];
        tmem_ld64(tbase + (uint32_t)(64 * hc), v1);
        tmem_ld64(tbase + 128u + (uint32_t)(64 * hc), v2);
        tmem_ld_wait();
        if (issuer) tma_wait_read_1();  // this half's previous reduce has left shared memory
        epi_bar_sync();
        {
          const int colbase = a.c0 + tn * kTcCols + 64 * hc;
#pragma unroll
          for (int i = 0; i < 64; ++i) {
            const float x = __shfl_xor_sync(0xffffffffu, v2[i], 1);
            const float val = p ? (v1[i] + x) : (v1[i] - x);
            ct[i * 128 + rho] = colbase + i < a.cend ? -val : 0.0f;
          }
        }
        if (hc == 1) {
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&t_empty[buf]);
        }
        fence_proxy_async();
        epi_bar_sync();
        if (issuer) tma_reduce_add_3d(&tm_c, 2 * (a.r0 + tm * kTcRows), a.c0 + tn * kTcCols + 64 * hc, b, ct);
      }
    }
    if (issuer) tma_store_wait_all();
  }
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

// ---------------------------------------------------------------------------
// k_gemm_tc2: the same update by CTA pairs (a cluster of 2 CTAs on one TPC,
// option "tc_pair").  A pair owns a 128-complex-row x 128-column tile of C:
// each CTA stages its own 64 complex rows of Lhat (128 real rows) and half of
// the tile's U columns (64 of U_re and U_im) per K chunk, the even CTA issues
// tcgen05.mma.cta_group::2 with M = 256, N = 128 (each CTA's tensor memory
// receives its own 128 real rows over all 128 columns) and each CTA's
// epilogue reduce-adds its own rows as in k_gemm_tc.  Per K chunk the pair
// reads 64 KB from L2 for a 128 x 128 complex tile where two single CTAs read
// 96 KB.  Protocol (no multicast load anywhere): every CTA loads into its own
// shared memory and the copies complete bytes of the even CTA's `full`
// barrier (cp.async.bulk.tensor.cta_group::2), which the even CTA alone
// arms; its MMA thread frees a stage in both CTAs with one multicast
// tcgen05.commit, signals both CTAs' accumulators full the same way, and
// waits until the four epilogue warps of both CTAs have arrived on its
// `t_empty`.  Tensor memory is allocated and freed by warp 1 of each CTA
// (cta_group::2).  Every wait is bounded.
// ---------------------------------------------------------------------------
constexpr uint32_t kHalfChunk = 64 * 32 * 4;           // U box of the pair: 64 rows x 32 floats = 8 KB
constexpr uint32_t kStage2Bytes = kChunk + 2 * kHalfChunk;  // 32 KB per CTA and stage
constexpr int kStages2 = 4;
constexpr size_t kTc2Smem = (size_t)kStages2 * kStage2Bytes + 2 * kHalfBytes + 1024;

__device__ __forceinline__ unsigned pair_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ void pair_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// Shared::cluster address of this CTA's variable p in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t pair_addr(const void* p, unsigned rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
  return r;
}
// TMA load into this CTA's shared memory whose completed bytes go to the
// mbarrier at shared::cluster address `bar` (the even CTA's).
__device__ __forceinline__ void tma_load_2d_pair(void* dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
      "[%4];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void umma_tf32_pair(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                               uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
// Arrives on the mbarrier at the same offset in both CTAs of the pair once the
// MMAs issued so far are complete.
__device__ __forceinline__ void umma_commit_pair(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
          smem_u32(bar)),
      "h"((unsigned short)0x3)
      : "memory");
}
__device__ __forceinline__ void mbar_arrive_remote(uint32_t bar) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(bar) : "memory");
}

__global__ void __launch_bounds__(256, 1) k_gemm_tc2(const __grid_constant__ CUtensorMap tm_l,
                                                     const __grid_constant__ CUtensorMap tm_ure,
                                                     const __grid_constant__ CUtensorMap tm_uim,
                                                     const __grid_constant__ CUtensorMap tm_c, TcArgs a) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* ring = smem;                                                 // kStages2 x (Lhat, U_re, U_im)
  float* stage_c = reinterpret_cast<float*>(smem + kStages2 * kStage2Bytes);  // 2 x [64 cols][128 floats]
  __shared__ uint64_t full[kStages2], empty[kStages2], t_full[2], t_empty[2];
  __shared__ uint32_t s_tmem;
  __shared__ int s_abort;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned rank = pair_rank();
  const bool even = rank == 0;
  const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
  const int total = a.mtiles * a.ntiles * a.batch;  // mtiles: 128-complex-row tiles here
  const int nchunks = (a.kw + 31) / 32;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages2; ++s) {
      mbar_init(&full[s], 1);   // the even CTA's expect_tx (bytes of both CTAs)
      mbar_init(&empty[s], 1);  // the multicast commit of the even CTA's MMA thread
    }
    for (int s = 0; s < 2; ++s) {
      mbar_init(&t_full[s], 1);   // multicast commit
      mbar_init(&t_empty[s], 8);  // the 4 epilogue warps of both CTAs (even CTA's copy)
    }
    s_abort = 0;
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  pair_sync();  // both CTAs' barriers are initialised before any remote arrival
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  volatile int* abort_flag = &s_abort;
  const unsigned long long wlim = wait_limit(a.status);
  const int tile_rows = 2 * kTcRows;  // complex rows per pair tile

  if (warp == 0 && lane == 0) {
    // ---- TMA producer of this CTA's operand halves (both CTAs) ----
    int s = 0;
    uint32_t ph = 0;
    bool ok = true;
    for (int t = pair; t < total && ok; t += npairs) {
      int b, tm, tn;
      tile_of(t, a, b, tm, tn);
      const int ly = b * a.lrows + 2 * (tm * tile_rows + (int)rank * kTcRows);
      const int uy = b * a.urows + a.urow_off + tn * kTcCols + (int)rank * (kTcCols / 2);
      for (int h = 0; h < nchunks; ++h) {
        if (!wait_or_abort(&empty[s], ph ^ 1u, abort_flag, a.status, wlim)) {
          ok = false;
          break;
        }
        unsigned char* st = ring + (size_t)s * kStage2Bytes;
        const uint32_t fb = pair_addr(&full[s], 0);
        if (even) mbar_expect_tx(&full[s], 2 * kStage2Bytes);
        tma_load_2d_pair(st, &tm_l, a.kbase + 32 * h, ly, fb);
        tma_load_2d_pair(st + kChunk, &tm_ure, a.kbase + 32 * h, uy, fb);
        tma_load_2d_pair(st + kChunk + kHalfChunk, &tm_uim, a.kbase + 32 * h, uy, fb);
        if (++s == kStages2) {
          s = 0;
          ph ^= 1u;
        }
      }
    }
  } else if (warp == 1 && lane == 0 && even) {
    // ---- MMA issuer of the pair ----
    // M = 256 (the pair's rows), N = 256: each CTA's 64 U_re and 64 U_im rows
    // of a stage are adjacent, so B is one 128-row operand per CTA and one
    // MMA per K step fills 256 accumulator columns: [U_re 0..63 | U_im 0..63]
    // from the even CTA's rows, then [U_re 64..127 | U_im 64..127].
    const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(2 * kTcCols >> 3) << 17) |
                           ((uint32_t)(256 >> 4) << 24);
    const uint64_t dbase = sdesc(smem_u32(ring));  // as in k_gemm_tc: constant offsets from one descriptor
    int s = 0;
    uint32_t ph = 0;
    int it = 0;
    bool ok = true;
    for (int t = pair; t < total && ok; t += npairs, ++it) {
      const int buf = it & 1;
      if (!wait_or_abort(&t_empty[buf], ((uint32_t)(it >> 1) & 1u) ^ 1u, abort_flag, a.status, wlim)) break;
      tc_fence_after();
      const uint32_t d1 = tmem + (uint32_t)buf * 256u;
      for (int h = 0; h < nchunks; ++h) {
        if (!wait_or_abort(&full[s], ph, abort_flag, a.status, wlim)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint64_t da = dbase + (uint64_t)(((uint32_t)s * kStage2Bytes) >> 4);
        const uint64_t du = da + (kChunk >> 4);
        const int ks = min(4, (a.kw - 32 * h) / 8);
        const uint32_t acc0 = h > 0 ? 1u : 0u;
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
          if (kk < ks) {
            const uint64_t o = (uint64_t)(2 * kk);
            umma_tf32_pair(d1, da + o, du + o, idesc, acc0 | (uint32_t)kk);
          }
        }
        umma_commit_pair(&empty[s]);
        if (++s == kStages2) {
          s = 0;
          ph ^= 1u;
        }
      }
      if (ok) umma_commit_pair(&t_full[buf]);
    }
  } else if (warp >= 4) {
    // ---- epilogue of this CTA's 64 complex rows (both CTAs) ----
    const int e = warp - 4;
    const int rho = 32 * e + lane;
    const int p = lane & 1;
    const bool issuer = (e == 0 && lane == 0);
    const uint32_t te0 = pair_addr(&t_empty[0], 0), te1 = pair_addr(&t_empty[1], 0);
    int it = 0;
    for (int t = pair; t < total; t += npairs, ++it) {
      const int buf = it & 1;
      if (!__all_sync(0xffffffffu, wait_or_abort(&t_full[buf], (uint32_t)(it >> 1) & 1u, abort_flag, a.status, wlim)))
        break;
      tc_fence_after();
      int b, tm, tn;
      tile_of(t, a, b, tm, tn);
      const int row0 = a.r0 + tm * tile_rows + (int)rank * kTcRows;  // this CTA's first complex row
      const uint32_t tbase = tmem + (uint32_t)buf * 256u + ((uint32_t)(32 * e) << 16);
      for (int hc = 0; hc < 2; ++hc) {
        float* ct = stage_c + (size_t)hc * (kHalfBytes / 4);
        // columns 64 hc .. 64 hc + 63 of the tile: the U_re part at
        // accumulator columns 128 hc.., the U_im part 64 further
        float v1[64], v2[64];
        tmem_ld64(tbase + (uint32_t)(128 * hc), v1);
        tmem_ld64(tbase + (uint32_t)(128 * hc + 64), v2);
        tmem_ld_wait();
        if (issuer) tma_wait_read_1();
        epi_bar_sync();
        {
          const int colbase = a.c0 + tn * kTcCols + 64 * hc;
#pragma unroll
          for (int i = 0; i < 64; ++i) {
            const float x = __shfl_xor_sync(0xffffffffu, v2[i], 1);
            const float val = p ? (v1[i] + x) : (v1[i] - x);
            ct[i * 128 + rho] = colbase + i < a.cend ? -val : 0.0f;
          }
        }
        if (hc == 1) {
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive_remote(buf ? te1 : te0);
        }
        fence_proxy_async();
        epi_bar_sync();
        if (issuer && row0 < a.nn) tma_reduce_add_3d(&tm_c, 2 * row0, a.c0 + tn * kTcCols + 64 * hc, b, ct);
      }
    }
    if (issuer) tma_store_wait_all();
  }
  __syncthreads();
  pair_sync();  // the pair's MMAs, commits and remote arrivals are all done
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

// Lhat: rows 2(r - r0) + p of problem b hold part p of L(r, k..k+kw-1),
// K-major at K slots koff..koff+kw-1 of a kKPitch-float row, rounded to TF32.
// With a gather list (a later panel's interchanges: count, then dst/src
// pairs), row r takes L from the row that the list moves to r, i.e. L in the
// later panel's row order; A itself is not changed.
// Panel z (blockIdx.z) of npanels consecutive 64-column panels: columns
// k + 64 z.., K slots koff + 64 z.., through problem b's row map z (at
// gmap + b * gstride + z * nn) when z < nmaps.
__global__ void __launch_bounds__(256) k_pack_l21(const float2* __restrict__ A, size_t lda, size_t bstride, int nn,
                                                  int k, int kw, int r0, int koff, float* lhat, int lrows,
                                                  const int* __restrict__ gmap, size_t gstride, int nmaps) {
  __shared__ float2 tile[64][33];
  __shared__ int s_src[32];
  const int b = blockIdx.y, z = blockIdx.z;
  const int* map = (gmap && z < nmaps) ? gmap + (size_t)b * gstride + (size_t)z * nn : nullptr;
  pack_l_rows(A + (size_t)b * bstride, lda, nn, k + 64 * z, kw, r0, r0 + blockIdx.x * 32, koff + 64 * z,
              lhat + (size_t)b * lrows * kKPitch, map, tile, s_src);
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// 2-D map over `rows` rows of kKPitch floats, 32 x box_rows boxes, 128B swizzle.
bool make_map(CUtensorMap* m, float* base, size_t rows, unsigned box_rows = 128) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {kKPitch, (cuuint64_t)rows};
  cuuint64_t strides[1] = {kKPitch * sizeof(float)};
  cuuint32_t box[2] = {32, box_rows};
  cuuint32_t estr[2] = {1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// 3-D map over the FP32 systems: floats of a column (2*nn, the rest of lda is
// padding), nn+1 columns, batch problems; 128 x 64 boxes (64 complex rows x
// 64 columns), no swizzle.
bool make_cmap(CUtensorMap* m, float2* base, int nn, size_t lda, size_t bstride, int batch) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[3] = {(cuuint64_t)2 * nn, (cuuint64_t)nn + 1, (cuuint64_t)batch};
  cuuint64_t strides[2] = {(cuuint64_t)lda * sizeof(float2), (cuuint64_t)bstride * sizeof(float2)};
  cuuint32_t box[3] = {128, 64, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

// 3-D map over the FP32 systems as 8-byte (complex) elements: nn rows, nn+1
// columns, batch problems; box_rows x 64 column boxes, no swizzle (the
// row shares of the triangular solves; rows past nn read as zero).
bool make_rows_map(CUtensorMap* m, const void* base, int nn, size_t lda, size_t bstride, int batch, int box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[3] = {(cuuint64_t)nn, (cuuint64_t)nn + 1, (cuuint64_t)batch};
  cuuint64_t strides[2] = {(cuuint64_t)lda * sizeof(float2), (cuuint64_t)bstride * sizeof(float2)};
  cuuint32_t box[3] = {(cuuint32_t)box_rows, 64, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void*>(base), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}


// tcgen05 kind::tf32 throughput: one elected thread per CTA issues `iters`
// x 4 MMAs (M=128, N=n, K=8) from zeroed shared-memory operands into one
// TMEM accumulator, then waits (bounded) for their completion.
__global__ void __launch_bounds__(128, 1) k_umma_peak(int iters, int n, int* status) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t abytes = kChunk, bbytes = (uint32_t)n * 128u;
  for (uint32_t i = threadIdx.x; i < (abytes + bbytes) / 16; i += blockDim.x)
    reinterpret_cast<uint4*>(smem)[i] = make_uint4(0, 0, 0, 0);
  __shared__ uint64_t done;
  __shared__ uint32_t s_tmem;
  const int warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) mbar_init(&done, 1);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(256)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  if (threadIdx.x == 0) {
    const uint32_t idesc =
        (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
    const uint32_t sa = smem_u32(smem), sb = sa + abytes;
    for (int it = 0; it < iters; ++it)
      for (int kk = 0; kk < 4; ++kk)
        umma_tf32(tmem, sdesc(sa + 32u * kk), sdesc(sb + 32u * kk), idesc, (it | kk) ? 1u : 0u);
    umma_commit(&done);
    if (!mbar_wait(&done, 0, wait_limit(status))) atomicExch(&status[ST_TIMEOUT], 1);
  }
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256) : "memory");
  }
}

int measure_tf32_peak(bem_ctx* ctx, int n, double* tflops) {
  if (n != 128 && n != 256) return fail(ctx, BEM_ERR_ARG, "UMMA peak probe: N must be 128 or 256");
  const size_t smem = kChunk + (size_t)n * 128 + 1024;
  BEM_CUDA(ctx, raise_smem_limit(reinterpret_cast<const void*>(k_umma_peak), smem));
  const int iters = 2048;
  cudaEvent_t e0, e1;
  BEM_CUDA(ctx, cudaEventCreate(&e0));
  BEM_CUDA(ctx, cudaEventCreate(&e1));
  k_umma_peak<<<ctx->num_sms, 128, smem, ctx->stream>>>(iters / 8, n, ctx->d_status);  // warm-up
  BEM_CUDA(ctx, cudaEventRecord(e0, ctx->stream));
  k_umma_peak<<<ctx->num_sms, 128, smem, ctx->stream>>>(iters, n, ctx->d_status);
  BEM_CUDA(ctx, cudaEventRecord(e1, ctx->stream));
  ctx->launches += 2;
  BEM_CUDA(ctx, cudaEventSynchronize(e1));
  float ms = 0.f;
  BEM_CUDA(ctx, cudaEventElapsedTime(&ms, e0, e1));
  *tflops = 2.0 * 128.0 * n * 8.0 * 4.0 * iters * ctx->num_sms / (ms * 1e-3) / 1e12;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return check_status(ctx);
}

int tc_ensure(bem_ctx* ctx, int nn, int batch) {
  TcWork& W = ctx->tc;
  const size_t lrows = (size_t)2 * nn * batch, urows = (size_t)(nn + 1) * batch;
  if (W.lhat && lrows <= W.lrows_cap && urows <= W.urows_cap) return BEM_OK;
  tc_release(ctx);
  BEM_CUDA(ctx, dev_alloc(ctx, &W.lhat, lrows * kKPitch * sizeof(float)));
  BEM_CUDA(ctx, dev_alloc(ctx, &W.ure, urows * kKPitch * sizeof(float)));
  BEM_CUDA(ctx, dev_alloc(ctx, &W.uim, urows * kKPitch * sizeof(float)));
  BEM_CUDA(ctx, cudaMemsetAsync(W.lhat, 0, lrows * kKPitch * sizeof(float), ctx->stream));
  BEM_CUDA(ctx, cudaMemsetAsync(W.ure, 0, urows * kKPitch * sizeof(float), ctx->stream));
  BEM_CUDA(ctx, cudaMemsetAsync(W.uim, 0, urows * kKPitch * sizeof(float), ctx->stream));
  // maps: 0 Lhat, 1-2 U_re/U_im (128-row boxes), 3 C (made per system), 4-5 U_re/U_im in
  // the 64-row boxes of the CTA-pair kernel
  W.maps = new CUtensorMap[6];
  CUtensorMap* maps = static_cast<CUtensorMap*>(W.maps);
  if (!make_map(&maps[0], W.lhat, lrows) || !make_map(&maps[1], W.ure, urows) || !make_map(&maps[2], W.uim, urows) ||
      !make_map(&maps[4], W.ure, urows, 64) || !make_map(&maps[5], W.uim, urows, 64))
    return fail(ctx, BEM_ERR_CUDA, "cuTensorMapEncodeTiled failed");
  W.lrows_cap = lrows;
  W.urows_cap = urows;
  BEM_CUDA(ctx, raise_smem_limit(reinterpret_cast<const void*>(k_gemm_tc), kTcSmem));
  BEM_CUDA(ctx, raise_smem_limit(reinterpret_cast<const void*>(k_gemm_tc2), kTc2Smem));
  return BEM_OK;
}

void tc_release(bem_ctx* ctx) {
  TcWork& W = ctx->tc;
  dev_free(ctx, W.lhat);
  dev_free(ctx, W.ure);
  dev_free(ctx, W.uim);
  delete[] static_cast<CUtensorMap*>(W.maps);
  W = TcWork{};
}

// Packs L (columns kcol..kcol+kw-1, rows r0..nn-1) into K slots
// koff..koff+kw-1 of Lhat, optionally through a row map (problem b's map at
// gmap + b * gstride: the storage row of L that is row r now); with npanels
// > 1, also the next 64-column panels into the next K slots in the same
// launch, the first nmaps of them through the maps that follow.
int tc_pack_l(bem_ctx* ctx, const float2* A, size_t lda, size_t bstride, int nn, int kcol, int kw, int r0, int koff,
              int batch, const int* gmap, size_t gstride, int npanels, int nmaps) {
  if (r0 >= nn) return BEM_OK;
  k_pack_l21<<<dim3((nn - r0 + 31) / 32, batch, npanels), 256, 0, ctx->stream>>>(
      A, lda, bstride, nn, kcol, kw, r0, koff, ctx->tc.lhat, 2 * nn, gmap, gstride, gmap ? nmaps : 0);
  ctx->launches++;
  BEM_CUDA(ctx, cudaGetLastError());
  return BEM_OK;
}

// C -= Lhat U for rows [r0, nn) and columns [c0, cend) of `batch` FP32
// systems, K = kw (packed Lhat and U_re/U_im; U row urow_off + (c - c0)).
int tc_gemm(bem_ctx* ctx, float2* A, size_t lda, size_t bstride, int nn, int r0, int c0, int cend, int kw,
            int urow_off, int batch, int kbase) {
  TcWork& W = ctx->tc;
  const int ncols = nn + 1;
  if (r0 >= nn || c0 >= cend) return BEM_OK;
  CUtensorMap* maps = static_cast<CUtensorMap*>(W.maps);
  if (W.cbase != A || W.clda != lda || W.cbstride != bstride || W.cbatch != batch) {
    if ((lda % 2) != 0 || (bstride % 2) != 0 || !make_cmap(&maps[3], A, nn, lda, bstride, batch))
      return fail(ctx, BEM_ERR_ARG, "tensor-core update needs an even leading dimension");
    W.cbase = A;
    W.clda = lda;
    W.cbstride = bstride;
    W.cbatch = batch;
  }
  TcArgs t{};
  t.A = A;
  t.lda = lda;
  t.bstride = bstride;
  t.nn = nn;
  t.r0 = r0;
  t.c0 = c0;
  t.ncols = ncols;
  t.kw = kw;
  t.kbase = kbase;
  t.cend = cend;
  t.urow_off = urow_off;
  t.mtiles = (nn - r0 + kTcRows - 1) / kTcRows;
  t.band = 48;  // 48 x 64 complex rows: 6 MB of Lhat at K = 256
  t.ntiles = (cend - c0 + kTcCols - 1) / kTcCols;
  t.batch = batch;
  t.lrows = 2 * nn;
  t.urows = nn + 1;
  t.status = ctx->d_status;
  const int ctas = ctx->gemm_ctas > 0 ? std::min(ctx->gemm_ctas, ctx->num_sms) : ctx->num_sms;
  if (ctx->tc_pair) {
    // CTA pairs: 128-complex-row tiles, as many pairs as can be resident at once
    t.mtiles = (nn - r0 + 2 * kTcRows - 1) / (2 * kTcRows);
    t.band = 24;  // 24 x 128 complex rows: 6 MB of Lhat at K = 256
    const int total = t.mtiles * t.ntiles * batch;
    if (W.pair_clusters == 0) {
      cudaLaunchConfig_t q = {};
      q.gridDim = dim3(2, 1, 1);
      q.blockDim = dim3(256, 1, 1);
      q.dynamicSmemBytes = kTc2Smem;
      cudaLaunchAttribute qa[1];
      qa[0].id = cudaLaunchAttributeClusterDimension;
      qa[0].val.clusterDim.x = 2;
      qa[0].val.clusterDim.y = 1;
      qa[0].val.clusterDim.z = 1;
      q.attrs = qa;
      q.numAttrs = 1;
      int n = 0;
      if (cudaOccupancyMaxActiveClusters(&n, k_gemm_tc2, &q) != cudaSuccess || n < 1) {
        cudaGetLastError();
        return fail(ctx, BEM_ERR_CUDA, "no resident CTA pair for the paired tensor-core update");
      }
      W.pair_clusters = n;
    }
    const int pairs = std::max(1, std::min({total, W.pair_clusters, ctas / 2}));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2 * pairs, 1, 1);
    cfg.blockDim = dim3(256, 1, 1);
    cfg.dynamicSmemBytes = kTc2Smem;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    BEM_CUDA(ctx, cudaLaunchKernelEx(&cfg, k_gemm_tc2, maps[0], maps[4], maps[5], maps[3], t));
    ctx->launches++;
    return BEM_OK;
  }
  const int total = t.mtiles * t.ntiles * batch;
  const int grid = std::min(total, ctas);
  k_gemm_tc<<<grid, 256, kTcSmem, ctx->stream>>>(maps[0], maps[1], maps[2], maps[3], t);
  ctx->launches++;
  BEM_CUDA(ctx, cudaGetLastError());
  return BEM_OK;
}

// One panel step: C -= L21 U12 for rows and columns from k + w on.
int tc_trailing_update(bem_ctx* ctx, float2* A, size_t lda, size_t bstride, int nn, int k, int w, int batch) {
  const int r0 = k + w;
  if (r0 >= nn) return BEM_OK;
  int rc = tc_pack_l(ctx, A, lda, bstride, nn, k, w, r0, 0, batch, nullptr, 0);
  if (rc) return rc;
  return tc_gemm(ctx, A, lda, bstride, nn, r0, r0, nn + 1, w, 0, batch, 0);
}

}  // namespace bem
